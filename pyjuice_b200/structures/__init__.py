from .hclt import HCLT, hclt_from_tree, chow_liu_tree, mutual_information, mutual_information_chunked
from .hmm import HMM, batched_hmms
from .pd import PD
