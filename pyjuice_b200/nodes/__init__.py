from .scope import BitSet
from .nodes import CircuitNodes, node_iterator
from .input_nodes import InputNodes
from .prod_nodes import ProdNodes
from .sum_nodes import SumNodes
from .construction import inputs, multiply, summate, set_block_size
from . import distributions
from .methods import get_subsumed_scopes
