from .layers import Layer, InputLayer, ProdLayer, SumLayer, LayerGroup
from .partition import partition_nodes_by_n_edges, next_power_of_2
