"""Node constructors ``inputs`` / ``multiply`` / ``summate`` and the block-size context.

Same signatures and semantics as the reference (src/pyjuice/nodes/construction.py:20-200).
"""

from __future__ import annotations

from typing import Callable, Optional, Sequence, Union

import torch

from .distributions import Distribution
from .input_nodes import InputNodes
from .nodes import CircuitNodes
from .prod_nodes import ProdNodes
from .sum_nodes import SumNodes


def inputs(var: Union[int, Sequence[int]], num_node_blocks: int = 0, dist: Distribution = None,
           params: Optional[torch.Tensor] = None, num_nodes: int = 0, block_size: int = 0, **kwargs) -> InputNodes:
    if block_size and block_size & (block_size - 1):
        raise ValueError("`block_size` must be a power of 2.")
    if num_nodes > 0:
        if num_node_blocks != 0:
            raise ValueError("Only one of `num_nodes` and `num_node_blocks` can be set.")
        if block_size == 0:
            block_size = CircuitNodes.DEFAULT_BLOCK_SIZE
        if num_nodes % block_size:
            raise ValueError("`num_nodes` must be divisible by `block_size`.")
        num_node_blocks = num_nodes // block_size
    if dist is None:
        raise ValueError("`dist` is required")
    return InputNodes(num_node_blocks=num_node_blocks, scope=[var] if isinstance(var, int) else list(var),
                      dist=dist, params=params, block_size=block_size, **kwargs)


def multiply(nodes1: CircuitNodes, *args, edge_ids: Optional[torch.Tensor] = None, sparse_edges: bool = False,
             **kwargs) -> ProdNodes:
    if not (nodes1.is_sum() or nodes1.is_input()):
        raise ValueError("Children of product nodes must be input or sum nodes.")
    chs = [nodes1]
    num_node_blocks = nodes1.num_node_blocks
    block_size = nodes1.block_size
    scope = nodes1.scope
    for ns in args:
        if not (ns.is_input() or ns.is_sum()):
            raise ValueError("Children of product nodes must be input or sum nodes.")
        if edge_ids is None and ns.num_node_blocks != num_node_blocks:
            raise ValueError("Input nodes should have the same `num_node_blocks`.")
        if ns.block_size != block_size:
            raise ValueError("Input nodes should have the same `block_size`.")
        if len(ns.scope & scope) != 0:
            raise ValueError("Children of a `ProdNodes` should have disjoint scopes.")
        chs.append(ns)
        scope = scope | ns.scope
    if edge_ids is not None:
        edge_ids = torch.as_tensor(edge_ids)
        if sparse_edges:
            if edge_ids.shape[0] % block_size:
                raise ValueError("sparse edge rows must be a multiple of block_size")
            num_node_blocks = edge_ids.shape[0] // block_size
        else:
            num_node_blocks = edge_ids.shape[0]
    return ProdNodes(num_node_blocks, chs, edge_ids, block_size=block_size, **kwargs)


def summate(nodes1: CircuitNodes, *args, num_node_blocks: int = 0, num_nodes: int = 0,
            edge_ids: Optional[torch.Tensor] = None, block_size: int = 0,
            sum_edge_ids_constructor: Optional[Callable] = None, **kwargs) -> SumNodes:
    if block_size and block_size & (block_size - 1):
        raise ValueError("`block_size` must be a power of 2.")
    if num_nodes > 0:
        if num_node_blocks != 0:
            raise ValueError("Only one of `num_nodes` and `num_node_blocks` can be set.")
        if block_size == 0:
            block_size = CircuitNodes.DEFAULT_BLOCK_SIZE
        if num_nodes % block_size:
            raise ValueError("`num_nodes` must be divisible by `block_size`.")
        num_node_blocks = num_nodes // block_size
    if not (nodes1.is_prod() or nodes1.is_input()):
        raise ValueError("Children of sum nodes must be input or product nodes.")
    if sum_edge_ids_constructor is not None:
        edge_ids = sum_edge_ids_constructor(nodes1, *args, num_node_blocks=num_node_blocks,
                                            block_size=block_size if block_size > 0 else CircuitNodes.DEFAULT_BLOCK_SIZE,
                                            **kwargs)
    if edge_ids is not None and not isinstance(edge_ids, (list, tuple)) and num_node_blocks == 0:
        num_node_blocks = int(torch.as_tensor(edge_ids)[0, :].max().item()) + 1
    if num_node_blocks <= 0:
        raise ValueError("Number of node blocks should be greater than 0.")
    chs = [nodes1]
    for ns in args:
        if not (ns.is_prod() or ns.is_input()):
            raise ValueError("Children of sum nodes must be input or product nodes.")
        if ns.scope != nodes1.scope:
            raise ValueError("Children of a `SumNodes` should have the same scope.")
        chs.append(ns)
    return SumNodes(num_node_blocks, chs, edge_ids, block_size=block_size, **kwargs)


class set_block_size:
    """Context manager (and decorator) setting the default block size of new nodes."""

    def __init__(self, block_size: int = 1):
        if block_size & (block_size - 1):
            raise ValueError("`block_size` must be a power of 2.")
        self.block_size = block_size
        self._saved = None

    def __enter__(self):
        self._saved = CircuitNodes.DEFAULT_BLOCK_SIZE
        CircuitNodes.DEFAULT_BLOCK_SIZE = self.block_size
        return self

    def __exit__(self, *exc):
        CircuitNodes.DEFAULT_BLOCK_SIZE = self._saved
        return False

    def __call__(self, fn):
        def wrapped(*a, **k):
            with set_block_size(self.block_size):
                return fn(*a, **k)
        return wrapped
