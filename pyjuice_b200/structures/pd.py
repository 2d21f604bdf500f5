"""Poon-Domingos structures over a grid of variables (src/pyjuice/structures/pd.py:17-220).

The root hypercube (the whole grid) is split recursively at fixed split points along every
axis; each split of a hypercube into two halves is a product of the halves' circuits, and
a hypercube's circuit is a sum over all its splits (at most ``max_prod_block_conns`` product
blocks per sum block, chosen by ``torch.rand`` when there are more). A hypercube without
split points becomes a sum over the product of its variables' input vectors. The root is
a single node (block size 1). Hypercubes are cached, so every hypercube has one circuit
(the "sum_dominated" structure) unless "prod_dominated" duplicates the halves per
product. The construction order, the random block choice and the node vectors follow the
reference exactly, so the same seed compiles to the same layout.
"""

from __future__ import annotations

from copy import deepcopy
from typing import Callable, Dict, Optional, Sequence, Tuple, Type, Union

import torch

from ..nodes import inputs, multiply, set_block_size, summate
from ..nodes.distributions import Categorical, Distribution
from ..nodes.scope import BitSet
from .hclt import _max_cdf_power_of_2


def PD(data_shape: Tuple, num_latents: int, split_intervals: Optional[Union[int, Tuple[int]]] = None,
       split_points: Optional[Sequence[Sequence[int]]] = None, max_split_depth: Optional[int] = None,
       max_prod_block_conns: int = 4, structure_type: str = "sum_dominated", input_ns_fn: Optional[Callable] = None,
       input_dist: Optional[Distribution] = None, input_node_type: Type[Distribution] = Categorical,
       input_node_params: Dict = {"num_cats": 256}, tie_homogeneous_params: bool = False,
       block_size: Optional[int] = None):
    if structure_type not in ("sum_dominated", "prod_dominated"):
        raise ValueError("structure_type must be 'sum_dominated' or 'prod_dominated'")
    if input_dist is not None:
        input_node_type, input_node_params = input_dist._get_constructor()
    if block_size is None:
        block_size = min(16 if num_latents <= 32 else 32, _max_cdf_power_of_2(num_latents))
    num_node_blocks = num_latents // block_size
    num_axes = len(data_shape)
    if split_intervals is not None:
        if isinstance(split_intervals, int):
            split_intervals = (split_intervals,) * num_axes
        split_points = [list(range(split_intervals[a], data_shape[a], split_intervals[a])) for a in range(num_axes)]
    else:
        if split_points is None or len(split_points) != num_axes:
            raise ValueError("give `split_intervals` or one list of `split_points` per axis")
        for a in range(num_axes):
            if not all(0 < x < data_shape[a] - 1 for x in split_points[a]):
                raise ValueError("split points must lie strictly inside every axis")
    sources = dict()
    cache = dict()

    def scope_of(cube):
        """Variables of a hypercube, numbered row-major over ``data_shape``."""
        lo, hi = cube
        vs = None
        stride = 1
        for a in range(num_axes - 1, -1, -1):
            r = torch.arange(lo[a], hi[a])
            vs = r if vs is None else (vs[None, :].repeat(hi[a] - lo[a], 1) + (r * stride)[:, None]).reshape(-1)
            stride *= data_shape[a]
        return BitSet.from_array(vs.tolist())

    def with_bound(cube, axis, s=None, e=None):
        lo, hi = list(cube[0]), list(cube[1])
        if s is not None:
            lo[axis] = s
        if e is not None:
            hi[axis] = e
        return tuple(lo), tuple(hi)

    def signature(cube, *chs):
        return tuple(cube[1][i] - cube[0][i] for i in range(num_axes)), tuple(len(ns.scope) for ns in chs)

    def tied_or_new(sig, make, chs):
        if not tie_homogeneous_params:
            return make()
        if sig in sources:
            return sources[sig].duplicate(*chs, tie_params=True)
        ns = make()
        sources[sig] = ns
        return ns

    def input_circuit(cube):
        scope = scope_of(cube)
        if input_ns_fn is not None:
            return input_ns_fn(scope, num_latents, block_size)
        leaves = []
        for v in scope:
            if tie_homogeneous_params and "input" in sources:
                leaves.append(sources["input"].duplicate(v, tie_params=True))
                continue
            ns = inputs(v, num_node_blocks=num_node_blocks, dist=input_node_type(**input_node_params))
            if tie_homogeneous_params:
                sources["input"] = ns
            leaves.append(ns)
        edge_ids = torch.arange(0, num_node_blocks)[None, :].repeat(2, 1)
        pns = multiply(*leaves)
        return tied_or_new(signature(cube, pns), lambda: summate(pns, num_node_blocks=num_node_blocks,
                                                                  edge_ids=edge_ids), [pns])

    def build(cube, depth=1):
        if cube in cache:
            return cache[cube]
        if max_split_depth is not None and depth > max_split_depth:
            cache[cube] = input_circuit(cube)
            return cache[cube]
        pns = []
        for a in range(num_axes):
            s, e = cube[0][a], cube[1][a]
            for sp in [p for p in global_points[a] if s < p < e]:
                left = build(with_bound(cube, a, e=sp))
                right = build(with_bound(cube, a, s=sp))
                pns.append(multiply(left, right) if structure_type == "sum_dominated" else
                           multiply(left.duplicate(), right.duplicate()))
        if not pns:
            ns = input_circuit(cube)
        elif cube == root_cube:
            ns = summate(*pns, num_node_blocks=1, block_size=1)
        elif len(pns) <= max_prod_block_conns:
            ns = tied_or_new(signature(cube, *pns), lambda: summate(*pns, num_node_blocks=num_node_blocks), pns)
        else:
            blocks = torch.topk(torch.rand([num_node_blocks, len(pns)]), k=max_prod_block_conns, dim=1).indices
            par = torch.arange(0, num_node_blocks)[:, None, None].repeat(1, max_prod_block_conns, num_node_blocks)
            chs = blocks[:, :, None] * num_node_blocks + torch.arange(0, num_node_blocks)[None, None, :]
            edge_ids = torch.stack((par.reshape(-1), chs.reshape(-1)), dim=0)
            ns = tied_or_new(signature(cube, *pns),
                             lambda: summate(*pns, num_node_blocks=num_node_blocks, edge_ids=edge_ids), pns)
        cache[cube] = ns
        return ns

    global_points = split_points
    with set_block_size(block_size=block_size):
        root_cube = ((0,) * num_axes, deepcopy(tuple(data_shape)))
        return build(root_cube)
