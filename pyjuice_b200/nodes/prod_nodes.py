"""Product node vectors (reference: src/pyjuice/nodes/prod_nodes.py:15).

``edge_ids`` is ``[num_node_blocks, num_chs]`` (block-sparse: block i uses block
``edge_ids[i, j]`` of child j) or ``[num_nodes, num_chs]`` (sparse: per node).
"""

from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from .nodes import CircuitNodes
from .scope import BitSet


class ProdNodes(CircuitNodes):
    SPARSE = 0
    BLOCK_SPARSE = 1

    def __init__(self, num_node_blocks: int, chs: Sequence[CircuitNodes], edge_ids: Optional[torch.Tensor] = None,
                 block_size: int = 0, **kwargs):
        scope = BitSet()
        for cs in chs:
            scope = scope | cs.scope
        super().__init__(num_node_blocks, scope, block_size=block_size, **kwargs)
        self.chs = list(chs)
        self._construct_edges(edge_ids)

    def is_prod(self):
        return True

    @property
    def num_edges(self):
        return self.num_nodes * self.num_chs

    @property
    def edge_type(self):
        if self.edge_ids.size(0) == self.num_node_blocks:
            return self.BLOCK_SPARSE
        if self.edge_ids.size(0) == self.num_nodes:
            return self.SPARSE
        raise RuntimeError(f"Unexpected shape of `edge_ids`: {tuple(self.edge_ids.shape)}")

    def is_block_sparse(self):
        return self.edge_type == self.BLOCK_SPARSE

    def is_sparse(self):
        return self.edge_type == self.SPARSE

    def duplicate(self, *args, tie_params: bool = False):
        chs = list(args) if len(args) > 0 else self.chs
        return ProdNodes(self.num_node_blocks, chs, self.edge_ids.clone(), block_size=self.block_size,
                         source_node=self if tie_params else None)

    def _construct_edges(self, edge_ids):
        if edge_ids is None:
            for c in self.chs:
                if c.num_node_blocks != self.num_node_blocks or c.block_size != self.block_size:
                    raise ValueError("Cannot create edges implicitly since # nodes do not match.")
            edge_ids = torch.arange(self.num_node_blocks).unsqueeze(1).repeat(1, self.num_chs)
        if isinstance(edge_ids, np.ndarray):
            edge_ids = torch.from_numpy(edge_ids)
        edge_ids = edge_ids.long()
        if edge_ids.dim() != 2 or edge_ids.size(1) != self.num_chs:
            raise ValueError(f"Expect edge_ids of shape (*, {self.num_chs}).")
        if edge_ids.size(0) == self.num_node_blocks:
            for cid in range(self.num_chs):
                if not (torch.all(edge_ids[:, cid] >= 0) and torch.all(edge_ids[:, cid] < self.chs[cid].num_node_blocks)):
                    raise ValueError("Edge index out of range.")
        elif edge_ids.size(0) == self.num_nodes:
            for cid in range(self.num_chs):
                if not (torch.all(edge_ids[:, cid] >= 0) and torch.all(edge_ids[:, cid] < self.chs[cid].num_nodes)):
                    raise ValueError("Edge index out of range.")
        else:
            raise ValueError(f"Unexpected shape of `edge_ids`: {tuple(edge_ids.shape)}")
        self.edge_ids = edge_ids

    def __repr__(self):
        kind = "sparse" if self.edge_type == self.SPARSE else "block_sparse"
        return f"ProdNodes(num_node_blocks={self.num_node_blocks}, block_size={self.block_size}, num_chs={self.num_chs}, edge_type='{kind}')"
