"""Sum node vectors (reference: src/pyjuice/nodes/sum_nodes.py:17).

``edge_ids`` is ``[2, num_edge_blocks]``: column ``[i, j]`` fully connects sum node
block ``i`` to child node block ``j`` (children of all ``chs`` concatenated).
``_params`` is ``[num_edge_blocks, block_size, ch_block_size]``.

The compiled layout of one vector's parameters in ``TensorCircuit.params`` (the
contract behind ``gather_parameters`` / ``update_parameters``, sum_nodes.py:280-347):
node blocks in order, and for node block ``g`` its child nodes ``k`` (in edge order)
each hold ``block_size`` consecutive entries, one per node of the block, i.e. the edge
block ``[ch_block_size, block_size]`` is stored transposed with the node index fastest.
"""

from __future__ import annotations

from typing import Optional, Sequence, Union

import numpy as np
import torch

from .nodes import CircuitNodes
from .prod_nodes import ProdNodes


def normalize_sum_params(params: torch.Tensor, node_ids: torch.Tensor, pseudocount: float = 0.0) -> None:
    """In place: each sum node's outgoing weights sum to one.

    ``params`` is ``[num_edge_blocks, block_size, ch_block_size]``; ``node_ids`` gives the
    sum-node block of each edge block. Follows the CPU branch of the reference's
    ``normalize_ns_parameters`` (src/pyjuice/nodes/backend/normalize.py:67-129): the
    per-node total is ``sum_children params + pseudocount`` and every weight becomes
    ``(w + pseudocount / nchs) / total``, with ``nchs`` the child-node count of the block.
    """
    num_blocks = int(node_ids.max().item()) + 1
    ch_bs = params.size(2)
    nchs = torch.bincount(node_ids, minlength=num_blocks).double() * ch_bs
    p64 = params.double()
    per_edge_block = p64.sum(dim=2)  # [E, bs]
    totals = torch.zeros([num_blocks, params.size(1)], dtype=torch.float64)
    totals.index_add_(0, node_ids, per_edge_block)
    totals = totals + pseudocount
    new = (p64 + pseudocount / nchs[node_ids][:, None, None]) / totals[node_ids][:, :, None]
    params.copy_(new.to(params.dtype))


class SumNodes(CircuitNodes):
    def __init__(self, num_node_blocks: int, chs: Sequence[CircuitNodes], edge_ids=None,
                 params: Optional[torch.Tensor] = None, zero_param_mask: Optional[torch.Tensor] = None,
                 block_size: int = 0, **kwargs):
        if len(chs) == 0:
            raise ValueError("`SumNodes` must have at least one child.")
        for i in range(1, len(chs)):
            if chs[0].block_size != chs[i].block_size:
                raise ValueError("`block_size` of the children of a `SumNodes` should be the same.")
        super().__init__(num_node_blocks, chs[0].scope, block_size=block_size, **kwargs)
        self.chs = self._standardize_chs(chs)
        self.num_ch_node_blocks = sum(c.num_node_blocks for c in self.chs)
        self.ch_block_size = self.chs[0].block_size
        self._construct_edges(edge_ids)
        self._zero_param_mask = None
        if zero_param_mask is not None:
            self.set_zero_param_mask(zero_param_mask)
        if params is not None:
            self.set_params(params, pseudocount=0.0)

    def is_sum(self):
        return True

    @property
    def num_edges(self):
        return self.edge_ids.size(1) * self.block_size * self.ch_block_size

    @property
    def num_ch_nodes(self):
        return self.num_ch_node_blocks * self.ch_block_size

    def duplicate(self, *args, tie_params: bool = False) -> "SumNodes":
        chs = list(args) if len(args) > 0 else self.chs
        params = None
        if self.provided("_params") and not tie_params:
            params = self._params.clone()
        return SumNodes(self.num_node_blocks, chs, self.edge_ids.clone(), params=params, block_size=self.block_size,
                        source_node=self if tie_params else None)

    def get_params(self, as_matrix: bool = False):
        if not as_matrix or self._params is None:
            return self._params
        nb, bs = self.num_node_blocks, self.block_size
        ncb, cbs = self.num_ch_node_blocks, self.ch_block_size
        full = torch.zeros([nb * ncb, bs, cbs], dtype=torch.float32)
        idxs = self.edge_ids[0, :] * ncb + self.edge_ids[1, :]
        full[idxs] = self._params
        return full.reshape(nb, ncb, bs, cbs).permute(0, 2, 1, 3).reshape(nb * bs, ncb * cbs)

    def set_params(self, params: torch.Tensor, normalize: bool = True, pseudocount: float = 0.0):
        if self._source_node is not None:
            return self._source_node.set_params(params, normalize=normalize, pseudocount=pseudocount)
        params = params.float()
        if params.dim() == 1:
            if not (self.block_size == 1 and self.ch_block_size == 1 and self.edge_ids.size(1) == params.size(0)):
                raise ValueError("1-D parameters need block sizes of 1.")
            self._params = params.clone().view(-1, 1, 1)
        elif params.dim() == 2:
            ncb = self.num_ch_node_blocks
            self._params = params.reshape(self.num_node_blocks, self.block_size, ncb, self.ch_block_size) \
                .permute(0, 2, 1, 3).flatten(0, 1)[self.edge_ids[0] * ncb + self.edge_ids[1]].contiguous()
        elif params.dim() == 3:
            self._params = params.clone()
        elif params.dim() == 4:
            self._params = params[self.edge_ids[0, :], self.edge_ids[1, :], :, :].clone().contiguous()
        else:
            raise ValueError("Unsupported parameter input.")
        if self._zero_param_mask is not None:
            self._params[self._zero_param_mask] = 0.0
        if normalize:
            normalize_sum_params(self._params, self.edge_ids[0, :], pseudocount=pseudocount)

    def set_zero_param_mask(self, zero_param_mask: Optional[torch.Tensor] = None):
        if zero_param_mask is None:
            return
        if self._source_node is not None:
            return self._source_node.set_zero_param_mask(zero_param_mask)
        if zero_param_mask.dtype != torch.bool or zero_param_mask.shape != (self.edge_ids.size(1), self.block_size, self.ch_block_size):
            raise ValueError("zero_param_mask must be a bool tensor of shape [num_edge_blocks, block_size, ch_block_size]")
        self._zero_param_mask = zero_param_mask

    def get_zero_param_mask(self):
        return self._zero_param_mask

    def init_parameters(self, perturbation: float = 2.0, recursive: bool = True, is_root: bool = True, **kwargs):
        if self._source_node is None:
            self._params = torch.exp(torch.rand([self.edge_ids.size(1), self.block_size, self.ch_block_size]) * -perturbation)
            if self._zero_param_mask is not None:
                self._params[self._zero_param_mask] = 0.0
            normalize_sum_params(self._params, self.edge_ids[0, :], pseudocount=0.0)
        if recursive:
            super().init_parameters(perturbation=perturbation, recursive=True, is_root=is_root, **kwargs)

    def update_parameters(self, params: torch.Tensor, clone: bool = True):
        """Copy this vector's slice of the compiled ``params`` back into ``_params``."""
        if not self.provided("_param_range"):
            raise RuntimeError("The `SumNodes` has not been compiled into a `TensorCircuit`.")
        if self.is_tied():
            return
        psid, peid = self._param_range
        p = params[psid:peid].detach().cpu()
        if clone:
            p = p.clone()
        local = (self._param_ids - psid) // (self.block_size * self.ch_block_size)
        p = p.reshape(-1, self.ch_block_size, self.block_size)
        self._params = p[local].permute(0, 2, 1).contiguous()

    def update_param_flows(self, param_flows: torch.Tensor, origin_ns_only: bool = True, clone: bool = True):
        if not self.provided("_param_flow_range"):
            raise RuntimeError("The `SumNodes` has not been compiled into a `TensorCircuit`.")
        if origin_ns_only and self.is_tied():
            return
        pfsid, pfeid = self._param_flow_range
        pf = param_flows[pfsid:pfeid].detach().cpu()
        if clone:
            pf = pf.clone()
        local = (self._param_flow_ids - pfsid) // (self.block_size * self.ch_block_size)
        pf = pf.reshape(-1, self.ch_block_size, self.block_size)
        self._param_flows = pf[local].permute(0, 2, 1).contiguous()

    def gather_parameters(self, params: torch.Tensor):
        """Write ``_params`` into this vector's slice of the compiled ``params``."""
        if not self.provided("_param_range"):
            raise RuntimeError("The `SumNodes` has not been compiled into a `TensorCircuit`.")
        if self.is_tied() or not self.has_params():
            return
        psid, peid = self._param_range
        flat = self._params[self._inverse_param_ids].permute(0, 2, 1).reshape(-1)
        params[psid:peid] = flat.to(params.device, params.dtype)

    def _standardize_chs(self, chs):
        out = []
        for cs in chs:
            if cs.is_input():
                out.append(ProdNodes(num_node_blocks=cs.num_node_blocks, chs=[cs],
                                     edge_ids=torch.arange(0, cs.num_node_blocks).reshape(-1, 1),
                                     block_size=cs.block_size))
            else:
                out.append(cs)
        return out

    def _construct_edges(self, edge_ids):
        if edge_ids is None:
            edge_ids = torch.stack((
                torch.arange(self.num_node_blocks).unsqueeze(1).repeat(1, self.num_ch_node_blocks).reshape(-1),
                torch.arange(self.num_ch_node_blocks).unsqueeze(0).repeat(self.num_node_blocks, 1).reshape(-1)), dim=0)
        elif isinstance(edge_ids, (list, tuple)):
            if len(edge_ids) != len(self.chs):
                raise ValueError("one edge tensor per child is required")
            parts, start = [], 0
            for cs_id, e in enumerate(edge_ids):
                e = torch.as_tensor(e).clone().long()
                e[1, :] += start
                start += self.chs[cs_id].num_node_blocks
                parts.append(e)
            edge_ids = torch.cat(parts, dim=1)
        if isinstance(edge_ids, np.ndarray):
            edge_ids = torch.from_numpy(edge_ids)
        if edge_ids.dtype == torch.bool:
            x, y = torch.where(edge_ids)
            edge_ids = torch.stack((x, y), dim=0)
        edge_ids = edge_ids.long()
        if edge_ids.dim() != 2 or edge_ids.size(0) != 2:
            raise ValueError("Expect `edge_ids.size(0) == 2`.")
        if not (torch.all(edge_ids >= 0) and torch.all(edge_ids[0] < self.num_node_blocks)
                and torch.all(edge_ids[1] < self.num_ch_node_blocks)):
            raise ValueError("Edge index out of range.")
        par = torch.unique(edge_ids[0, :])
        if par.numel() != self.num_node_blocks:
            raise ValueError("Some node has no edge.")
        self.edge_ids = edge_ids

    def __repr__(self):
        return (f"SumNodes(num_node_blocks={self.num_node_blocks}, block_size={self.block_size}, "
                f"num_chs={self.num_chs}, num_edges={self.num_edges})")
