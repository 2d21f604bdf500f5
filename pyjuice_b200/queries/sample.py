"""Ancestral sampling on the device.

Same distribution as the reference's ``queries.sample`` (src/pyjuice/queries/sample.py:335-474):
walk the layer groups top-down from the root; a sum node picks one child with
probability equal to its weight, a product node activates all children, an input node
draws its category. Unlike the reference there is no host round trip per layer: each
sample carries its active node / element lists on the device
(``csrc/sample_kernels.cu``), and the uniforms are a counter-based hash of
``(seed, node id, sample index)``, so a given seed reproduces the samples bit for bit
(the CPU oracle restates the same draws).
"""

from __future__ import annotations

import random
from typing import Optional

import torch

from .. import _native as nat


def _scope_bounds(pc):
    """List capacities: #scopes over input+sum layer groups, max #scopes of a product group."""
    if hasattr(pc, "_num_nscopes") and hasattr(pc, "_num_escopes"):
        return pc._num_nscopes, pc._num_escopes
    n_scopes, e_scopes = 0, 0
    for group in pc.layers(ret_layer_groups=True):
        cur = sum(len(layer.scopes) for layer in group)
        if group.is_input() or group.is_sum():
            n_scopes += cur
        else:
            e_scopes = max(e_scopes, cur)
    pc._num_nscopes, pc._num_escopes = n_scopes, e_scopes
    return n_scopes, e_scopes


def sample(pc, num_samples: Optional[int] = None, conditional: bool = False, seed: Optional[int] = None,
           _sample_input_ns: bool = True, **kwargs) -> torch.Tensor:
    """Draw ``num_samples`` joint samples ``[num_samples, num_vars]`` (int64)."""
    if conditional:
        raise NotImplementedError("conditional sampling has no CUDA path yet")
    if num_samples is None or num_samples <= 0:
        raise ValueError("`num_samples` should be a positive integer.")
    if pc.num_root_nodes != 1:
        raise ValueError("It is ambiguous to sample from multi-head PCs.")
    if pc.device.type != "cuda":
        raise RuntimeError("sampling runs on CUDA only")
    if seed is None:
        seed = random.randint(0, 2 ** 62)
    dev = pc.device
    S = int(num_samples)
    cap_n, cap_e = _scope_bounds(pc)
    cap_n = max(cap_n, 1)
    cap_e = max(cap_e, 1)
    nlist = torch.zeros([S, cap_n], dtype=torch.int32, device=dev)
    nlist[:, 0] = pc._root_node_range[0]
    ncnt = torch.ones([S], dtype=torch.int32, device=dev)
    elist = torch.zeros([S, cap_e], dtype=torch.int32, device=dev)
    ecnt = torch.zeros([S], dtype=torch.int32, device=dev)
    err = torch.zeros([1], dtype=torch.int32, device=dev)
    st = nat.stream()
    for layer_id in range(len(pc.inner_layer_groups) - 1, -1, -1):
        group = pc.inner_layer_groups[layer_id]
        for layer in group:
            d = layer._desc(dev)
            if group.is_sum():
                lo, hi = layer._layer_nid_range
                nat.call("pcb_sample_sum", nat.ptr(nlist), nat.ptr(ncnt), nat.ptr(elist), nat.ptr(ecnt), S, cap_n,
                         cap_e, lo, hi, layer.block_size, nat.ptr(d["node2blk"]), nat.ptr(d["blk_nid"]),
                         nat.ptr(d["blk_koff"]), nat.ptr(d["blk_kcnt"]), nat.ptr(d["krow"]), nat.ptr(d["kw"]),
                         nat.ptr(pc.params), seed, nat.ptr(err), st)
            else:
                lo, hi = layer._layer_nid_range
                nat.call("pcb_sample_prod", nat.ptr(nlist), nat.ptr(ncnt), nat.ptr(elist), nat.ptr(ecnt), S, cap_n,
                         cap_e, lo, hi, nat.ptr(d["elem2blk"]), nat.ptr(d["fw_row"]), nat.ptr(d["fw_off"]),
                         nat.ptr(d["fw_cnt"]), nat.ptr(d["fw_chs"]), nat.ptr(err), st)
    if not _sample_input_ns:
        return nlist, ncnt
    samples = torch.zeros([S, pc.num_vars], dtype=torch.long, device=dev)
    for layer in pc.input_layer_group:
        d = layer._desc(dev)
        lo, hi = layer._output_ind_range
        nat.call("pcb_sample_input", nat.ptr(nlist), nat.ptr(ncnt), S, cap_n, lo, hi, nat.ptr(d["vids"]),
                 nat.ptr(d["s_pids"]), nat.ptr(d["ncats"]), nat.ptr(layer.params), nat.ptr(samples), pc.num_vars,
                 seed, st)
    e = int(err.item())
    if e != 0:
        raise RuntimeError(f"sampling failed on the device (code {e}: "
                           f"{'active list overflow' if e == 1 else 'element outside its product layer'})")
    return samples
