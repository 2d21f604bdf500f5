"""Ancestral sampling on the device.

Same distribution as the reference's ``queries.sample`` (src/pyjuice/queries/sample.py:335-474):
walk the layer groups top-down from the root; a sum node picks one child with
probability equal to its weight, a product node activates all children, an input node
draws its category. Unlike the reference there is no host round trip per layer: each
sample carries its active node / element lists on the device
(``csrc/sample_kernels.cu``), and the uniforms are a counter-based hash of
``(seed, node id, sample index)``, so a given seed reproduces the samples bit for bit
(the CPU oracle restates the same draws), or come from a caller's table indexed by
(node id, sample index): given the uniform each of the reference's ``tl.rand`` draws
produced for a (node, sample) (sample.py:77 for sums, categorical.py:144 for inputs),
the device sampler returns the reference's samples exactly.
"""

from __future__ import annotations

import ctypes
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
           _sample_input_ns: bool = True, uniforms: Optional[torch.Tensor] = None, **kwargs) -> torch.Tensor:
    """Draw ``num_samples`` joint samples ``[num_samples, num_vars]`` (int64).

    ``uniforms``: optional ``[num_nodes, >= num_samples]`` FP32 table on the circuit's
    device; node ``n`` of sample ``s`` then draws with ``uniforms[n, s]`` instead of the
    seeded hash. With the draws the reference's ``tl.rand`` made for each (node, sample),
    the samples equal the reference's bit for bit.

    The result has the data type of the first input layer (int64 for Categorical, bool for
    Bernoulli, float32 for Gaussian and DiscreteLogistic; src/pyjuice/queries/sample.py:456-457).
    SoftEvidenceCategorical input layers draw from their categorical distribution times the
    evidence ``categorical_evidence_logp`` ``[num_samples, num_vars, K]`` (log-weights, dense),
    which such circuits need (softevi_categorical.py:196-222, 683-761).
    """
    if conditional:
        raise NotImplementedError("conditional sampling has no CUDA path yet")
    if num_samples is None or num_samples <= 0:
        raise ValueError("`num_samples` should be a positive integer.")
    if pc.num_root_nodes != 1:
        raise ValueError("It is ambiguous to sample from multi-head PCs.")
    if pc.device.type != "cuda":
        raise RuntimeError("sampling runs on CUDA only")
    evidence = kwargs.get("categorical_evidence_logp")
    for layer in pc.input_layer_group:
        kind = getattr(layer, "kind", 0)
        if kind == 4:
            if evidence is None:
                raise ValueError("sampling a SoftEvidenceCategorical layer needs `categorical_evidence_logp`")
            if (evidence.dtype != torch.float32 or evidence.dim() != 3 or evidence.size(0) != num_samples or
                    evidence.device != pc.device or evidence.stride(2) != 1 or
                    evidence.size(1) < layer._desc(pc.device)["num_layer_vars"] or
                    evidence.size(2) > layer._desc(pc.device)["min_ncats"]):
                raise ValueError("`categorical_evidence_logp` must be a float32 [num_samples, num_vars, K <= num_cats] "
                                 "tensor on the circuit's device, contiguous over categories")
        elif kind not in (0, 1, 2, 3):
            raise NotImplementedError(f"the device sampler has no draw for input layer kind {kind}")
    if seed is None:
        seed = random.randint(0, 2 ** 62)
    dev = pc.device
    S = int(num_samples)
    u_ld = 0
    if uniforms is not None:
        if (uniforms.dtype != torch.float32 or uniforms.dim() != 2 or uniforms.size(0) < pc.num_nodes
                or uniforms.size(1) < S or uniforms.stride(1) != 1 or uniforms.device != dev):
            raise ValueError("`uniforms` must be a row-major float32 [num_nodes, >= num_samples] tensor on "
                             f"the circuit's device {dev}")
        u_ld = uniforms.stride(0)
    with torch.cuda.device(dev):
        return _sample_on_device(pc, S, seed, uniforms, u_ld, _sample_input_ns, evidence)


def _sample_on_device(pc, S, seed, uniforms, u_ld, _sample_input_ns, evidence=None):
    dev = pc.device
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
                         nat.ptr(pc.params), nat.ptr(uniforms), u_ld, seed, nat.ptr(err), st)
            else:
                lo, hi = layer._layer_nid_range
                nat.call("pcb_sample_prod", nat.ptr(nlist), nat.ptr(ncnt), nat.ptr(elist), nat.ptr(ecnt), S, cap_n,
                         cap_e, lo, hi, nat.ptr(d["elem2blk"]), nat.ptr(d["fw_row"]), nat.ptr(d["fw_off"]),
                         nat.ptr(d["fw_cnt"]), nat.ptr(d["fw_chs"]), nat.ptr(err), st)
    if not _sample_input_ns:
        return nlist, ncnt
    samples = torch.zeros([S, pc.num_vars], dtype=torch.long, device=dev)
    fsamples, fvars = None, []  # values of Bernoulli / Gaussian / DiscreteLogistic layers (FP32)
    for layer in pc.input_layer_group:
        d = layer._desc(dev)
        lo, hi = layer._output_ind_range
        if getattr(layer, "kind", 0) in (1, 2, 3):
            if fsamples is None:
                fsamples = torch.zeros([S, pc.num_vars], dtype=torch.float32, device=dev)
            nat.call("pcb_sample_input_dist", layer.kind, nat.ptr(nlist), nat.ptr(ncnt), S, cap_n, lo, hi,
                     nat.ptr(d["vids"]), nat.ptr(d["s_pids"]), nat.ptr(d["node_meta"]), nat.ptr(layer.params),
                     nat.ptr(fsamples), pc.num_vars, nat.ptr(uniforms), u_ld, seed, st)
            fvars.append(d["vids"].long())
            continue
        if getattr(layer, "kind", 0) == 4:
            nat.call("pcb_sample_input_poe", nat.ptr(nlist), nat.ptr(ncnt), S, cap_n, lo, hi, nat.ptr(d["vids"]),
                     nat.ptr(d["s_pids"]), nat.ptr(d["node_lvid"]), nat.ptr(layer.params), nat.ptr(evidence),
                     evidence.stride(0), evidence.stride(1), evidence.size(2), nat.ptr(samples), pc.num_vars,
                     nat.ptr(uniforms), u_ld, seed, st)
            continue
        nat.call("pcb_sample_input", nat.ptr(nlist), nat.ptr(ncnt), S, cap_n, lo, hi, nat.ptr(d["vids"]),
                 nat.ptr(d["s_pids"]), nat.ptr(d["ncats"]), nat.ptr(layer.params), nat.ptr(samples), pc.num_vars,
                 nat.ptr(uniforms), u_ld, seed, st)
    e = int(err.item())
    if e != 0:
        raise RuntimeError(f"sampling failed on the device (code {e}: "
                           f"{'active list overflow' if e == 1 else 'element outside its product layer'})")
    dtype = pc.input_layer_group[0].get_data_dtype()
    if fsamples is None:
        return samples if dtype == torch.long else samples.to(dtype)
    out = samples.to(dtype)
    cols = torch.unique(torch.cat(fvars))
    out[:, cols] = fsamples[:, cols].to(dtype)
    return out


class _SampleStep(ctypes.Structure):
    """Mirror of ``PcbSampleStep`` (include/pcb200.h)."""
    _fields_ = [("kind", ctypes.c_int32), ("lo", ctypes.c_int32), ("hi", ctypes.c_int32), ("bs", ctypes.c_int32),
                ("node2blk", ctypes.c_void_p), ("blk_first", ctypes.c_void_p), ("blk_off", ctypes.c_void_p),
                ("blk_cnt", ctypes.c_void_p), ("children", ctypes.c_void_p), ("weight_base", ctypes.c_void_p),
                ("params", ctypes.c_void_p), ("vids", ctypes.c_void_p), ("s_pids", ctypes.c_void_p),
                ("ncats", ctypes.c_void_p)]


def noalloc_sample_plan(pc):
    """Step table for ``pcb_sample_circuit_noalloc``: ``(table, num_steps, root_id, cap_n, cap_e)``.

    Building the plan allocates (the table is copied to the device once); the calls that
    use it do not. The table holds raw pointers to the circuit's index tables and
    parameters, so it is valid while ``pc`` keeps those tensors; it is cached on ``pc``
    and rebuilt when a parameter tensor moves.
    """
    if pc.num_root_nodes != 1:
        raise ValueError("It is ambiguous to sample from multi-head PCs.")
    if pc.device.type != "cuda":
        raise RuntimeError("sampling runs on CUDA only")
    if any(getattr(layer, "kind", 0) != 0 for layer in pc.input_layer_group):
        raise NotImplementedError("the allocation-free sampler draws Categorical inputs only")
    dev = pc.device
    key = (str(dev), pc.params.data_ptr(), tuple(layer.params.data_ptr() for layer in pc.input_layer_group))
    cached = getattr(pc, "_noalloc_sample_plan", None)
    if cached is not None and cached[0] == key:
        return cached[1]
    steps = []
    for layer_id in range(len(pc.inner_layer_groups) - 1, -1, -1):
        group = pc.inner_layer_groups[layer_id]
        for layer in group:
            d = layer._desc(dev)
            lo, hi = layer._layer_nid_range
            if group.is_sum():
                steps.append(_SampleStep(0, lo, hi, layer.block_size, d["node2blk"].data_ptr(),
                                         d["blk_nid"].data_ptr(), d["blk_koff"].data_ptr(), d["blk_kcnt"].data_ptr(),
                                         d["krow"].data_ptr(), d["kw"].data_ptr(), pc.params.data_ptr(), None, None,
                                         None))
            else:
                steps.append(_SampleStep(1, lo, hi, 1, d["elem2blk"].data_ptr(), d["fw_row"].data_ptr(),
                                         d["fw_off"].data_ptr(), d["fw_cnt"].data_ptr(), d["fw_chs"].data_ptr(),
                                         None, None, None, None, None))
    for layer in pc.input_layer_group:
        d = layer._desc(dev)
        lo, hi = layer._output_ind_range
        steps.append(_SampleStep(2, lo, hi, 1, None, None, None, None, None, None, layer.params.data_ptr(),
                                 d["vids"].data_ptr(), d["s_pids"].data_ptr(), d["ncats"].data_ptr()))
    arr = (_SampleStep * len(steps))(*steps)
    table = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(dev)
    cap_n, cap_e = _scope_bounds(pc)
    plan = (table, len(steps), int(pc._root_node_range[0]), max(cap_n, 1), max(cap_e, 1))
    pc._noalloc_sample_plan = (key, plan)
    return plan


def sample_noalloc(pc, samples: torch.Tensor, err: torch.Tensor, seed: int, plan=None) -> None:
    """Fill ``samples`` ([S, num_vars] int64, caller-allocated) without any device allocation.

    Same draws as :func:`sample` with the same ``seed``. ``err`` (one int32 on the device)
    receives 0, or 1 on list overflow, 2 on an element outside its product layer, 3 on a
    malformed step table; the call does not synchronise, so read it when the stream reaches that point. Variables a
    sample does not draw keep their value in ``samples``. At most
    ``PCB_SAMPLE_NOALLOC_MAX_INTS // (cap_n + cap_e)`` samples per call; calls that
    overlap in time on one device share the library's working lists and must be
    serialised. For callers that cannot allocate when they sample (a pre-reserved memory
    pool, a plugin inside another framework's allocator).
    """
    if plan is None:
        plan = noalloc_sample_plan(pc)
    table, num_steps, root_id, cap_n, cap_e = plan
    if samples.dtype != torch.long or samples.dim() != 2 or samples.stride(1) != 1:
        raise ValueError("`samples` must be a row-major int64 tensor [S, num_vars]")
    if samples.size(1) < pc.num_vars or samples.stride(0) < pc.num_vars:
        raise ValueError(f"`samples` must have at least num_vars = {pc.num_vars} columns")
    if samples.size(0) >= 2 ** 31:
        raise ValueError("at most 2^31 - 1 samples per call")
    if err.dtype != torch.int32 or err.numel() < 1:
        raise ValueError("`err` must hold one int32")
    if samples.device != pc.device or err.device != pc.device:
        raise ValueError(f"`samples` and `err` must be on the circuit's device {pc.device}")
    # the kernel runs on the current device: make it the one that holds the tables
    with torch.cuda.device(pc.device):
        nat.call("pcb_sample_circuit_noalloc", nat.ptr(table), num_steps, root_id, samples.size(0), cap_n, cap_e,
                 nat.ptr(samples), samples.stride(0), int(seed), nat.ptr(err), nat.stream())
