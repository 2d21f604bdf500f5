"""Loader and thin Python binding of ``libpcb200.so`` (the C ABI in ``include/pcb200.h``).

The shared library is built in-tree by :func:`build` (nvcc, sm_100a) and loaded with
``ctypes``. Every call passes raw device pointers, sizes and the current CUDA stream;
a non-zero return status raises ``RuntimeError`` with the library's error message.
There is no fallback: if the library is missing or a tensor is not on a CUDA device,
the call fails.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_double, c_float, c_int32, c_int64, c_uint64, c_void_p

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpcb200.so")
CSRC = os.path.join(_HERE, "csrc")
SOURCES = ["capi_common.cu", "lse_contract.cu", "lse_contract_tc.cu", "lse_short.cu", "lse_tc05.cu", "prod_kernels.cu", "sum_pflows.cu",
           "sum_pflows_tc05.cu", "sum_generic.cu", "em_kernels.cu", "input_kernels.cu", "sample_kernels.cu", "sample_noalloc.cu",
           "input_soft.cu", "input_dists.cu", "input_poe.cu"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-shared",
              "-Xcompiler", "-fPIC"]

_lib = None


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile ``libpcb200.so`` for sm_100a if it is missing or older than its sources.

    Each source is compiled to its own object (in parallel, under ``_build/``; an object is
    rebuilt when it is older than its source or a shared header), then the objects are
    linked. The kernels of different files share no device symbols, so no relocatable
    device code is needed.
    """
    from concurrent.futures import ThreadPoolExecutor
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    headers.append(os.path.join(_HERE, "..", "include", "pcb200.h"))
    newest_header = max(os.path.getmtime(h) for h in headers if os.path.exists(h))
    if not force and os.path.exists(LIB_PATH):
        lib_m = os.path.getmtime(LIB_PATH)
        if all(os.path.getmtime(d) <= lib_m for d in srcs) and newest_header <= lib_m:
            return LIB_PATH
    bdir = os.path.join(_HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]

    def compile_one(src):
        obj = os.path.join(bdir, os.path.basename(src)[:-3] + ".o")
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header):
            return obj, None
        res = subprocess.run([_nvcc()] + compile_flags + ["-c", "-o", obj + ".tmp", src], capture_output=True, text=True)
        if res.returncode != 0:
            return obj, res.stdout + res.stderr
        os.replace(obj + ".tmp", obj)
        return obj, (res.stdout + res.stderr) if verbose else None

    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, srcs))
    errors = [msg for obj, msg in results if msg and not os.path.exists(obj)]
    if errors:
        raise RuntimeError("building libpcb200.so failed:\n" + "\n".join(errors))
    if verbose:
        for _, msg in results:
            if msg:
                print(msg)
    tmp = LIB_PATH + ".tmp"
    res = subprocess.run([_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp]
                         + [obj for obj, _ in results], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("linking libpcb200.so failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_SIGS = {
    "pcb_version": ([], c_int32),
    "pcb_last_error": ([], ctypes.c_char_p),
    "pcb_num_sms": ([], c_int32),
    "pcb_device_status": ([c_void_p, c_int32, c_void_p], c_int32),
    "pcb_status_selftest": ([c_int32, c_void_p], c_int32),
    "pcb_fill_rows": ([c_void_p, c_int64, c_int64, c_int64, c_float, c_void_p], c_int32),
    "pcb_input_cat_fwd": ([c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p,
                           c_int64, c_int32, c_void_p, c_int64, c_int64, c_void_p], c_int32),
    "pcb_input_cat_bwd": ([c_void_p, c_int64, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                           c_int32, c_int32, c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_int64, c_int64,
                           c_void_p, c_void_p, c_int32, c_void_p], c_int32),
    "pcb_input_cat_em": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double, c_double,
                          c_int32, c_void_p], c_int32),
    "pcb_input_dist_fwd": ([c_int32, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32,
                            c_void_p, c_int64, c_int32, c_void_p, c_int64, c_int64, c_void_p], c_int32),
    "pcb_input_dist_bwd": ([c_int32, c_void_p, c_int64, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p,
                            c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_int64, c_int64,
                            c_int32, c_void_p], c_int32),
    "pcb_input_dist_em": ([c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double,
                           c_double, c_void_p], c_int32),
    "pcb_input_poe_fwd": ([c_void_p, c_int64, c_void_p, c_void_p, c_int64, c_int64, c_int32, c_void_p, c_void_p,
                           c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_void_p,
                           c_int32, c_void_p, c_int64, c_int32, c_void_p, c_int64, c_int64, c_void_p], c_int32),
    "pcb_input_poe_evidence_bwd": ([c_void_p, c_int64, c_void_p, c_void_p, c_int64, c_int32, c_int32, c_void_p,
                                    c_void_p, c_int64, c_int64, c_int32, c_void_p, c_int64, c_int64, c_void_p,
                                    c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p,
                                    c_int32, c_void_p], c_int32),
    "pcb_pflow_accum": ([c_void_p, c_int64, c_int64, c_void_p, c_int32, c_void_p], c_int32),
    "pcb_prod_gather_sum": ([c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_int32,
                             c_int32, c_int32, c_int32, c_void_p], c_int32),
    "pcb_prod_gather_sum_modify": ([c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_int32, c_int32, c_void_p, c_void_p, c_void_p], c_int32),
    "pcb_lse_contract": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_int32,
                          c_int32, c_int32, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p], c_int32),
    "pcb_lse_contract_short": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p,
                                c_int32, c_int32, c_int32, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p,
                                c_int32, c_int32, c_void_p, c_void_p], c_int32),
    "pcb_pack_weights": ([c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_void_p], c_int32),
    "pcb_pack_weights_fp8": ([c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_void_p], c_int32),
    "pcb_pack_weights_multi": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p], c_int32),
    "pcb_lse_contract_tc05": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_int32,
                               c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p], c_int32),
    "pcb_lse_contract_tc05_accum": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p,
                                     c_int32, c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p], c_int32),
    "pcb_lse_levels_short": ([c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                              c_int32, c_int32, c_int32, c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p],
                             c_int32),
    "pcb_lse_contract_tc05_ws": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_int64, c_int64, c_void_p,
                                  c_void_p, c_int32, c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_void_p],
                                 c_int32),
    "pcb_sum_fwd_generic": ([c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_int32, c_int32, c_void_p,
                             c_void_p, c_int32, c_int32, c_float, c_void_p], c_int32),
    "pcb_sum_ele_generic": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_int32,
                             c_int32, c_void_p, c_void_p, c_int32, c_int32, c_float, c_int32, c_int32, c_void_p],
                            c_int32),
    "pcb_sum_par_generic": ([c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_int32,
                             c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p], c_int32),
    "pcb_modify_flows": ([c_void_p, c_void_p, c_int64, c_int32, c_int64, c_int64, c_void_p], c_int32),
    "pcb_sum_pflows": ([c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_int32,
                        c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p], c_int32),
    "pcb_sum_pflows_tc05": ([c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_int32,
                             c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p],
                            c_int32),
    "pcb_sum_pflows_tc05_tied": ([c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p,
                                  c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32,
                                  c_void_p, c_int32, c_void_p], c_int32),
    "pcb_sum_em": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double, c_double, c_int32,
                    c_void_p], c_int32),
    "pcb_sum_em_f64flows": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double,
                             c_double, c_int32, c_void_p], c_int32),
    "pcb_input_cat_em_f64flows": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double,
                                   c_double, c_int32, c_void_p], c_int32),
    "pcb_flows_accumulate_f64": ([c_void_p, c_void_p, c_int64, c_void_p], c_int32),
    "pcb_pflow_accum_f64": ([c_void_p, c_int64, c_int64, c_void_p, c_int32, c_void_p], c_int32),
    "pcb_sum_logit_grad": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double, c_void_p,
                            c_void_p], c_int32),
    "pcb_sum_softmax": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_void_p], c_int32),
    "pcb_input_cat_logit_grad": ([c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double,
                                  c_void_p, c_void_p], c_int32),
    "pcb_input_cat_soft_fwd": ([c_void_p, c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                c_int32, c_int32, c_void_p, c_int32, c_void_p, c_int64, c_int32, c_void_p, c_int64,
                                c_int64, c_void_p], c_int32),
    "pcb_input_cat_evidence_bwd": ([c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_int32,
                                    c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p], c_int32),
    "pcb_sum_normalize": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double, c_void_p], c_int32),
    "pcb_ll_sum_f64": ([c_void_p, c_int64, c_int32, c_int64, c_void_p, c_void_p], c_int32),
    "pcb_sample_sum": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32,
                        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                        c_uint64, c_void_p, c_void_p], c_int32),
    "pcb_sample_prod": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32,
                         c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int32),
    "pcb_sample_input": ([c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_void_p,
                          c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_uint64, c_void_p], c_int32),
    "pcb_sample_input_poe": ([c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_void_p,
                              c_void_p, c_void_p, c_int64, c_int64, c_int32, c_void_p, c_int64, c_void_p, c_int64,
                              c_uint64, c_void_p], c_int32),
    "pcb_sample_input_dist": ([c_int32, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_uint64, c_void_p], c_int32),
    "pcb_chunk_combine": ([c_void_p, c_int64, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_void_p],
                          c_int32),
    "pcb_sample_circuit_noalloc": ([c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_void_p, c_int64, c_uint64,
                                    c_void_p, c_void_p], c_int32),
}

EXPORTED_SYMBOLS = sorted(_SIGS.keys())


def load() -> ctypes.CDLL:
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run pyjuice_b200._native.build() (or __graft_entry__.build()) first")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


CALLS = 0  # number of entry-point calls (each launches at most one kernel)


def call(name: str, *args):
    global CALLS
    lib = load()
    CALLS += 1
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.pcb_last_error().decode(errors="replace")
        raise RuntimeError(f"{name} failed ({rc}): {msg}")
    return rc


class ShortFusion(ctypes.Structure):
    """PcbShortFusion (include/pcb200.h): a product layer fused into pcb_lse_contract_short."""
    _fields_ = [("term_children", c_void_p), ("element_out", c_void_p), ("out_children", c_void_p)]


def short_fusion(term_children=None, element_out=None, out_children=None):
    """Pointer to a PcbShortFusion built from device tensors (None when nothing is fused)."""
    if term_children is None and out_children is None:
        return c_void_p(0)
    return ctypes.pointer(ShortFusion(ptr(term_children), ptr(element_out), ptr(out_children)))


def ptr(t) -> c_void_p:
    """Device pointer of a CUDA tensor (None -> NULL)."""
    if t is None:
        return c_void_p(0)
    if not t.is_cuda:
        raise RuntimeError("pyjuice_b200 kernels need CUDA tensors (no CPU path)")
    return c_void_p(t.data_ptr())


def stream() -> c_void_p:
    return c_void_p(torch.cuda.current_stream().cuda_stream)


STATUS_BITS = {1: "a bounded device wait ran out", 2: "a contraction tile had more terms than the kernel handles",
               4: "an input value outside [0, num_cats)"}


def device_status(clear: bool = True) -> int:
    """OR of the fault bits the kernels reported on the current device since the last clear
    (``pcb_device_status``; waits for the current stream)."""
    out = c_int32(0)
    call("pcb_device_status", ctypes.byref(out), 1 if clear else 0, stream())
    return int(out.value)


def check_device_status(clear: bool = True) -> None:
    """Raise ``RuntimeError`` naming every fault bit that is set (see :func:`device_status`)."""
    st = device_status(clear)
    if st:
        what = "; ".join(msg for bit, msg in STATUS_BITS.items() if st & bit) or "unknown"
        raise RuntimeError(f"device status {st:#x}: {what}")
