"""Import shim that runs the reference PyJuice on CPU (fixture generation only).

Used by ``make_golden.py`` in a container that holds the reference sources; nothing in
the test suite, ``__graft_entry__`` or ``bench.py`` imports it. The reference needs
CUDA; on CPU it runs through Triton's interpreter (``TRITON_INTERPRET=1``) once its
``.cuda()`` calls and device checks are neutralised and matplotlib (used only by its
plotting module) is stubbed. Its FP32 path (``force_use_fp32=True``) is exact under
the interpreter; its BF16 ``tl.dot`` path is not used.
"""

from __future__ import annotations

import contextlib
import os
import sys
import tempfile
import types



def _ref_src() -> str:
    """Source directory of the reference package (``PYJUICE_REF_SRC``, required)."""
    src = os.environ.get("PYJUICE_REF_SRC")
    if not src or not os.path.isdir(os.path.join(src, "pyjuice")):
        raise RuntimeError("set PYJUICE_REF_SRC to the reference's `src` directory (the one holding `pyjuice/`)")
    return src


def load_reference():
    os.environ["TRITON_INTERPRET"] = "1"
    stub = tempfile.mkdtemp(prefix="mplstub_")
    os.makedirs(os.path.join(stub, "matplotlib"), exist_ok=True)
    with open(os.path.join(stub, "matplotlib", "__init__.py"), "w") as f:
        f.write("")
    with open(os.path.join(stub, "matplotlib", "pyplot.py"), "w") as f:
        f.write("")
    sys.path.insert(0, stub)
    sys.path.insert(0, _ref_src())

    import torch

    torch.Tensor.cuda = lambda self, *a, **k: self
    torch.cuda.current_device = lambda: 0

    @contextlib.contextmanager
    def _nodev(*a, **k):
        yield

    torch.cuda.device = _nodev

    # libdevice calls have no interpreter implementation: log1p(x) becomes log(1 + x), ceil
    # the language's ceil
    # (the log-space flow kernels use it; the difference is within FP32 rounding)
    import triton.language as tl
    libdev = getattr(tl.extra.cuda, "libdevice", None)
    if libdev is not None:
        libdev.log1p = lambda x, *a, **k: tl.log(x + 1.0)
        libdev.ceil = lambda x, *a, **k: tl.ceil(x)

    import pyjuice as juice
    from pyjuice.layer import input_layer as il

    class _FakeCuda:
        type = "cuda"
        index = None

        def __str__(self):
            return "cpu"

    fake = _FakeCuda()

    def _map_dev(kw):
        if kw.get("device", None) is fake:
            kw["device"] = "cpu"
        return kw

    def _wrap_factory(fn):
        def w(*a, **kw):
            return fn(*a, **_map_dev(kw))
        return w

    for name in ("tensor", "zeros", "empty", "ones", "full", "arange", "zeros_like"):
        setattr(torch, name, _wrap_factory(getattr(torch, name)))
    _orig_to = torch.Tensor.to

    def _to(self, *a, **kw):
        if a and a[0] is fake:
            a = ("cpu",) + a[1:]
        return _orig_to(self, *a, **_map_dev(kw))

    torch.Tensor.to = _to

    def _wrap_method(name):
        orig = getattr(il.InputLayer, name)

        def w(self, *a, **kw):
            saved = self.device
            self.device = fake
            try:
                return orig(self, *a, **kw)
            finally:
                self.device = saved
        setattr(il.InputLayer, name, w)

    for name in ("forward", "backward", "mini_batch_em", "sample"):
        _wrap_method(name)
    return juice


def install_uniform_table(juice, table):
    """Make the reference's sampler draw ``table[node id, sample]`` (a float32 numpy array
    ``[num_nodes, S]``) wherever it calls ``tl.rand``.

    The reference draws ``tl.rand(seed, offset)`` where ``offset`` indexes the list of
    (node, sample) pairs a launch processes: for sum layers the pairs of
    ``torch.where`` over ``node_samples`` (queries/sample.py:77, list built at 418), for
    input layers the pairs of ``torch.where(node_flows > 1e-8)`` (input_layer.py:592,
    categorical.py:144). The launchers are wrapped to record each launch's pair list, and
    ``triton.language.rand`` is replaced by a lookup of the table through that list, so
    every draw is a known function of the node and the sample.
    """
    import numpy as np
    import torch
    import triton.language as tl
    from triton.runtime.interpreter import TensorHandle
    import pyjuice.queries  # noqa: F401  (the package re-exports the function `sample`)
    from pyjuice.layer import input_layer as il
    qs = sys.modules["pyjuice.queries.sample"]

    ctx = {"nodes": None, "samples": None}

    def rand(seed, offset, *a, **k):
        off = np.asarray(offset.handle.data).astype(np.int64).reshape(-1)
        nodes, samples = ctx["nodes"], ctx["samples"]
        ok = off < nodes.shape[0]
        o = np.where(ok, off, 0)
        vals = np.where(ok, table[nodes[o], samples[o]], 0.0).astype(np.float32)
        shape = list(offset.type.shape) if offset.type.is_block() else []
        ty = tl.core.block_type(tl.float32, shape) if shape else tl.float32
        return tl.core.tensor(TensorHandle(vals.reshape(shape) if shape else vals.reshape(()), tl.float32), ty)

    tl.rand = rand
    orig_sum = qs.sample_sum_layer

    def sample_sum_layer(pc, layer, nids, cids, pids, node_mars, element_mars, params, node_samples,
                         element_samples, ind_target, ind_n, ind_b, *a, **k):
        ctx["nodes"] = node_samples[ind_n, ind_b].numpy().astype(np.int64)
        ctx["samples"] = ind_b.numpy().astype(np.int64)
        return orig_sum(pc, layer, nids, cids, pids, node_mars, element_mars, params, node_samples,
                        element_samples, ind_target, ind_n, ind_b, *a, **k)

    qs.sample_sum_layer = sample_sum_layer
    orig_in = il.InputLayer.sample

    def in_sample(self, samples, node_flows, *a, **k):
        sid, eid = self._output_ind_range
        xs, ys = torch.where(node_flows[sid:eid, :] > 1e-8)
        ctx["nodes"] = (xs.numpy() + sid).astype(np.int64)
        ctx["samples"] = ys.numpy().astype(np.int64)
        return orig_in(self, samples, node_flows, *a, **k)

    il.InputLayer.sample = in_sample
