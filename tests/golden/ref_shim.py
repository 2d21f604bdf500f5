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

REF_SRC = os.environ.get("PYJUICE_REF_SRC", "/root/reference/src")


def load_reference():
    os.environ["TRITON_INTERPRET"] = "1"
    stub = tempfile.mkdtemp(prefix="mplstub_")
    os.makedirs(os.path.join(stub, "matplotlib"), exist_ok=True)
    with open(os.path.join(stub, "matplotlib", "__init__.py"), "w") as f:
        f.write("")
    with open(os.path.join(stub, "matplotlib", "pyplot.py"), "w") as f:
        f.write("")
    sys.path.insert(0, stub)
    sys.path.insert(0, REF_SRC)

    import torch

    torch.Tensor.cuda = lambda self, *a, **k: self
    torch.cuda.current_device = lambda: 0

    @contextlib.contextmanager
    def _nodev(*a, **k):
        yield

    torch.cuda.device = _nodev

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
