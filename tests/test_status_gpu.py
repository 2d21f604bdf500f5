"""The device status word: faults that kernels detect on the device (a bounded wait that
runs out, a contraction tile longer than the kernel handles, an input value outside the
categories) are reported through pcb_device_status, not only as NaN outputs, and the
context stays usable afterwards. No test here faults the GPU: the wait test polls an
mbarrier that nothing completes a bounded number of times, and the oversize tiles are
rejected by the kernels before they read anything."""

import ctypes

import numpy as np
import pytest
import torch

from conftest import load_fixture
from helpers import build_fixture_circuit, load_fixture_params

from pyjuice_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _tile_table(k_cnt, n_rows, device):
    # PcbLseTile: out_row, n_rows, k_off, k_cnt, w_add, aux_row, g_stride, reserved
    return torch.tensor([[0, n_rows, 0, k_cnt, 0, 0, 0, 0]], dtype=torch.int32, device=device)


def test_bounded_wait_timeout_is_reported(cuda_device):
    nat.device_status(clear=True)
    nat.call("pcb_status_selftest", 2000, nat.stream())
    assert nat.device_status(clear=True) == 1
    assert nat.device_status(clear=True) == 0  # cleared
    # the context is still usable
    x = torch.arange(10, device=cuda_device, dtype=torch.float32)
    assert float(x.sum().item()) == 45.0


@pytest.mark.parametrize("kernel", ["short", "tc05"])
def test_oversize_tile_is_reported(kernel, cuda_device):
    B = 64
    src = torch.zeros([256, B], dtype=torch.float32, device=cuda_device)
    out = torch.zeros([128, B], dtype=torch.float32, device=cuda_device)
    params = torch.ones([1024], dtype=torch.float32, device=cuda_device)
    krow = torch.zeros([256], dtype=torch.int32, device=cuda_device)
    kw = torch.zeros([256], dtype=torch.int32, device=cuda_device)
    tiles = _tile_table(129, 128 if kernel == "tc05" else 32, cuda_device)
    nat.device_status(clear=True)
    if kernel == "short":
        nat.call("pcb_lse_contract_short", nat.ptr(src), nat.ptr(None), nat.ptr(None), nat.ptr(out), B, B,
                 nat.ptr(params), nat.ptr(tiles), 1, 32, 32, nat.ptr(krow), nat.ptr(kw), 1, 0, 0, nat.ptr(None), 0, 32,
                 nat.ptr(None), nat.stream())
        rows = out[:32]
    else:
        packed = torch.zeros([65536], dtype=torch.uint8, device=cuda_device)
        nat.call("pcb_lse_contract_tc05", nat.ptr(src), nat.ptr(None), nat.ptr(None), nat.ptr(out), B, B,
                 nat.ptr(packed), nat.ptr(tiles), 1, nat.ptr(krow), 0, 2, 64, 1, nat.stream())
        rows = out
    assert nat.device_status(clear=True) == 2
    assert torch.isnan(rows).all()


def test_bad_category_is_reported(cuda_device):
    fx = load_fixture("tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"][:8]).to(cuda_device).clone()
    nat.device_status(clear=True)
    with torch.no_grad():
        pc(x, force_use_fp32=True)
    assert nat.device_status(clear=True) == 0
    x[0, 0] = 99
    with torch.no_grad():
        pc(x, force_use_fp32=True)
    with pytest.raises(RuntimeError, match="outside"):
        nat.check_device_status()
    assert nat.device_status() == 0
