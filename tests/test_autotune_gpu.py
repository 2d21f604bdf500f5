"""The launch-shape autotuner: with tuning on, the first pass times the candidate shapes of
every contraction, parameter-flow and single-stage launch and keeps the fastest; results
equal the static shapes' (within the FP32 summation-order differences of the kernels), and a capture after tuning replays the same."""

import numpy as np
import pytest
import torch

from conftest import load_fixture
from helpers import build_fixture_circuit, load_fixture_params

from pyjuice_b200.autotune import TUNER

pytestmark = pytest.mark.gpu


def test_autotuned_step_matches_static(cuda_device):
    fx = load_fixture("hclt784")
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.integers(0, 256, size=(128, 784))).to(cuda_device)
    out = []
    saved = (TUNER.enabled, dict(TUNER.choices))
    try:
        for enabled in (False, True):
            TUNER.enabled = enabled
            TUNER.choices.clear()
            pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
            load_fixture_params(pc, fx)
            pc.init_param_flows(flows_memory=0.0)
            with torch.no_grad():
                lls = pc(x, force_use_bf16=True)
            pc.backward(inputs=x, allow_modify_flows=True)
            torch.cuda.synchronize()
            out.append((lls.clone(), pc.param_flows.clone()))
        assert any(k.startswith("tc05") for k in TUNER.choices)
        assert any(k.startswith("pflows") for k in TUNER.choices)
        assert any(k.startswith("short") for k in TUNER.choices)
        assert all(np.isfinite(v).all() for t in TUNER.timings.values() for v in [np.array(list(t.values()))]
                   if np.isfinite(v).any())
    finally:
        TUNER.enabled = saved[0]
        TUNER.choices.clear()
        TUNER.choices.update(saved[1])
    (l0, p0), (l1, p1) = out
    assert (l1 - l0).abs().max().item() <= 1e-5 * l0.abs().max().item()
    rel = (p1 - p0).abs().max().item() / p0.abs().max().item()
    assert rel <= 1e-5
