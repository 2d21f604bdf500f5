import os
import sys

# Launch shapes stay at their static defaults in the tests (the autotuner's choices depend on
# timing); tests/test_autotune_gpu.py switches the tuner on explicitly.
os.environ.setdefault("PCB_AUTOTUNE", "0")

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(TESTS, "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libpcb200.so")


def load_fixture(name: str):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"fixture {name}.npz not generated")
    return dict(np.load(path))


@pytest.fixture
def cuda_device():
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    return torch.device("cuda:0")
