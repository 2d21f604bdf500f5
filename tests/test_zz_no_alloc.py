"""Whole-circuit sampling without allocation (pcb_sample_circuit_noalloc, called through
the C ABI) gives the same samples as the per-layer sampling path, call after call.
Collected last so that it also runs after everything else in one process."""

import numpy as np
import pytest
import torch

from conftest import load_fixture
from helpers import build_fixture_circuit, load_fixture_params

import pyjuice_b200 as juice
from pyjuice_b200 import _native as nat
from pyjuice_b200.queries.sample import noalloc_sample_plan

pytestmark = pytest.mark.gpu

MAX_INTS = 1 << 21  # PCB_SAMPLE_NOALLOC_MAX_INTS


def _call(plan, samples, err, seed, S=None):
    table, num_steps, root_id, cap_n, cap_e = plan
    nat.call("pcb_sample_circuit_noalloc", nat.ptr(table), num_steps, root_id,
             samples.size(0) if S is None else S, cap_n, cap_e, nat.ptr(samples), samples.stride(0), seed,
             nat.ptr(err), nat.stream())


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_noalloc_matches_per_layer_sampling(name, cuda_device):
    fx = load_fixture(name)
    pc = build_fixture_circuit(name, fx).to(cuda_device)
    load_fixture_params(pc, fx)
    S = 257  # not a multiple of the 128-thread block
    plan = noalloc_sample_plan(pc)
    assert S * (plan[3] + plan[4]) <= MAX_INTS
    seeds = [1234567, 99]
    outs = [torch.zeros([S, pc.num_vars], dtype=torch.long, device=cuda_device) for _ in seeds]
    err = torch.full([1], 7, dtype=torch.int32, device=cuda_device)
    _call(plan, outs[0], err, 5)  # first call on the device: address look-up
    torch.cuda.synchronize()
    outs[0].zero_()
    before = torch.cuda.memory_allocated(cuda_device)
    for out, seed in zip(outs, seeds):  # two calls in a row, no synchronisation between them
        _call(plan, out, err, seed)
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated(cuda_device) == before
    assert int(err.item()) == 0
    for out, seed in zip(outs, seeds):
        ref = juice.queries.sample(pc, S, seed=seed)
        assert torch.equal(out, ref)
    assert not torch.equal(outs[0], outs[1])


def test_noalloc_rejects_oversize(cuda_device):
    fx = load_fixture("tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    plan = noalloc_sample_plan(pc)
    samples = torch.zeros([1, pc.num_vars], dtype=torch.long, device=cuda_device)
    err = torch.zeros([1], dtype=torch.int32, device=cuda_device)
    too_many = MAX_INTS // (plan[3] + plan[4]) + 1
    with pytest.raises(RuntimeError, match="exceed the fixed working area"):
        _call(plan, samples, err, 0, S=too_many)  # rejected on the host, nothing launched
    # the largest accepted batch still works
    S = MAX_INTS // (plan[3] + plan[4])
    big = torch.zeros([S, pc.num_vars], dtype=torch.long, device=cuda_device)
    _call(plan, big, err, 3)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(big[:64], juice.queries.sample(pc, 64, seed=3))
