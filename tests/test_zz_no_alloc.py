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
    errs = [torch.full([1], 7, dtype=torch.int32, device=cuda_device) for _ in seeds]
    _call(plan, outs[0], errs[0], 5)  # first call on the device: address look-up
    torch.cuda.synchronize()
    outs[0].zero_()
    errs[0].fill_(7)
    before = torch.cuda.memory_allocated(cuda_device)
    for out, err, seed in zip(outs, errs, seeds):  # two calls in a row, no synchronisation between them
        _call(plan, out, err, seed)
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated(cuda_device) == before
    assert [int(e.item()) for e in errs] == [0, 0]  # each call cleared and kept its own error word
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


def test_noalloc_reports_list_overflow(cuda_device):
    """Element lists one slot too short: the kernel skips the writes past the cap and reports
    code 1 (the working area is sized from the caps the caller passes, so nothing is written
    out of bounds)."""
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    table, num_steps, root_id, cap_n, cap_e = noalloc_sample_plan(pc)
    samples = torch.zeros([64, pc.num_vars], dtype=torch.long, device=cuda_device)
    err = torch.zeros([1], dtype=torch.int32, device=cuda_device)
    _call((table, num_steps, root_id, cap_n, cap_e - 1), samples, err, 1)
    torch.cuda.synchronize()
    assert int(err.item()) == 1


def test_noalloc_python_wrapper(cuda_device):
    """queries.sample_noalloc (argument checks, then the same entry point) equals queries.sample;
    a samples tensor narrower than num_vars is refused before anything is launched."""
    from pyjuice_b200.queries.sample import sample_noalloc
    fx = load_fixture("tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    out = torch.zeros([100, pc.num_vars], dtype=torch.long, device=cuda_device)
    err = torch.full([1], 9, dtype=torch.int32, device=cuda_device)
    sample_noalloc(pc, out, err, seed=42)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(out, juice.queries.sample(pc, 100, seed=42))
    narrow = torch.zeros([100, pc.num_vars - 1], dtype=torch.long, device=cuda_device)
    with pytest.raises(ValueError, match="num_vars"):
        sample_noalloc(pc, narrow, err, seed=42)
