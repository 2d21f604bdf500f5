"""``.jpc`` files move between the reference and pyjuice_b200 in both directions (CPU only):
the reference's own file of the tiny circuit loads and compiles to the same parameters and
layout, the reference loaded a file written here and reproduced the circuit's parameters
and log-likelihoods (fixture io_tiny.npz), and save/load round-trips here."""

import os
import tempfile

import numpy as np
import torch

from conftest import load_fixture
from circuits import build_tiny_dag
from helpers import layout_mismatches

import pyjuice_b200 as juice
from pyjuice_b200.nodes import distributions as dists
from oracle import pc_oracle as orc


def test_load_reference_file():
    fx = load_fixture("tiny")
    io_fx = load_fixture("io_tiny")
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ref.jpc")
        with open(path, "wb") as f:
            f.write(io_fx["ref_jpc"].tobytes())
        pc = juice.compile(juice.load(path), max_tied_ns_per_parflow_block=1)
    assert layout_mismatches(pc, fx) == []
    # loading renormalises the sum weights (as the reference does), within FP32 rounding
    assert np.abs(pc.params.numpy() - fx["params0"]).max() <= 1e-6
    assert np.array_equal(pc.input_layer_group[0].params.numpy()[:fx["in_params0"].shape[0]], fx["in_params0"])


def test_reference_loads_our_file():
    """What the reference computed from a file saved here equals the circuit saved."""
    fx = load_fixture("tiny")
    io_fx = load_fixture("io_tiny")
    assert np.abs(io_fx["ref_loads_ours_params"] - fx["params0"]).max() <= 1e-6
    lay = orc.layout_from_fixture(fx, ncats=4)
    _, _, lls = orc.forward(lay, fx["params0"], fx["in_params0"], fx["x"])
    assert np.allclose(io_fx["ref_loads_ours_lls"], lls, rtol=1e-6, atol=1e-5)


def test_save_load_round_trip():
    torch.manual_seed(3)
    pc = juice.compile(build_tiny_dag(juice, dists), max_tied_ns_per_parflow_block=1)
    with torch.no_grad():
        pc.params.mul_(torch.rand_like(pc.params) + 0.5)  # parameters that differ from the nodes'
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "c.jpc")
        juice.save(path, pc)
        pc2 = juice.compile(juice.load(path), max_tied_ns_per_parflow_block=1)
    assert torch.equal(pc.input_layer_group[0].params, pc2.input_layer_group[0].params)
    # the file holds the circuit's current weights; loading renormalises them
    pc.update_parameters()
    ref = pc.params.clone()
    juice.TensorCircuit._normalize_host(pc, ref)
    assert torch.allclose(pc2.params, ref, atol=1e-6)
    assert pc2.num_nodes == pc.num_nodes and pc2.num_edges == pc.num_edges
