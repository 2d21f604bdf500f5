"""``.jpc`` files move between the reference and pyjuice_b200 in both directions (CPU only):
the reference's own file of the tiny circuit loads and compiles to the same parameters and
layout, the reference loaded a file written here and reproduced the circuit's parameters
and log-likelihoods (fixture io_tiny.npz), and save/load round-trips here."""

import os
import tempfile

import numpy as np
import pytest
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


@pytest.mark.parametrize("name,cls", [("bern", "Bernoulli"), ("gauss", "Gaussian"), ("dlog", "DiscreteLogistic"),
                                      ("poe", "SoftEvidenceCategorical")])
def test_distribution_files_both_ways(name, cls):
    """.jpc files of circuits over Bernoulli, Gaussian, DiscreteLogistic and
    SoftEvidenceCategorical inputs (io_dists.npz): the reference's file loads here with its
    distribution class, attributes and parameters; the reference loaded the file saved here to
    the same parameters and (dists.npz data) the log-likelihoods it computes for its own
    circuit."""
    io_fx = load_fixture("io_dists")
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ref.jpc")
        with open(path, "wb") as f:
            f.write(io_fx[name + "_ref_jpc"].tobytes())
        pc = juice.compile(juice.load(path))
    layer = pc.input_layer_group[0]
    dist = layer.nodes[0].dist
    assert type(dist).__name__ == cls
    if cls == "DiscreteLogistic":
        assert dist.val_range == (-2.0, 2.0) and dist.num_cats == 8 and dist.min_std == 0.01
    if cls == "Gaussian":
        assert dist.mu == 0.0 and dist.sigma == 1.0 and dist.min_sigma == 0.01
    if cls == "SoftEvidenceCategorical":
        assert dist.num_cats == 6
    ref_in = io_fx[name + "_in_params"]
    assert np.array_equal(layer.params.numpy()[:ref_in.shape[0]], ref_in)
    assert np.abs(pc.params.numpy() - io_fx[name + "_params"]).max() <= 1e-6
    # the reference's view of our file
    assert np.abs(io_fx[name + "_ref_loads_ours_params"] - io_fx[name + "_params"]).max() <= 1e-6
    assert np.array_equal(io_fx[name + "_ref_loads_ours_in_params"], ref_in)
    if name != "poe":
        lls = load_fixture("dists")[name + "_lls"]
        assert np.allclose(io_fx[name + "_ref_loads_ours_lls"], lls, rtol=1e-6, atol=1e-6)
