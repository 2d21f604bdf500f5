"""The PD and HMM generators build the same circuits as the reference's (structures.npz):
the compiled layouts are identical, and the oracle evaluates the reference's parameters on
our layout to the reference's log-likelihoods (and, for the homogeneous HMM, its flows and
EM step with tied transition and emission vectors). Also the host plans that tied layers
enable (shared packed weights, one parameter-flow launch per tied set) and the
DiscreteLogistic layer's layout. CPU only."""

import numpy as np
import torch

from conftest import load_fixture
from helpers import layout_mismatches

import pyjuice_b200 as juice
from pyjuice_b200.nodes import distributions as dists
from oracle import pc_oracle as orc


def _sub(fx, prefix):
    return {k[len(prefix):]: v for k, v in fx.items() if k.startswith(prefix)}


def test_pd_matches_reference():
    fx = _sub(load_fixture("structures"), "pd_")
    torch.manual_seed(7)
    root = juice.structures.PD((3, 3), 32, split_intervals=1, max_prod_block_conns=2,
                               input_dist=dists.Categorical(num_cats=4))
    pc = juice.compile(root)
    assert layout_mismatches(pc, fx) == []
    lay = orc.layout_from_circuit(pc)
    _, _, lls = orc.forward(lay, fx["params"], fx["in_params"], fx["x"])
    assert np.allclose(lls, fx["lls"], rtol=1e-6, atol=1e-5)


def test_hmm_matches_reference():
    fx = _sub(load_fixture("structures"), "hmm_")
    root = juice.structures.HMM(6, 32, 10, homogeneous=True, alpha=torch.from_numpy(fx["alpha"]),
                                beta=torch.from_numpy(fx["beta"]), gamma=torch.from_numpy(fx["gamma"]))
    pc = juice.compile(root)
    assert layout_mismatches(pc, fx) == []
    assert np.abs(pc.params.numpy() - fx["params"]).max() <= 1e-6
    assert np.abs(pc.input_layer_group[0].params.numpy()[:fx["in_params"].shape[0]] - fx["in_params"]).max() <= 1e-6
    lay = orc.layout_from_circuit(pc)
    nm, ems, lls = orc.forward(lay, fx["params"], fx["in_params"], fx["x"])
    assert np.allclose(lls, fx["lls"], rtol=1e-6, atol=1e-5)
    _, pf, ipf = orc.backward(lay, fx["params"], fx["x"], nm, ems)
    assert np.abs(pf - fx["param_flows"]).max() <= 1e-5 * np.abs(pf).max()
    ref_ipf = fx["in_param_flows"][:ipf.shape[0]]
    assert np.abs(ipf - ref_ipf).max() <= 1e-5 * np.abs(ref_ipf).max()
    p1, q1 = orc.em_update(lay, fx["params"], fx["param_flows"].astype(np.float64), fx["in_params"],
                           fx["in_param_flows"].astype(np.float64), 0.5, 0.01)
    assert np.abs(p1 - fx["params1"]).max() <= 1e-6
    assert np.abs(q1 - fx["in_params1"][:q1.shape[0]]).max() <= 1e-6


def test_discrete_logistic_layer_matches_reference_layout():
    """A DiscreteLogistic input layer compiles to the reference's sizes (two parameters and
    three flow slots per node, dists.npz), with seeded initial parameters equal to the
    reference's (same torch draws), and the per-node metadata the kernels read is
    (lo, hi, num_cats, min_std) of each node. CPU only."""
    from circuits import build_dist_dag
    fx = load_fixture("dists")
    torch.manual_seed(11)
    pc = juice.compile(build_dist_dag(juice, lambda: dists.DiscreteLogistic(val_range=(-2.0, 2.0), num_cats=8)))
    layer = pc.input_layer_group[0]
    assert layer.num_parameters == fx["dlog_in_params0"].shape[0]
    assert layer.num_param_flows == fx["dlog_in_param_flows"].shape[0]
    assert np.abs(layer.params.detach().numpy()[:layer.num_parameters] - fx["dlog_in_params0"]).max() <= 1e-6
    assert pc.params.numel() == fx["dlog_params0"].shape[0]
    meta = layer._host_desc()["node_meta"].numpy().reshape(-1, 4)
    assert meta.shape[0] == layer.num_nodes
    assert np.allclose(meta, np.array([-2.0, 2.0, 8.0, 0.01], np.float32))


def test_tied_hmm_layers_share_packed_weights():
    """Packed-weight buffers: the tied time steps of a homogeneous HMM share one (forward and
    element-flow tables alike); an HMM without tied transitions shares none. CPU only (the
    buffers are planned, not filled)."""
    pc = juice.compile(juice.structures.HMM(6, 32, 10, homogeneous=True))
    pc._share_tied_packs()
    layers = [l for g in pc.inner_layer_groups if g.is_sum() for l in g]
    fw = [l._desc(pc.device)["fw_pack"].data_ptr() for l in layers]
    el = [l._desc(pc.device)["el_groups"][0]["pack"].data_ptr() for l in layers]
    assert len(set(fw[:-1])) == 1 and len(set(el[:-1])) == 1  # the transitions; the last layer is the root
    assert fw[-1] != fw[0]
    pc = juice.compile(juice.structures.HMM(6, 32, 10, homogeneous=False))
    pc._share_tied_packs()
    fw = [l._desc(pc.device)["fw_pack"].data_ptr() for g in pc.inner_layer_groups if g.is_sum() for l in g]
    assert len(set(fw)) == len(fw)


def test_tied_hmm_layers_form_one_parameter_flow_set():
    """The tied-set plan of the parameter flows: a homogeneous HMM's transition layers (the
    tied time steps and their source) form one set whose node / element row shifts follow the
    layers' positions; the source layer adds with atomics like its tied layers; an HMM
    without tied transitions has no set. CPU only (planning, no launch)."""
    pc = juice.compile(juice.structures.HMM(8, 64, 10, homogeneous=True))
    sums = [(gi, l) for gi, g in enumerate(pc.inner_layer_groups) if g.is_sum() for l in g]
    assert all(l._has_tied for _, l in sums[:-1]) and not sums[-1][1]._has_tied  # the root is untied
    sets = pc._tied_pflow_sets({gi: False for gi, _ in sums})
    assert len(sets) == 1
    ts = sets[0]
    assert len(ts["layers"]) == len(sums) - 1 and ts["last_gi"] == sums[0][0]
    deltas = ts["deltas"].view(-1, 2).numpy()
    ref = ts["ref"]
    for (dn, de), layer in zip(deltas, ts["layers"]):
        assert dn == layer._layer_nid_range[0] - ref._layer_nid_range[0]
        assert de % 128 == 0  # element-value regions of 2 x 64 rows per time step
    pc = juice.compile(juice.structures.HMM(8, 64, 10, homogeneous=False))
    sums = [(gi, l) for gi, g in enumerate(pc.inner_layer_groups) if g.is_sum() for l in g]
    assert pc._tied_pflow_sets({gi: False for gi, _ in sums}) == []
