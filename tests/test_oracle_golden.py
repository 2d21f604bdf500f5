"""Pins the CPU oracle to the reference: its FP64 restatement reproduces the outputs that
the reference itself produced on the same circuits, parameters and data (golden fixtures
from ``tests/golden/make_golden.py``). CPU only."""

import numpy as np
import pytest

from conftest import load_fixture
from oracle import pc_oracle as orc

NCATS = {"tiny": 4, "hclt64": 4}


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_oracle_forward_backward_em(name):
    fx = load_fixture(name)
    lay = orc.layout_from_fixture(fx, ncats=NCATS[name])
    nm, ems, lls = orc.forward(lay, fx["params0"], fx["in_params0"], fx["x"])
    # the reference ran in FP32: agreement to FP32 rounding of the LL scale
    assert np.allclose(lls, fx["lls"], rtol=1e-6, atol=1e-5)
    nf, pf, in_pf = orc.backward(lay, fx["params0"], fx["x"], nm, ems)
    scale = np.abs(fx["param_flows"]).max()
    assert np.abs(pf - fx["param_flows"]).max() <= 1e-5 * scale
    assert np.abs(in_pf - fx["in_param_flows"]).max() <= 1e-5 * np.abs(fx["in_param_flows"]).max()
    p1, ip1 = orc.em_update(lay, fx["params0"], fx["param_flows"].astype(np.float64), fx["in_params0"],
                            fx["in_param_flows"].astype(np.float64), 0.1, 0.1)
    assert np.abs(p1 - fx["params1"]).max() <= 1e-6
    assert np.abs(ip1 - fx["in_params1"]).max() <= 1e-6


def test_oracle_node_values_tiny():
    fx = load_fixture("tiny")
    lay = orc.layout_from_fixture(fx, ncats=4)
    nm, ems, _ = orc.forward(lay, fx["params0"], fx["in_params0"], fx["x"])
    ref = fx["node_mars"]
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(nm))
    assert np.abs(nm[fin] - ref[fin]).max() < 1e-5


def test_oracle_probabilities_sum_to_one():
    """Sum of p(x) over every assignment of the tiny circuit is 1 (a size-independent property)."""
    import itertools
    fx = load_fixture("tiny")
    lay = orc.layout_from_fixture(fx, ncats=4)
    x = np.array(list(itertools.product(range(4), repeat=6)), dtype=np.int64)
    _, _, lls = orc.forward(lay, fx["params0"], fx["in_params0"], x)
    # parameters are FP32-normalised, so the total is 1 up to FP32 rounding
    assert abs(np.exp(lls).sum() - 1.0) < 2e-6


def test_uniform_hash_known_values():
    # SplitMix64 of the counter: fixed outputs guard the sampler's draw contract
    u = [float(orc.uniform(0, 0, 0)), float(orc.uniform(12345, 7, 3)), float(orc.uniform(2 ** 62, 2 ** 31, 1023))]
    assert all(0.0 <= v < 1.0 for v in u)
    assert len(set(u)) == 3
    assert orc.uniform(1, 2, 3) == orc.uniform(1, 2, 3)


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_oracle_sampler_matches_reference_draws(name):
    """The oracle's sampler reproduces the samples the reference's own queries.sample drew
    when each of its tl.rand draws for node n in sample s was uniform_table(seed)[n, s]
    (fixtures samples_*.npz, made by running the reference): pins the draw rules (sum: first
    child whose running weight sum exceeds u; categorical: first category whose running sum
    reaches u) to the reference's."""
    fx = load_fixture(name)
    sf = load_fixture("samples_" + name)
    lay = orc.layout_from_fixture(fx, ncats=NCATS[name])
    assert lay["num_nodes"] == int(sf["num_nodes"])
    got = orc.sample(lay, fx["params0"], fx["in_params0"], int(sf["num_samples"]), int(sf["uniform_seed"]),
                     sf["samples"].shape[1])
    assert np.array_equal(got, sf["samples"])


def test_oracle_keep_zero_em_and_normalisation():
    """keep_zero_params EM and the sum-to-one normalisation of the oracle against the
    reference's own outputs (fixture em_tiny.npz)."""
    fx = load_fixture("em_tiny")
    lay = orc.layout_from_fixture(load_fixture("tiny"), ncats=4)
    nm, ems, _ = orc.forward(lay, fx["params0"], fx["in_params0"], fx["x"])
    _, pf, in_pf = orc.backward(lay, fx["params0"], fx["x"], nm, ems)
    assert np.abs(pf - fx["param_flows"]).max() <= 1e-5 * np.abs(fx["param_flows"]).max()
    p1, ip1 = orc.em_update(lay, fx["params0"], fx["param_flows"].astype(np.float64), fx["in_params0"],
                            fx["in_param_flows"].astype(np.float64), 0.1, 0.1, keep_zero_params=True)
    assert np.abs(p1 - fx["params1_keep_zero"]).max() <= 1e-6
    assert np.all(p1[fx["params0"] == 0] == 0)
    assert np.abs(ip1 - fx["in_params1_keep_zero"]).max() <= 1e-6
    got = orc.normalize(lay, fx["norm_in"], 0.3)
    assert np.abs(got - fx["norm_out"]).max() <= 1e-6


ALG_CASES = [("mpe", "MPE", 1.0, False, False), ("gll", "GeneralLL", 0.5, False, False),
             ("logspace", "LL", 1.0, True, False), ("negate", "LL", 1.0, False, True)]


@pytest.mark.parametrize("case", ALG_CASES, ids=[c[0] for c in ALG_CASES])
def test_oracle_propagation_algorithms_match_reference(case):
    """MPE and GeneralLL(0.5) passes, log-space flows and negated parameter flows of the
    oracle against the reference's own outputs on the tiny circuit (fixture alg_tiny.npz)."""
    name, alg, alpha, logspace, negate = case
    fx = load_fixture("tiny")
    ref = load_fixture("alg_tiny")
    lay = orc.layout_from_fixture(fx, ncats=4)
    nm, ems, lls = orc.forward_alg(lay, fx["params0"], fx["in_params0"], fx["x"], alg, alpha)
    assert np.allclose(lls, ref[name + "_lls"], rtol=1e-6, atol=1e-5)
    nf, pf, ipf = orc.backward_alg(lay, fx["params0"], fx["x"], nm, ems, alg=alg, alpha=alpha, logspace=logspace,
                                   negate=negate)
    rpf = ref[name + "_param_flows"]
    assert np.abs(pf - rpf).max() <= 1e-5 * np.abs(rpf).max()
    ripf = ref[name + "_in_param_flows"][:ipf.shape[0]]
    assert np.abs(ipf - ripf).max() <= 1e-5 * np.abs(ripf).max()
    rnf = ref[name + "_node_flows"]
    fin = np.isfinite(rnf)
    assert np.array_equal(fin, np.isfinite(nf))
    assert np.abs(nf[fin] - rnf[fin]).max() <= 1e-5


def test_oracle_queries_match_reference():
    """Marginals with a per-sample missing mask, the conditional query with hard evidence
    (missing mask) and with soft evidence, and input flows with a per-variable missing mask,
    against the reference's own outputs (fixture query_tiny.npz)."""
    fx = load_fixture("tiny")
    q = load_fixture("query_tiny")
    lay = orc.layout_from_fixture(fx, ncats=4)
    p0, q0, x = fx["params0"], fx["in_params0"], fx["x"]
    nm, ems, lls = orc.forward(lay, p0, q0, x, missing_mask=q["mask"])
    assert np.allclose(lls, q["marginal_lls"], rtol=1e-6, atol=1e-5)
    nf, _, _ = orc.backward(lay, p0, x, nm, ems)
    assert np.abs(orc.conditional(lay, q0, nf) - q["cond_hard_full"]).max() <= 1e-6
    nm, ems, lls = orc.forward(lay, p0, q0, evidence=q["soft"])
    assert np.allclose(lls, q["soft_lls"], rtol=1e-6, atol=1e-5)
    nf, _, _ = orc.backward(lay, p0, None, nm, ems)
    assert np.abs(orc.conditional(lay, q0, nf) - q["cond_soft"]).max() <= 1e-6
    nm, ems, lls = orc.forward(lay, p0, q0, x, missing_mask=q["vmask"])
    assert np.allclose(lls, q["vmask_lls"], rtol=1e-6, atol=1e-5)
    _, pf, ipf = orc.backward(lay, p0, x, nm, ems, missing_mask=q["vmask"], in_params=q0)
    assert np.abs(pf - q["vmask_param_flows"]).max() <= 1e-5 * np.abs(pf).max()
    ref_ipf = q["vmask_in_param_flows"][:ipf.shape[0]]
    assert np.abs(ipf - ref_ipf).max() <= 1e-5 * np.abs(ref_ipf).max()


def test_oracle_evidence_free_flows_match_reference():
    """Flows of the evidence-free pass (every variable missing), whose per-sample node flows
    are the top-down probabilities, against the reference's own (fixture tdp_tiny.npz)."""
    fx = load_fixture("tiny")
    t = load_fixture("tdp_tiny")
    lay = orc.layout_from_fixture(fx, ncats=4)
    x = np.zeros([4, 6], dtype=np.int64)
    miss = np.ones(6, dtype=bool)
    nm, ems, lls = orc.forward(lay, fx["params0"], fx["in_params0"], x, missing_mask=miss)
    assert np.abs(lls - t["lls"]).max() <= 1e-5
    nf, pf, ipf = orc.backward(lay, fx["params0"], x, nm, ems, missing_mask=miss, in_params=fx["in_params0"])
    # the reference's backward rewrote the node flows of its large sum layers in place as
    # log f - log m (allow_modify_flows): every row matches in one of the two forms
    ref = t["node_flows"]
    with np.errstate(divide="ignore"):
        rewritten = np.log(nf) - nm
    ok = np.all(np.abs(nf - ref) <= 1e-5, axis=1) | np.all(np.abs(rewritten - ref) <= 1e-5, axis=1)
    assert ok.all()
    n_in0 = lay["input"]["nid_start"]
    assert np.abs(nf[n_in0:n_in0 + lay["input"]["vids"].shape[0]] -
                  ref[n_in0:n_in0 + lay["input"]["vids"].shape[0]]).max() <= 1e-5
    assert np.abs(pf - t["param_flows"]).max() <= 1e-5 * np.abs(pf).max()
    ref_ipf = t["in_param_flows"][:ipf.shape[0]]
    assert np.abs(ipf - ref_ipf).max() <= 1e-5 * np.abs(ref_ipf).max()


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_torch_port_matches_oracle(name):
    """The FP32 torch CPU restatement (CPU baseline and reference arm of bench.py) against the
    FP64 oracle: log-likelihoods, parameter flows and the EM update."""
    import torch
    from oracle import torch_port as tp
    fx = load_fixture(name)
    lay = orc.layout_from_fixture(fx, ncats=NCATS[name])
    tl = tp.TorchLayout(lay)
    p0, q0 = torch.from_numpy(fx["params0"]), torch.from_numpy(fx["in_params0"])
    x = torch.from_numpy(fx["x"])
    nm, ems, lls = tp.forward(tl, p0, q0, x)
    assert np.allclose(lls.numpy(), fx["lls"], rtol=1e-5, atol=1e-5)
    pf, ipf = tp.backward(tl, p0, x, nm, ems)
    assert np.abs(pf.numpy() - fx["param_flows"]).max() <= 1e-4 * np.abs(fx["param_flows"]).max()
    ref_ipf = fx["in_param_flows"]
    assert np.abs(ipf.numpy()[:ref_ipf.shape[0]] - ref_ipf).max() <= 1e-4 * np.abs(ref_ipf).max()
    p1, q1 = tp.em_update(tl, p0, torch.from_numpy(fx["param_flows"]), q0, torch.from_numpy(fx["in_param_flows"]),
                          0.1, 0.1)
    assert np.abs(p1.numpy() - fx["params1"]).max() <= 1e-6
    assert np.abs(q1.numpy()[:fx["in_params1"].shape[0]] - fx["in_params1"]).max() <= 1e-6
