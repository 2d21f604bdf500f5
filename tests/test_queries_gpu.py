"""Queries and the differentiable soft-evidence log-likelihood on the GPU:

* ``queries.marginal`` (per-sample missing mask) and ``queries.conditional`` (hard evidence
  with a missing mask; soft evidence) against the reference's own outputs (query_tiny.npz);
* a forward + backward pass with a per-variable missing mask (parameter and input flows)
  against the reference;
* ``autograd.circuit_ll``: gradients with respect to the sum logits and the soft evidence
  against FP64 central differences of the oracle, for all-positive, all-negative and
  mixed-sign upstream gradients.
"""

import numpy as np
import pytest
import torch

from conftest import load_fixture
from helpers import build_fixture_circuit, load_fixture_params
from oracle import pc_oracle as orc

import pyjuice_b200 as juice

pytestmark = pytest.mark.gpu


def _tiny(device):
    fx = load_fixture("tiny")
    pc = build_fixture_circuit("tiny", fx).to(device)
    load_fixture_params(pc, fx)
    return pc, fx


def test_marginal_matches_reference(cuda_device):
    pc, fx = _tiny(cuda_device)
    q = load_fixture("query_tiny")
    lls = juice.queries.marginal(pc, torch.from_numpy(fx["x"]), missing_mask=torch.from_numpy(q["mask"]))
    ref = q["marginal_lls"]
    assert np.all(np.abs(lls.cpu().numpy() - ref) <= 1e-5 * np.abs(ref) + 1e-6)
    # everything missing: log 1
    allm = torch.ones(fx["x"].shape, dtype=torch.bool)
    assert torch.allclose(juice.queries.marginal(pc, torch.from_numpy(fx["x"]), missing_mask=allm).cpu(),
                          torch.zeros([fx["x"].shape[0], 1]), atol=1e-5)


def test_conditional_hard_and_soft_match_reference(cuda_device):
    pc, fx = _tiny(cuda_device)
    q = load_fixture("query_tiny")
    x = torch.from_numpy(fx["x"])
    got = juice.queries.conditional(pc, x, missing_mask=torch.from_numpy(q["mask"])).cpu().numpy()
    assert np.abs(got - q["cond_hard_full"]).max() <= 1e-5
    sel = juice.queries.conditional(pc, x, missing_mask=torch.from_numpy(q["mask"]), target_vars=[0, 2, 5])
    assert np.abs(sel.cpu().numpy() - q["cond_hard_full"][:, [0, 2, 5]]).max() <= 1e-5
    soft = juice.queries.conditional(pc, torch.from_numpy(q["soft"])).cpu().numpy()
    assert np.abs(soft - q["cond_soft"]).max() <= 1e-5
    r0, r1 = pc._root_node_range
    assert np.abs(pc.node_mars[r0:r1].cpu().numpy().T - q["soft_lls"]).max() <= 1e-5


def test_missing_mask_flows_match_reference(cuda_device):
    pc, fx = _tiny(cuda_device)
    q = load_fixture("query_tiny")
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, missing_mask=torch.from_numpy(q["vmask"]), force_use_fp32=True)
    assert np.abs(lls.detach().cpu().numpy() - q["vmask_lls"]).max() <= 1e-5
    lls.mean().backward()
    pf = pc.param_flows.cpu().numpy()
    assert np.abs(pf - q["vmask_param_flows"]).max() <= 1e-4 * np.abs(q["vmask_param_flows"]).max()
    ref = q["vmask_in_param_flows"]
    ipf = pc.input_layer_group[0].param_flows.cpu().numpy()[:ref.shape[0]]
    assert np.abs(ipf - ref).max() <= 1e-4 * np.abs(ref).max()


def _softmax_params(pc, logits):
    p = np.zeros_like(logits)
    for pb, k, bs in zip(pc._em_pbase.tolist(), pc._em_nch.tolist(), pc._em_bs.tolist()):
        z = logits[pb:pb + k * bs].reshape(k, bs)
        e = np.exp(z - z.max(axis=0))
        p[pb:pb + k * bs] = (e / e.sum(axis=0)).reshape(-1)
    return p


@pytest.mark.parametrize("sign", ["pos", "neg", "mixed"])
def test_circuit_ll_adjoint_vs_central_differences(sign, cuda_device):
    """d(weighted LL)/d(sum logits) and d/d(soft evidence) of autograd.circuit_ll against FP64
    central differences (h = 1e-6) of the oracle on the tiny circuit."""
    pc, fx = _tiny(cuda_device)
    lay = orc.layout_from_circuit(pc)
    rng = np.random.default_rng(17)
    B, V, K = 16, 6, 4
    ev = rng.dirichlet(np.ones(K), size=(B, V))
    z = rng.normal(size=pc.params.numel())
    wts = {"pos": np.full(B, 1.0 / B), "neg": np.full(B, -1.0 / B), "mixed": rng.normal(size=B)}[sign]
    q0 = fx["in_params0"].astype(np.float64)

    def f(zz, ee):
        _, _, lls = orc.forward(lay, _softmax_params(pc, zz), q0, evidence=ee)
        return float((lls[:, 0] * wts).sum())

    zt = torch.tensor(z, dtype=torch.float32, device=cuda_device, requires_grad=True)
    et = torch.tensor(ev, dtype=torch.float32, device=cuda_device, requires_grad=True)
    lls = juice.autograd.circuit_ll(pc, zt, et)
    (lls[:, 0] * torch.tensor(wts, dtype=torch.float32, device=cuda_device)).sum().backward()
    gz, ge = zt.grad.double().cpu().numpy(), et.grad.double().cpu().numpy()
    # FD at the FP32-rounded point the device evaluated
    z32, e32 = z.astype(np.float32).astype(np.float64), ev.astype(np.float32).astype(np.float64)
    h = 1e-6
    used = np.concatenate([np.arange(pb, pb + k * bs) for pb, k, bs in
                           zip(pc._em_pbase.tolist(), pc._em_nch.tolist(), pc._em_bs.tolist())])
    for i in rng.choice(used, size=12, replace=False):
        d = np.zeros_like(z32)
        d[i] = h
        fd = (f(z32 + d, e32) - f(z32 - d, e32)) / (2 * h)
        assert abs(gz[i] - fd) <= 2e-3 * max(abs(fd), 1e-2), (i, gz[i], fd)
    for _ in range(12):
        b, v, k = rng.integers(B), rng.integers(V), rng.integers(K)
        d = np.zeros_like(e32)
        d[b, v, k] = h
        fd = (f(z32, e32 + d) - f(z32, e32 - d)) / (2 * h)
        assert abs(ge[b, v, k] - fd) <= 2e-3 * max(abs(fd), 1e-2), ((b, v, k), ge[b, v, k], fd)


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_partial_evaluation(name, cuda_device):
    """After a full pass, changing one variable and re-evaluating only the node vectors whose
    scope contains it (forward, from the cached node values) gives the full pass's
    log-likelihoods; a partial backward pass over the same scopes gives the full pass's flows
    of those input nodes."""
    from pyjuice_b200.nodes import get_subsumed_scopes
    fx = load_fixture(name)
    pc = build_fixture_circuit(name, fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"][:64]).to(cuda_device)
    K = 4
    v = 2
    with torch.no_grad():
        _, cache = pc(x, force_use_fp32=True, return_cache=True)
    x2 = x.clone()
    x2[:, v] = (x2[:, v] + 1) % K
    scopes = get_subsumed_scopes(pc, [v])
    pc.enable_partial_evaluation(scopes, forward=True)
    with torch.no_grad():
        part = pc(x2, force_use_fp32=True, cache=cache).clone()
    pc.disable_partial_evaluation()
    with torch.no_grad():
        full = pc(x2, force_use_fp32=True)
    assert torch.allclose(part, full, rtol=1e-6, atol=1e-5)
    # backward: full pass, then partial over the same scopes
    pc.init_param_flows(flows_memory=0.0)
    pc.backward(inputs=x2, allow_modify_flows=False, force_use_fp32=True)
    il = pc.input_layer_group[0]
    lo, hi = il._output_ind_range
    sel = (il.vids[:, 0] == v).nonzero().view(-1) + lo
    nf_full = pc.node_flows[sel].clone()
    ipf_full = il.param_flows.clone()
    pc.enable_partial_evaluation(scopes, backward=True)
    pc.init_param_flows(flows_memory=0.0)
    pc.backward(inputs=x2, force_use_fp32=True)
    pc.disable_partial_evaluation()
    assert torch.allclose(pc.node_flows[sel], nf_full, rtol=1e-5, atol=1e-6)
    slots = torch.cat([il.s_pfids[s - lo] + torch.arange(K, device=cuda_device) for s in sel.tolist()])
    assert torch.allclose(il.param_flows[slots], ipf_full[slots], rtol=1e-5, atol=1e-6)
