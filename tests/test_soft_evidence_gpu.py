"""Input distributions beyond the Categorical on the GPU.

SoftEvidenceCategorical layers (categorical nodes times per-sample evidence), with the known
answers of the reference's own tests (tests/distributions/soft_evidence_cat_test.py:10-196): a product of such inputs under one sum
node gives, per variable, ``log_softmax(L + log theta)[x]``, and the evidence gradient that
``pc.backward`` accumulates equals torch autograd's gradient of those log-likelihoods. The
sparse evidence form (category ids per entry) is checked against the dense one, and the
parameter flows and EM step against the plain Categorical layer. Sampling: under evidence
(the reference's test), and for Bernoulli / DiscreteLogistic / Gaussian layers against the
circuit's own marginals and moments."""

import math

import pytest
import torch

from circuits import build_dist_dag

import pyjuice_b200 as juice
from pyjuice_b200.nodes import distributions as dists

pytestmark = pytest.mark.gpu


def _poe_circuit(num_vars, num_cats, num_nodes, device, scale_first=None):
    nis = [juice.inputs(v, num_nodes=num_nodes, dist=dists.SoftEvidenceCategorical(num_cats=num_cats))
           for v in range(num_vars)]
    ns = juice.summate(juice.multiply(*nis), num_nodes=1)
    ns.init_parameters(perturbation=0.0)
    if scale_first is not None:  # the first categories three times as likely
        for ni in nis:
            ni._params[:scale_first] *= 3
            ni._params /= 4
    return juice.compile(ns).to(device)


def _target(data, logits, add_logits=None):
    logits = logits.clone().requires_grad_(True)
    z = logits if add_logits is None else logits + add_logits
    lls = torch.log_softmax(z, dim=2).gather(2, data.unsqueeze(2)).squeeze(2).sum(dim=1)
    lls.sum().backward()
    return lls.detach(), logits.grad


@pytest.mark.parametrize("num_cats,num_nodes,varied", [(1278, 1, False), (1000, 1, True), (1278, 4, False),
                                                       (1278, 32, False), (43, 2, False)])
def test_soft_evidence_forward_and_evidence_gradient(num_cats, num_nodes, varied, cuda_device):
    torch.manual_seed(4343442)
    B, V = 64, 32
    pc = _poe_circuit(V, num_cats, num_nodes, cuda_device, scale_first=500 if varied else None)
    data = torch.randint(0, num_cats, [B, V], device=cuda_device)
    logits = torch.rand([B, V, num_cats], device=cuda_device) * 2 - 1
    add = None
    if varied:
        add = torch.zeros_like(logits)
        add[:, :, :500] = math.log(3)
    target_lls, target_grad = _target(data, logits, add)
    lls = pc(data, categorical_evidence_logp=logits)
    assert torch.all((lls.view(-1) - target_lls).abs() / V < 1e-3)
    grad = torch.zeros_like(logits)
    pc.backward(data, allow_modify_flows=False, logspace_flows=True, categorical_evidence_logp=logits,
                categorical_evidence_logp_grad=grad)
    assert torch.all((grad - target_grad).abs() < 1e-5)
    # linear-space flows give the same gradient
    grad2 = torch.zeros_like(logits)
    pc.backward(data, allow_modify_flows=False, logspace_flows=False, categorical_evidence_logp=logits,
                categorical_evidence_logp_grad=grad2)
    assert torch.all((grad2 - target_grad).abs() < 1e-5)


def test_sparse_evidence_equals_dense(cuda_device):
    """Evidence given as (category id, log-weight) entries, in a shuffled order, gives the
    forward values and (permuted) gradients of the dense evidence over all categories."""
    torch.manual_seed(7)
    B, V, K = 48, 8, 40
    pc = _poe_circuit(V, K, 4, cuda_device, scale_first=10)
    data = torch.randint(0, K, [B, V], device=cuda_device)
    logits = torch.randn([B, V, K], device=cuda_device)
    perm = torch.stack([torch.stack([torch.randperm(K) for _ in range(V)]) for _ in range(B)]).to(cuda_device)
    sp_logits = logits.gather(2, perm)
    lls_d = pc(data, categorical_evidence_logp=logits)
    nm_d = pc.node_mars.clone()
    lls_s = pc(data, categorical_evidence_logp=sp_logits, soft_evidence_cat_ids=perm)
    assert torch.allclose(lls_s, lls_d, rtol=1e-5, atol=1e-4)
    lo, hi = pc.input_layer_group[0]._output_ind_range
    assert torch.allclose(pc.node_mars[lo:hi], nm_d[lo:hi], rtol=1e-5, atol=1e-5)
    g_d = torch.zeros_like(logits)
    pc(data, categorical_evidence_logp=logits)
    pc.backward(data, allow_modify_flows=False, logspace_flows=True, categorical_evidence_logp=logits,
                categorical_evidence_logp_grad=g_d)
    g_s = torch.zeros_like(logits)
    pc(data, categorical_evidence_logp=sp_logits, soft_evidence_cat_ids=perm)
    pc.backward(data, allow_modify_flows=False, logspace_flows=True, categorical_evidence_logp=sp_logits,
                soft_evidence_cat_ids=perm, categorical_evidence_logp_grad=g_s)
    assert torch.allclose(g_s, g_d.gather(2, perm), rtol=1e-4, atol=1e-6)


def test_soft_evidence_parameter_flows_and_em(cuda_device):
    """The parameter flows are the categorical histogram of the observed categories weighted by
    node flows, and the EM step is the Categorical's: same results as a Categorical layer of
    the same circuit and parameters fed the same data."""
    torch.manual_seed(3)
    B, V, K = 64, 6, 12
    out = []
    for dist in (dists.SoftEvidenceCategorical, dists.Categorical):
        torch.manual_seed(5)
        nis = [juice.inputs(v, num_nodes=4, dist=dist(num_cats=K)) for v in range(V)]
        ns = juice.summate(juice.multiply(*nis), num_nodes=1)
        pc = juice.compile(ns).to(cuda_device)
        out.append(pc)
    poe, cat = out
    with torch.no_grad():
        poe.params.copy_(cat.params)
        poe.input_layer_group[0].params.copy_(cat.input_layer_group[0].params)
    data = torch.randint(0, K, [B, V], device=cuda_device)
    zero = torch.zeros([B, V, K], device=cuda_device)  # uniform evidence: the node values are log theta[x]
    for pc, kw in ((poe, dict(categorical_evidence_logp=zero)), (cat, {})):
        pc.init_param_flows(flows_memory=0.0)
        lls = pc(data, **kw)
        lls.mean().backward()
        pc.mini_batch_em(step_size=0.2, pseudocount=0.05)
    assert torch.allclose(poe.input_layer_group[0].param_flows, cat.input_layer_group[0].param_flows, rtol=1e-5,
                          atol=1e-7)
    assert torch.allclose(poe.params, cat.params, rtol=1e-5, atol=1e-7)
    assert torch.allclose(poe.input_layer_group[0].params, cat.input_layer_group[0].params, rtol=1e-5, atol=1e-7)


def test_soft_evidence_needs_evidence(cuda_device):
    pc = _poe_circuit(4, 8, 1, cuda_device)
    with pytest.raises(ValueError):
        pc(torch.zeros([4, 4], dtype=torch.long, device=cuda_device))
    with pytest.raises(ValueError):  # more categories than the nodes have
        pc(torch.zeros([4, 4], dtype=torch.long, device=cuda_device),
           categorical_evidence_logp=torch.zeros([4, 4, 9], device=cuda_device))


def test_soft_evidence_sampling(cuda_device):
    """Samples follow the evidence-weighted distribution (the reference's test: evidence
    concentrated on category 10 makes more than 80 % of the draws 10), and with a table of
    uniforms each draw is the first category whose cumulative tilted probability exceeds
    its uniform (checked against a float64 restatement)."""
    torch.manual_seed(11)
    B, K = 64, 43
    ni0 = juice.inputs(0, num_nodes=1, dist=dists.SoftEvidenceCategorical(num_cats=K))
    ni1 = juice.inputs(1, num_nodes=1, dist=dists.SoftEvidenceCategorical(num_cats=K))
    ns = juice.summate(juice.multiply(ni0, ni1), num_nodes=1)
    ns.init_parameters(perturbation=0.0)
    pc = juice.compile(ns).to(cuda_device)
    probs = torch.rand([B, 2, K], device=cuda_device)
    probs /= probs.sum(dim=2, keepdim=True)
    probs *= 0.1
    probs[:, :, 10] += 0.9
    logits = probs.log()
    samples = juice.queries.sample(pc, num_samples=B, categorical_evidence_logp=logits)
    assert (samples == 10).float().mean() > 0.8
    # exact draws under a uniform table
    u = torch.rand([pc.num_nodes, B], device=cuda_device)
    samples = juice.queries.sample(pc, num_samples=B, categorical_evidence_logp=logits, uniforms=u)
    layer = pc.input_layer_group[0]
    lo = layer._output_ind_range[0]
    for n in range(2):
        v, sp = int(layer.vids[n, 0]), int(layer.s_pids[n])
        theta = layer.params[sp:sp + K].double()
        w = theta[None, :] * logits[:, v, :].double().exp()
        cum = (w / w.sum(dim=1, keepdim=True)).cumsum(dim=1)
        expect = (cum <= u[lo + n][:, None].double()).sum(dim=1).clamp(max=K - 1)
        agree = (samples[:, v] == expect).float().mean()
        assert agree >= 0.98  # a uniform within rounding of a cumulative boundary may differ
    with pytest.raises(ValueError):
        juice.queries.sample(pc, num_samples=B)


@pytest.mark.parametrize("name", ["bern", "dlog"])
def test_bernoulli_and_discrete_logistic_sampling_marginals(name, cuda_device):
    """Samples of a circuit over Bernoulli (DiscreteLogistic) inputs: the frequency of each
    value of each variable matches the circuit's own marginal probability of that value
    (the forward pass with the other variables missing), within 0.015 at 40,000 samples; the
    result has the inputs' data type."""
    torch.manual_seed(2)
    factory = (lambda: dists.Bernoulli()) if name == "bern" else \
        (lambda: dists.DiscreteLogistic(val_range=(-2.0, 2.0), num_cats=8))
    pc = juice.compile(build_dist_dag(juice, factory)).to(cuda_device)
    S = 40000
    samples = juice.queries.sample(pc, num_samples=S, seed=5)
    assert samples.dtype == (torch.bool if name == "bern" else torch.float32)
    values = [0, 1] if name == "bern" else list(range(8))
    for v in range(4):
        mask = torch.ones([len(values), 4], dtype=torch.bool, device=cuda_device)
        mask[:, v] = False
        x = torch.zeros([len(values), 4], dtype=torch.float32, device=cuda_device)
        x[:, v] = torch.tensor(values, dtype=torch.float32, device=cuda_device)
        with torch.no_grad():
            p = pc(x if name != "bern" else x.bool(), missing_mask=mask).exp().view(-1)
        assert abs(float(p.sum()) - 1.0) < 1e-4
        col = samples[:, v].float()
        freq = torch.stack([(col == val).float().mean() for val in values])
        assert (freq - p).abs().max() < 0.015


def test_gaussian_sampling_moments(cuda_device):
    """Gaussian inputs: with every sum weight on one child (a single mixture component per
    variable), the samples of each variable have that component's mean and deviation."""
    torch.manual_seed(4)
    pc = juice.compile(build_dist_dag(juice, lambda: dists.Gaussian(mu=0.0, sigma=1.0))).to(cuda_device)
    S = 40000
    samples = juice.queries.sample(pc, num_samples=S, seed=9)
    assert samples.dtype == torch.float32 and torch.isfinite(samples).all()
    # the sample mean of each variable is the marginal mean sum_n P(node n active) mu_n, which
    # lies inside the range of the variable's node means
    layer = pc.input_layer_group[0]
    prm = layer.params[:2 * layer.num_nodes].view(-1, 2)
    for v in range(4):
        nodes = (layer.vids[:, 0] == v).nonzero().view(-1)
        mus = prm[layer.s_pids[nodes].long() // 2, 0]
        m = samples[:, v].mean()
        assert float(mus.min()) - 0.05 <= float(m) <= float(mus.max()) + 0.05
