"""Parity of the backward pass and the EM update against the FP64 oracle and the reference's
own outputs, in every precision form the EM step runs in:

* HCLT over 28x28 variables, 256 categories, 128 latents, block size 32 (the benchmarked
  circuit) at batch 32: node flows, parameter flows, input flows and the EM update, for
  plain FP32 and the two BF16 tensor-core forms (split hi + lo operands, single operands),
  through the tcgen05 kernels of the large layers in both element-flow modes;
* keep_zero_params EM and the device normalisation against the reference's outputs;
* non-uniform root weights (``ll_weights``), the FP64 dataset log-likelihood reducer and
  FP64 epoch-level parameter flows against the oracle.

Error bounds, relative to the largest magnitude of the compared quantity: FP32 1e-3 (node
values of this circuit are log-likelihoods near -3000 nats, where one FP32 ulp is 2.4e-4, so
every exp(element value - node value) carries that relative error); split
BF16 2e-3; single BF16 5e-2 (its operands keep 8 mantissa bits).
"""

import numpy as np
import pytest
import torch

from conftest import load_fixture
from helpers import build_fixture_circuit, fixture_params, load_fixture_params
from oracle import pc_oracle as orc

import pyjuice_b200 as juice
from pyjuice_b200.layer.layers import SumLayer
from pyjuice_b200.synthetic import gaussian_field_data

pytestmark = pytest.mark.gpu

FORMS = {"fp32": (0, 1e-3), "bf16_split": (2, 2e-3), "bf16_single": (1, 5e-2)}
_CACHE = {}


def _hclt784(device):
    """The benchmarked circuit with the fixture's seeded parameters, its oracle layout and a
    batch of 32 quantised random fields (compiled once per module)."""
    if "pc" not in _CACHE:
        fx = load_fixture("hclt784")
        pc = build_fixture_circuit("hclt784", fx)
        p0, q0 = fixture_params(pc, fx)
        x = gaussian_field_data(32, side=28, num_cats=256, length_scale=3.0, seed=1).numpy()
        lay = orc.layout_from_circuit(pc)
        nm, ems, lls = orc.forward(lay, p0, q0, x)
        nf, pf, ipf = orc.backward(lay, p0, x, nm, ems)
        _CACHE.update(pc=pc, fx=fx, p0=p0, q0=q0, x=x, lay=lay, lls=lls, nf=nf, pf=pf, ipf=ipf)
    c = _CACHE
    pc = c["pc"].to(device)
    load_fixture_params(pc, c["fx"])
    return pc, c


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("form", list(FORMS))
@pytest.mark.parametrize("modify", [True, False])
def test_hclt784_flows_and_em_vs_fp64(form, modify, cuda_device):
    bf16_form, tol = FORMS[form]
    pc, c = _hclt784(cuda_device)
    x = torch.from_numpy(c["x"]).to(cuda_device)
    kw = {"force_use_fp32": True} if bf16_form == 0 else {"force_use_bf16": True}
    saved = SumLayer.bf16_form
    try:
        if bf16_form:
            SumLayer.bf16_form = bf16_form
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            lls = pc(x, **kw)
        pc.backward(inputs=x, allow_modify_flows=modify, force_use_fp32=bf16_form == 0)
        torch.cuda.synchronize()
    finally:
        SumLayer.bf16_form = saved
    # the large layers ran on the tcgen05 kernels in the BF16 forms (element-flow mode 1 when
    # the node flows are rewritten in place, mode 2 when they are not)
    if bf16_form:
        assert any(l._fw_tc05(l._desc(cuda_device), 32, True, False)[1]
                   for g in pc.inner_layer_groups if g.is_sum() for l in g)
    dll = np.abs(lls.cpu().numpy() - c["lls"])
    if bf16_form == 0:
        assert np.all(dll <= 1e-5 * np.abs(c["lls"]))
    else:  # mean absolute LL error in nats
        assert dll.mean() <= (1e-3 if bf16_form == 2 else 5e-2)
    assert _rel(pc.param_flows.cpu().numpy(), c["pf"]) <= tol
    il = pc.input_layer_group[0]
    ipf = c["ipf"]
    assert _rel(il.param_flows.cpu().numpy()[:ipf.shape[0]], ipf) <= tol
    lo, hi = il._output_ind_range
    assert _rel(pc.node_flows[lo:hi].cpu().numpy(), c["nf"][lo:hi]) <= tol
    if not modify:  # no row was rewritten: every node flow is comparable
        assert _rel(pc.node_flows.cpu().numpy(), c["nf"]) <= tol
    # EM from the device flows equals the oracle's EM from the same flows (FP64 update), and
    # stays within the flow bound of the EM from the oracle's own flows
    gpf = pc.param_flows.cpu().numpy().astype(np.float64)
    gipf = il.param_flows.cpu().numpy()[:ipf.shape[0]].astype(np.float64)
    pc.mini_batch_em(step_size=0.1, pseudocount=0.1)
    p1, q1 = orc.em_update(c["lay"], c["p0"], gpf, c["q0"], gipf, 0.1, 0.1)
    assert np.abs(pc.params.cpu().numpy() - p1).max() <= 1e-6
    assert np.abs(il.params.cpu().numpy()[:q1.shape[0]] - q1).max() <= 1e-6
    p1o, _ = orc.em_update(c["lay"], c["p0"], c["pf"], c["q0"], c["ipf"], 0.1, 0.1)
    assert np.abs(pc.params.cpu().numpy() - p1o).max() <= max(tol, 1e-5)


def test_keep_zero_em_matches_reference(cuda_device):
    fx = load_fixture("em_tiny")
    pc = build_fixture_circuit("tiny", load_fixture("tiny")).to(cuda_device)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(fx["params0"]).to(cuda_device))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(fx["in_params0"]).to(cuda_device))
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, force_use_fp32=True)
    lls.mean().backward()
    assert _rel(pc.param_flows.cpu().numpy(), fx["param_flows"]) <= 1e-4
    pc.mini_batch_em(step_size=0.1, pseudocount=0.1, keep_zero_params=True)
    got = pc.params.cpu().numpy()
    assert np.abs(got - fx["params1_keep_zero"]).max() <= 1e-5
    assert np.all(got[fx["params0"] == 0] == 0)
    ip = pc.input_layer_group[0].params.cpu().numpy()[:fx["in_params1_keep_zero"].shape[0]]
    assert np.abs(ip - fx["in_params1_keep_zero"]).max() <= 1e-5
    assert np.all(ip[fx["in_params0"] == 0] == 0)


def test_normalize_parameters_matches_reference(cuda_device):
    fx = load_fixture("em_tiny")
    pc = build_fixture_circuit("tiny", load_fixture("tiny")).to(cuda_device)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(fx["norm_in"]).to(cuda_device))
    pc.normalize_parameters(pseudocount=0.3)
    assert np.abs(pc.params.cpu().numpy() - fx["norm_out"]).max() <= 1e-6


def test_nonuniform_ll_weights(cuda_device):
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    B = 200
    xn = fx["x"][:B]
    x = torch.from_numpy(xn).to(cuda_device)
    w = np.random.default_rng(3).uniform(0.1, 3.0, size=(1, B))
    lay = orc.layout_from_circuit(pc)
    nm, ems, _ = orc.forward(lay, fx["params0"], fx["in_params0"], xn)
    _, pf, ipf = orc.backward(lay, fx["params0"], xn, nm, ems, ll_weights=w)
    pc.init_param_flows(flows_memory=0.0)
    with torch.no_grad():
        pc(x, force_use_fp32=True)
    pc.backward(inputs=x, ll_weights=torch.from_numpy(w).float().to(cuda_device), force_use_fp32=True)
    assert _rel(pc.param_flows.cpu().numpy(), pf) <= 1e-4
    assert _rel(pc.input_layer_group[0].param_flows.cpu().numpy()[:ipf.shape[0]], ipf) <= 1e-4
    # lls.mean().backward() normalises the weights to sum to the batch size (all ones here)
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, force_use_fp32=True)
    (lls * torch.from_numpy(w.T).float().to(cuda_device)).sum().backward()
    _, pf_n, _ = orc.backward(lay, fx["params0"], xn, nm, ems, ll_weights=w / w.sum() * B)
    assert _rel(pc.param_flows.cpu().numpy(), pf_n) <= 1e-4


def test_dataset_ll_accumulate_fp64(cuda_device):
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    acc = torch.zeros([], dtype=torch.float64, device=cuda_device)
    total = 0.0
    for b0 in range(0, 512, 128):
        x = torch.from_numpy(fx["x"][b0:b0 + 128]).to(cuda_device)
        with torch.no_grad():
            lls = pc(x, force_use_fp32=True)
        pc.dataset_ll_accumulate(lls, acc)
        total += lls.double().sum().item()
    assert abs(acc.item() - total) <= 1e-9 * abs(total)


def test_fp64_epoch_flows_and_em(cuda_device):
    """Three batches: the FP64 epoch flows equal the sum of each batch's flows (oracle), and
    EM from them equals the oracle's EM from the summed flows."""
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    lay = orc.layout_from_circuit(pc)
    pc.init_param_flows_f64()
    pf_sum, ipf_sum = 0.0, 0.0
    for b0 in (0, 100, 300):
        xn = fx["x"][b0:b0 + 100]
        nm, ems, _ = orc.forward(lay, fx["params0"], fx["in_params0"], xn)
        _, pf, ipf = orc.backward(lay, fx["params0"], xn, nm, ems)
        pf_sum, ipf_sum = pf_sum + pf, ipf_sum + ipf
        x = torch.from_numpy(xn).to(cuda_device)
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            pc(x, force_use_fp32=True)
        pc.backward(inputs=x, force_use_fp32=True)
        pc.accumulate_param_flows_f64()
    assert pc.param_flows_f64.dtype == torch.float64
    assert _rel(pc.param_flows_f64.cpu().numpy(), pf_sum) <= 1e-4
    il = pc.input_layer_group[0]
    assert _rel(il.param_flows_f64.cpu().numpy()[:ipf_sum.shape[0]], ipf_sum) <= 1e-4
    gpf = pc.param_flows_f64.cpu().numpy()
    gipf = il.param_flows_f64.cpu().numpy()[:ipf_sum.shape[0]]
    pc.mini_batch_em(step_size=1.0, pseudocount=0.1, use_f64_flows=True)
    p1, q1 = orc.em_update(lay, fx["params0"], gpf, fx["in_params0"], gipf, 1.0, 0.1)
    assert np.abs(pc.params.cpu().numpy() - p1).max() <= 1e-6
    assert np.abs(il.params.cpu().numpy()[:q1.shape[0]] - q1).max() <= 1e-6


def test_cumulate_flows_fp64_matches_fp32_accumulation(cuda_device):
    """cumulate_flows(fp64=True) over batches gives the same epoch flows as the reference's
    FP32 accumulation (flows_memory=1), up to FP32 rounding of the latter."""
    fx = load_fixture("hclt64")
    out = []
    for fp64 in (False, True):
        pc = build_fixture_circuit("hclt64", fx).to(cuda_device)
        load_fixture_params(pc, fx)
        pc.init_param_flows(flows_memory=0.0)
        if fp64:
            pc.init_param_flows_f64()
        for b0 in (0, 128, 256, 384):
            pc.cumulate_flows(torch.from_numpy(fx["x"][b0:b0 + 128]).to(cuda_device), fp64=fp64)
        out.append((pc.param_flows_f64 if fp64 else pc.param_flows).double().cpu().numpy())
    assert _rel(out[1], out[0]) <= 1e-5


ALG_CASES = [("mpe", "MPE", 1.0, False, False), ("gll", "GeneralLL", 0.5, False, False),
             ("logspace", "LL", 1.0, True, False), ("negate", "LL", 1.0, False, True)]


@pytest.mark.parametrize("case", ALG_CASES, ids=[c[0] for c in ALG_CASES])
def test_propagation_algorithms_match_reference(case, cuda_device):
    """MPE / GeneralLL forward and backward, log-space flows and negated parameter flows on
    the tiny circuit (partitions, sparse edges, ties, pass-through) against the reference's
    own outputs (alg_tiny.npz), through the public API."""
    name, alg, alpha, logspace, negate = case
    fx = load_fixture("tiny")
    ref = load_fixture("alg_tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    fw = dict(propagation_alg=alg) if alg == "MPE" else (dict(propagation_alg=alg, alpha=alpha) if alg != "LL" else {})
    pc.init_param_flows(flows_memory=0.0)
    with torch.no_grad():
        lls = pc(x, force_use_fp32=True, **fw)
    pc.backward(inputs=x, allow_modify_flows=False, force_use_fp32=True, logspace_flows=logspace,
                negate_pflows=negate, **fw)
    rl = ref[name + "_lls"]
    assert np.all(np.abs(lls.cpu().numpy() - rl) <= 1e-5 * np.abs(rl) + 1e-6)
    assert _rel(pc.param_flows.cpu().numpy(), ref[name + "_param_flows"]) <= 1e-4
    ripf = ref[name + "_in_param_flows"]
    assert _rel(pc.input_layer_group[0].param_flows.cpu().numpy()[:ripf.shape[0]], ripf) <= 1e-4
    rnf = ref[name + "_node_flows"]
    nf = pc.node_flows.cpu().numpy()
    fin = np.isfinite(rnf)
    assert np.array_equal(fin, np.isfinite(nf))
    assert np.abs(nf[fin] - rnf[fin]).max() <= 1e-4 * max(1.0, np.abs(rnf[fin]).max())


def test_set_propagation_alg_and_forward_mpe(cuda_device):
    fx = load_fixture("tiny")
    ref = load_fixture("alg_tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    with torch.no_grad():
        a = pc.forward_mpe(x, force_use_fp32=True).cpu().numpy()
        pc.set_propagation_alg("GeneralLL", alpha=0.5)
        b = pc(x, force_use_fp32=True).cpu().numpy()
        pc.set_propagation_alg("LL")
    assert np.abs(a - ref["mpe_lls"]).max() <= 1e-4
    assert np.abs(b - ref["gll_lls"]).max() <= 1e-4
    with pytest.raises(ValueError):
        pc.set_propagation_alg("GeneralLL")


@pytest.mark.parametrize("tkc", [64, 128])
@pytest.mark.parametrize("modified", [True, False])
@pytest.mark.parametrize("form", [2, 1])
def test_pflows_tc05_matches_mma_sync(tkc, modified, form, cuda_device):
    """The tcgen05 parameter-flow kernel (accumulators in tensor memory) against the warp-level
    mma.sync kernel on every sum layer of the 28x28 circuit at batch 96 (a partial last
    chunk), for 64- and 128-child tiles, rewritten and raw node flows, both BF16 forms."""
    pc, c = _hclt784(cuda_device)
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.integers(0, 256, size=(96, 784))).to(cuda_device)
    saved = (SumLayer.pflow_tc05, SumLayer.pflow_tile_children, SumLayer.bf16_form)
    try:
        SumLayer.bf16_form = form
        SumLayer.pflow_tile_children = tkc
        with torch.no_grad():
            pc(x, force_use_bf16=True)
        pc.init_param_flows(flows_memory=0.0)
        pc.backward(inputs=x, allow_modify_flows=False, compute_param_flows=False)
        nfl = pc.node_flows
        if modified:  # the kernels' other input form: log f - log m
            nfl = torch.where(torch.isinf(pc.node_mars), torch.full_like(nfl, -float("inf")),
                              torch.log(pc.node_flows) - pc.node_mars)
        torch.cuda.synchronize()
        out = []
        for tc05 in (False, True):
            SumLayer.pflow_tc05 = tc05
            pf = torch.zeros_like(pc.param_flows)
            for gi, g in enumerate(pc.inner_layer_groups):
                if g.is_sum():
                    for layer in g:
                        layer.param_flows_only(nfl, pc.node_mars, pc._em_view(gi - 1), pc.params, pf,
                                               allow_modify_flows=modified)
            torch.cuda.synchronize()
            out.append(pf.double().cpu().numpy())
    finally:
        SumLayer.pflow_tc05, SumLayer.pflow_tile_children, SumLayer.bf16_form = saved
    ref, got = out
    assert np.isfinite(got).all()
    assert np.abs(got - ref).max() <= (1e-5 if form == 2 else 1e-2) * np.abs(ref).max()


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_top_down_probs_and_step_size_rescaling(name, cuda_device):
    """Top-down probabilities (node flows of the evidence-free pass, oracle pinned to the
    reference's flows) and one mini-batch EM step with step-size rescaling
    (tensorcircuit.py:566-590) against the oracle."""
    from pyjuice_b200.model.top_down import eval_top_down_probs
    fx = load_fixture(name)
    pc = build_fixture_circuit(name, fx).to(cuda_device)
    load_fixture_params(pc, fx)
    lay = orc.layout_from_circuit(pc)
    p0, q0 = fx["params0"], fx["in_params0"]
    V = pc.num_vars
    z, miss = np.zeros([1, V], dtype=np.int64), np.ones(V, dtype=bool)
    nm, ems, _ = orc.forward(lay, p0, q0, z, missing_mask=miss)
    tdp, tdp_pf, tdp_ipf = orc.backward(lay, p0, z, nm, ems, missing_mask=miss, in_params=q0)
    pc.init_param_flows(flows_memory=0.0)
    eval_top_down_probs(pc, update_pflow=True, scale=0.5)
    assert np.abs(pc._single_node_flows.cpu().numpy() - tdp[:, 0]).max() <= 1e-5
    assert _rel(pc.param_flows.cpu().numpy(), 0.5 * tdp_pf) <= 1e-4
    il = pc.input_layer_group[0]
    assert _rel(il.param_flows.cpu().numpy()[:tdp_ipf.shape[0]], 0.5 * tdp_ipf) <= 1e-4
    # a batch, then EM with the step rescaled by the batch's root flow
    B = min(64, fx["x"].shape[0])
    xb = fx["x"][:B]
    nmb, emb, _ = orc.forward(lay, p0, q0, xb)
    _, pf, ipf = orc.backward(lay, p0, xb, nmb, emb)
    pc.init_param_flows(flows_memory=0.0)
    pc._cum_flow_dev = None
    lls = pc(torch.from_numpy(xb).to(cuda_device), force_use_fp32=True)
    lls.mean().backward()
    pc.mini_batch_em(step_size=0.3, pseudocount=0.1, step_size_rescaling=True)
    s = 0.3
    p1, q1 = orc.em_update(lay, p0, pf * (s / B) + (1 - s) * tdp_pf, q0, ipf * (s / B) + (1 - s) * tdp_ipf, 1.0, 0.1)
    assert np.abs(pc.params.cpu().numpy() - p1).max() <= 1e-4
    assert np.abs(il.params.cpu().numpy()[:q1.shape[0]] - q1).max() <= 1e-4
    assert pc._cum_flow == 0.0


def test_pd_and_hmm_match_reference(cuda_device):
    """The PD and homogeneous-HMM circuits (tied transition and emission vectors) through the
    device kernels against the reference's own outputs (structures.npz): FP32 log-likelihoods,
    flows and one EM step of the HMM."""
    fx = load_fixture("structures")
    sub = lambda p: {k[len(p):]: v for k, v in fx.items() if k.startswith(p)}
    pd = sub("pd_")
    torch.manual_seed(7)
    pc = juice.compile(juice.structures.PD((3, 3), 32, split_intervals=1, max_prod_block_conns=2,
                                           input_dist=juice.distributions.Categorical(num_cats=4))).to(cuda_device)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(pd["params"]).to(cuda_device))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(pd["in_params"]).to(cuda_device))
        lls = pc(torch.from_numpy(pd["x"]).to(cuda_device), force_use_fp32=True).cpu().numpy()
    assert np.all(np.abs(lls - pd["lls"]) <= 1e-5 * np.abs(pd["lls"]) + 1e-6)
    hm = sub("hmm_")
    pc = juice.compile(juice.structures.HMM(6, 32, 10, alpha=torch.from_numpy(hm["alpha"]),
                                            beta=torch.from_numpy(hm["beta"]),
                                            gamma=torch.from_numpy(hm["gamma"]))).to(cuda_device)
    x = torch.from_numpy(hm["x"]).to(cuda_device)
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, force_use_fp32=True)
    assert np.all(np.abs(lls.detach().cpu().numpy() - hm["lls"]) <= 1e-5 * np.abs(hm["lls"]) + 1e-6)
    lls.mean().backward()
    assert _rel(pc.param_flows.cpu().numpy(), hm["param_flows"]) <= 1e-4
    ipf = hm["in_param_flows"]
    assert _rel(pc.input_layer_group[0].param_flows.cpu().numpy()[:ipf.shape[0]], ipf) <= 1e-4
    pc.mini_batch_em(step_size=0.5, pseudocount=0.01)
    assert np.abs(pc.params.cpu().numpy() - hm["params1"]).max() <= 1e-5
    q1 = hm["in_params1"]
    assert np.abs(pc.input_layer_group[0].params.cpu().numpy()[:q1.shape[0]] - q1).max() <= 1e-5


def test_batched_hmms_forest_vs_oracle(cuda_device):
    """Four HMMs of different lengths and hidden sizes in one circuit (batched_hmms): the
    log-likelihood equals the sum of the four HMMs' own (FP64 oracle, each HMM compiled
    alone), and the forest's parameter and input flows match the oracle on the forest."""
    rng = np.random.default_rng(0)
    specs = [(5, 16), (3, 32), (7, 16), (4, 64)]
    V = 12
    params = []
    for T, L in specs:
        params.append(tuple(torch.from_numpy(rng.dirichlet(np.full(n, 0.5), size=m) if m else
                                             rng.dirichlet(np.full(n, 0.5))).float()
                            for m, n in ((L, L), (L, V), (0, L))))
    pc = juice.compile(juice.structures.batched_hmms(specs, V, params=params)).to(cuda_device)
    x = rng.integers(0, V, size=(64, sum(T for T, _ in specs)))
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(torch.from_numpy(x).to(cuda_device), force_use_fp32=True)
    lls.mean().backward()
    lay = orc.layout_from_circuit(pc)
    p0 = pc.params.double().cpu().numpy()
    q0 = pc.input_layer_group[0].params.double().cpu().numpy()
    nm, ems, lls_o = orc.forward(lay, p0, q0, x)
    _, pf_o, ipf_o = orc.backward(lay, p0, x, nm, ems)
    got = lls.detach().double().cpu().numpy()
    assert np.abs(got - lls_o).max() <= 1e-5 * np.abs(lls_o).max()
    assert _rel(pc.param_flows.cpu().numpy(), pf_o) <= 1e-4  # mean-LL gradient: unit root flows
    ipf = pc.input_layer_group[0].param_flows.cpu().numpy()[:ipf_o.shape[0]]
    assert _rel(ipf, ipf_o) <= 1e-4
    ref, off = np.zeros(64), 0
    for (T, L), (a, b, g) in zip(specs, params):
        h = juice.compile(juice.structures.HMM(T, L, V, alpha=a, beta=b, gamma=g, block_size=16))
        hl = orc.layout_from_circuit(h)
        _, _, l1 = orc.forward(hl, h.params.double().numpy(), h.input_layer_group[0].params.double().numpy(),
                               x[:, off:off + T])
        ref += l1[:, 0]
        off += T
    assert np.abs(lls_o[:, 0] - ref).max() <= 1e-9 * np.abs(ref).max()


def test_pd_with_parentless_products_flows_vs_oracle(cuda_device):
    """A PD circuit with products that no sum node selects (max_prod_block_conns = 1): FP32
    parameter and input flows against the FP64 oracle on two consecutive backward passes
    (the parentless elements' flow rows must read as zero in every pass), and the second pass
    equal to the first."""
    torch.manual_seed(7)
    pc = juice.compile(juice.structures.PD((4, 4), 16, split_intervals=1, max_prod_block_conns=1,
                                           input_dist=juice.distributions.Categorical(num_cats=4))).to(cuda_device)
    assert pc._ef_init_ranges
    lay = orc.layout_from_circuit(pc)
    rng = np.random.default_rng(3)
    x = rng.integers(0, 4, size=(64, 16))
    p0 = pc.params.double().cpu().numpy()
    q0 = pc.input_layer_group[0].params.double().cpu().numpy()
    nm, ems, _ = orc.forward(lay, p0, q0, x)
    _, pf_o, ipf_o = orc.backward(lay, p0, x, nm, ems)
    out = []
    for _ in range(2):
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            pc(torch.from_numpy(x).to(cuda_device), force_use_fp32=True)
        pc.backward(inputs=torch.from_numpy(x).to(cuda_device), allow_modify_flows=False, force_use_fp32=True)
        pf = pc.param_flows.double().cpu().numpy()
        ipf = pc.input_layer_group[0].param_flows.double().cpu().numpy()[:ipf_o.shape[0]]
        assert _rel(pf, pf_o) <= 1e-4 and _rel(ipf, ipf_o) <= 1e-4
        out.append((pf, ipf))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("name", ["bern", "gauss", "dlog"])
def test_bernoulli_and_gaussian_layers_match_reference(name, cuda_device):
    """Bernoulli, Gaussian and DiscreteLogistic input layers: FP32 forward, flows and one EM
    step against the reference's own outputs (dists.npz; four-variable circuit, seeded
    parameters and data)."""
    from circuits import build_dist_dag
    fx = load_fixture("dists")
    g = lambda k: fx[f"{name}_{k}"]
    factory = {"bern": lambda: juice.distributions.Bernoulli(),
               "gauss": lambda: juice.distributions.Gaussian(mu=0.0, sigma=1.0),
               "dlog": lambda: juice.distributions.DiscreteLogistic(val_range=(-2.0, 2.0), num_cats=8)}[name]
    pc = juice.compile(build_dist_dag(juice, factory)).to(cuda_device)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(g("params0")).to(cuda_device))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(g("in_params0")).to(cuda_device))
    x = torch.from_numpy(g("x")).to(cuda_device)
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, force_use_fp32=True)
    ref = g("lls")
    assert np.all(np.abs(lls.detach().cpu().numpy() - ref) <= 1e-5 * np.abs(ref) + 1e-5)
    lls.mean().backward()
    assert _rel(pc.param_flows.cpu().numpy(), g("param_flows")) <= 1e-4
    ipf = g("in_param_flows")
    assert _rel(pc.input_layer_group[0].param_flows.cpu().numpy()[:ipf.shape[0]], ipf) <= 1e-4
    pc.mini_batch_em(step_size=0.3, pseudocount=0.1)
    assert np.abs(pc.params.cpu().numpy() - g("params1")).max() <= 1e-5
    q1 = g("in_params1")
    assert np.abs(pc.input_layer_group[0].params.cpu().numpy()[:q1.shape[0]] - q1).max() <= 1e-4 * max(1.0, np.abs(q1).max())


@pytest.mark.parametrize("K,B", [(4096, 64), (4096, 200), (37, 70)])
def test_one_row_sum_forward_vs_oracle(K, B, cuda_device):
    """A block-size-1 sum node over K product children (the one-row FP32 forward kernel: lanes
    over samples, warps over terms, online log-sum-exp): log-likelihoods against the FP64
    oracle, ragged batch, children with -inf values (zero input probabilities) included."""
    torch.manual_seed(5)
    n0 = juice.inputs(0, num_nodes=K, dist=juice.distributions.Categorical(num_cats=4))
    n1 = juice.inputs(1, num_nodes=K, dist=juice.distributions.Categorical(num_cats=4))
    root = juice.summate(juice.multiply(n0, n1), num_nodes=1)
    pc = juice.compile(root)
    with torch.no_grad():
        q = pc.input_layer_group[0].params
        q[: 4 * K: 7] = 0.0  # some categories impossible for some nodes
    pc = pc.to(cuda_device)
    x = np.random.default_rng(2).integers(0, 4, size=(B, 2))
    lls = pc(torch.from_numpy(x).to(cuda_device), force_use_fp32=True).detach().double().cpu().numpy()
    lay = orc.layout_from_circuit(pc)
    _, _, ref = orc.forward(lay, pc.params.double().cpu().numpy(),
                            pc.input_layer_group[0].params.double().cpu().numpy(), x)
    assert np.all(np.abs(lls - ref) <= 1e-5 * np.abs(ref) + 1e-5)
