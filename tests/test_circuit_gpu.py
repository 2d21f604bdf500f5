"""Full-circuit parity on the GPU: CUDA path vs the reference's own outputs (golden
fixtures) and vs the FP64 oracle, through pyjuice_b200's public API."""

import itertools

import numpy as np
import pytest
import torch

from conftest import load_fixture
from helpers import build_fixture_circuit, fixture_params, load_fixture_params
from oracle import pc_oracle as orc

import pyjuice_b200 as juice
from pyjuice_b200 import _native as nat

pytestmark = pytest.mark.gpu

# FP32 plain path vs the reference: per-sample LL within 1e-5 relative.
LL_RTOL = 1e-5


def _step(pc, x, **fw):
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, **fw)
    lls.mean().backward()
    return lls


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_fp32_step_matches_reference(name, cuda_device):
    fx = load_fixture(name)
    torch.manual_seed(0)
    pc = build_fixture_circuit(name, fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    lls = _step(pc, x, force_use_fp32=True)
    ref = fx["lls"]
    got = lls.detach().cpu().numpy()
    assert np.all(np.abs(got - ref) <= LL_RTOL * np.abs(ref) + 1e-6)
    pf = pc.param_flows.cpu().numpy()
    assert np.abs(pf - fx["param_flows"]).max() <= 1e-4 * np.abs(fx["param_flows"]).max()
    ipf = pc.input_layer_group[0].param_flows.cpu().numpy()[: fx["in_param_flows"].shape[0]]
    assert np.abs(ipf - fx["in_param_flows"]).max() <= 1e-4 * np.abs(fx["in_param_flows"]).max()
    pc.mini_batch_em(step_size=0.1, pseudocount=0.1)
    assert np.abs(pc.params.cpu().numpy() - fx["params1"]).max() <= 1e-5
    ip1 = pc.input_layer_group[0].params.cpu().numpy()[: fx["in_params1"].shape[0]]
    assert np.abs(ip1 - fx["in_params1"]).max() <= 1e-5


def test_fp32_node_values_match_reference_tiny(cuda_device):
    fx = load_fixture("tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    with torch.no_grad():
        pc(x, force_use_fp32=True)
    nm = pc.node_mars.cpu().numpy()
    ref = fx["node_mars"]
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(nm), fin)
    assert np.abs(nm[fin] - ref[fin]).max() <= 1e-5 * max(1.0, np.abs(ref[fin]).max())


def test_fp32_hclt784_matches_reference(cuda_device):
    fx = load_fixture("hclt784")
    pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    with torch.no_grad():
        lls = pc(x, force_use_fp32=True).cpu().numpy()
    ref = fx["lls"]
    assert np.all(np.abs(lls - ref) <= LL_RTOL * np.abs(ref))


@pytest.mark.parametrize("B", [1, 3, 17, 64, 200])
def test_fp32_batch_sizes_vs_oracle(B, cuda_device):
    """Ragged batches (not multiples of 4 or of the sample tile) against the oracle."""
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"][:B]).to(cuda_device)
    lay = orc.layout_from_circuit(pc)
    nm, ems, lls_o = orc.forward(lay, fx["params0"], fx["in_params0"], fx["x"][:B])
    lls = _step(pc, x, force_use_fp32=True).detach().cpu().numpy()
    assert np.all(np.abs(lls - lls_o) <= LL_RTOL * np.abs(lls_o))
    _, pf, ipf = orc.backward(lay, fx["params0"], fx["x"][:B], nm, ems)
    assert np.abs(pc.param_flows.cpu().numpy() - pf).max() <= 1e-4 * max(np.abs(pf).max(), 1e-6)
    got_ipf = pc.input_layer_group[0].param_flows.cpu().numpy()[: ipf.shape[0]]
    assert np.abs(got_ipf - ipf).max() <= 1e-4 * max(np.abs(ipf).max(), 1e-6)


def test_probabilities_sum_to_one_tiny(cuda_device):
    fx = load_fixture("tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.tensor(list(itertools.product(range(4), repeat=6)), device=cuda_device)
    with torch.no_grad():
        lls = pc(x, force_use_fp32=True)
    assert abs(lls.double().exp().sum().item() - 1.0) < 1e-5


def test_bf16_forward_error_vs_fp64(cuda_device):
    """BF16 tensor-core form on HCLT-784 (128 latents, block size 32): mean LL within
    1e-3 nats of the FP64 oracle; FP32 form within 1e-5 relative per sample."""
    fx = load_fixture("hclt784")
    pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    lay = orc.layout_from_circuit(pc)
    p0, q0 = fixture_params(pc, fx)
    _, _, lls_o = orc.forward(lay, p0, q0, fx["x"])
    with torch.no_grad():
        lls_bf = pc(x, force_use_bf16=True).double().cpu().numpy()
        lls_32 = pc(x, force_use_fp32=True).double().cpu().numpy()
    assert np.all(np.abs(lls_32 - lls_o) <= LL_RTOL * np.abs(lls_o))
    assert abs(lls_bf.mean() - lls_o.mean()) < 1e-3


def test_bf16_single_operand_form(cuda_device):
    """The single-bf16 variant (one MMA per fragment) stays within its rounding error."""
    from pyjuice_b200.layer.layers import SumLayer
    fx = load_fixture("hclt784")
    pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    p0, q0 = fixture_params(pc, fx)
    _, _, lls_o = orc.forward(orc.layout_from_circuit(pc), p0, q0, fx["x"])
    saved = SumLayer.bf16_form
    try:
        SumLayer.bf16_form = 1
        with torch.no_grad():
            lls = pc(x, force_use_bf16=True).double().cpu().numpy()
    finally:
        SumLayer.bf16_form = saved
    assert np.abs(lls - lls_o).max() < 0.05


def test_cuda_graph_replay_matches_eager(cuda_device):
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    with torch.no_grad():
        eager = pc(x, force_use_fp32=True).clone()
        pc(x, force_use_fp32=True, record_cudagraph=True)
        replay = pc(x, force_use_fp32=True, apply_cudagraph=True)
    assert torch.equal(eager, replay)


def test_recorded_backward_matches_eager(cuda_device):
    """A backward pass recorded as a CUDA graph (through the autograd hook) leaves the same node
    and parameter flows as the eager pass, including flows kept from an earlier batch
    (flows_memory=1) and after EM steps have moved the parameters away from their start."""
    fx = load_fixture("hclt784")
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    out = []
    for rec in (False, True):
        pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
        load_fixture_params(pc, fx)
        for _ in range(3):
            _step(pc, x, force_use_fp32=True)
            pc.mini_batch_em(step_size=0.5, pseudocount=0.01)
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            pc(x, force_use_fp32=True)
        pc.backward(inputs=x, allow_modify_flows=True, force_use_fp32=True)
        pc._optim_hyperparams["flows_memory"] = 1.0
        lls = pc(x, force_use_bf16=True, record_cudagraph=rec)
        lls.mean().backward()
        torch.cuda.synchronize()
        out.append((pc.node_flows.clone(), pc.param_flows.clone()))
    (nf_e, pf_e), (nf_r, pf_r) = out
    assert torch.isfinite(pf_r).all()
    assert torch.equal(nf_e, nf_r)
    assert torch.equal(pf_e, pf_r)


def test_tc05_multi_slice_equals_per_slice(cuda_device):
    """On HCLT-784 at batch 128 (two 64-sample slices per tile), tcgen05 CTAs that walk both
    slices (loading the second while the first is processed) give the same node values,
    node flows and parameter flows as one CTA per slice, and the log-likelihoods stay within
    1e-3 nats of the FP64 oracle."""
    from pyjuice_b200.layer.layers import SumLayer
    fx = load_fixture("hclt784")
    rng = np.random.default_rng(11)
    xn = rng.integers(0, 256, size=(128, 784))
    x = torch.from_numpy(xn).to(cuda_device)
    saved = SumLayer.tc05_slices_per_cta
    out = []
    try:
        for spc in (1, 2):
            SumLayer.tc05_slices_per_cta = spc
            pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
            load_fixture_params(pc, fx)
            pc.init_param_flows(flows_memory=0.0)
            with torch.no_grad():
                lls = pc(x, force_use_bf16=True)
            pc.backward(inputs=x, allow_modify_flows=True)
            torch.cuda.synchronize()
            out.append((lls.clone(), pc.node_mars.clone(), pc.node_flows.clone(), pc.param_flows.clone()))
    finally:
        SumLayer.tc05_slices_per_cta = saved
    for a, b in zip(out[0], out[1]):
        assert torch.equal(a, b)
    p0, q0 = fixture_params(pc, fx)
    _, _, lls_o = orc.forward(orc.layout_from_circuit(pc), p0, q0, xn[:16])
    assert abs(out[1][0][:16].double().cpu().numpy().mean() - lls_o.mean()) < 1e-3


@pytest.mark.parametrize("name,B,kw", [("hclt64", 100, dict(force_use_fp32=True)),
                                       ("hclt784", 256, dict(force_use_bf16=True))])
def test_persistent_small_levels_forward_equals_per_level(name, B, kw, cuda_device):
    """The forward of the run of small levels in one persistent launch (pcb_lse_levels_short:
    per-slice completion counters instead of one product and one sum launch per level)
    gives bit-identical log-likelihoods, node values, element values, flows and EM
    parameters, with a clean device status word (no wait ran out)."""
    from pyjuice_b200.model.tensorcircuit import TensorCircuit
    fx = load_fixture(name)
    rng = np.random.default_rng(8)
    ncat = 4 if name == "hclt64" else 256
    nvar = 64 if name == "hclt64" else 784
    x = torch.from_numpy(rng.integers(0, ncat, size=(B, nvar))).to(cuda_device)
    saved = TensorCircuit.fuse_levels_forward
    out = []
    try:
        for on in (False, True):
            TensorCircuit.fuse_levels_forward = on
            pc = build_fixture_circuit(name, fx).to(cuda_device)
            load_fixture_params(pc, fx)
            if on:
                assert len(pc._level_run(B, kw.get("force_use_bf16", False), kw.get("force_use_fp32", False))) >= 2
            nat.device_status(clear=True)
            pc.init_param_flows(flows_memory=0.0)
            with torch.no_grad():
                lls = pc(x, **kw)
            pc.backward(inputs=x, allow_modify_flows=True, force_use_fp32="force_use_fp32" in kw)
            pc.mini_batch_em(step_size=0.1, pseudocount=0.1)
            torch.cuda.synchronize()
            assert nat.device_status(clear=True) == 0
            out.append((lls.clone(), pc.node_mars.clone(), pc._em_resident.clone(), pc.node_flows.clone(),
                        pc.param_flows.clone(), pc.params.clone()))
    finally:
        TensorCircuit.fuse_levels_forward = saved
    for a, b in zip(out[0], out[1]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("name,B,kw", [("hclt64", 64, dict(force_use_fp32=True)),
                                       ("hclt784", 128, dict(force_use_bf16=True))])
def test_recomputed_element_values_equal_resident(name, B, kw, cuda_device):
    """``recompute_element_values``: the element values share element_mars and the backward
    pass recomputes each product group's values before the sum group above it (no resident
    buffer is allocated); LLs, node flows and parameter flows are bit-identical to the
    resident default, and one EM step gives the same parameters."""
    fx = load_fixture(name)
    rng = np.random.default_rng(4)
    ncat = 4 if name == "hclt64" else 256
    nvar = 64 if name == "hclt64" else 784
    x = torch.from_numpy(rng.integers(0, ncat, size=(B, nvar))).to(cuda_device)
    out = []
    for recompute in (False, True):
        pc = build_fixture_circuit(name, fx).to(cuda_device)
        load_fixture_params(pc, fx)
        pc.recompute_element_values = recompute
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            lls = pc(x, **kw)
        pc.backward(inputs=x, allow_modify_flows=True, force_use_fp32="force_use_fp32" in kw)
        pc.mini_batch_em(step_size=0.1, pseudocount=0.1)
        torch.cuda.synchronize()
        assert ("_em_resident" in pc.__dict__) != recompute
        out.append((lls.clone(), pc.node_flows.clone(), pc.param_flows.clone(), pc.params.clone()))
    for a, b in zip(out[0], out[1]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("modify", [True, False])
def test_tc05_persistent_equals_per_slice(modify, cuda_device):
    """On HCLT-784 at batch 256, the persistent warp-specialised tcgen05 kernel (TMA-staged
    child rows, every layer of >= 6 tiles) gives bit-identical node values, node flows and
    parameter flows to the CTA-per-slice kernel, with modified (mode 1) and unmodified
    (mode 2) node flows."""
    from pyjuice_b200.layer.layers import SumLayer
    fx = load_fixture("hclt784")
    rng = np.random.default_rng(12)
    x = torch.from_numpy(rng.integers(0, 256, size=(256, 784))).to(cuda_device)
    saved = SumLayer.tc05_ws
    out = []
    try:
        for ws in (False, True):
            SumLayer.tc05_ws = ws
            pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
            load_fixture_params(pc, fx)
            pc.init_param_flows(flows_memory=0.0)
            with torch.no_grad():
                lls = pc(x, force_use_bf16=True)
            pc.backward(inputs=x, allow_modify_flows=modify)
            torch.cuda.synchronize()
            out.append((lls.clone(), pc.node_mars.clone(), pc.node_flows.clone(), pc.param_flows.clone()))
    finally:
        SumLayer.tc05_ws = saved
    assert all(l._desc(cuda_device)["fw_run"] == 32 for g in pc.inner_layer_groups if g.is_sum() for l in g.layers
               if l._desc(cuda_device)["fw_tiles"].size(0) >= SumLayer.tc05_min_tiles)
    for a, b in zip(out[0], out[1]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("name,B,fw", [("hclt64", 37, dict(force_use_fp32=True)), ("hclt784", 64, dict(force_use_bf16=True)),
                                       ("tiny", 19, dict(force_use_fp32=True))])
def test_fused_products_equal_unfused(name, B, fw, cuda_device):
    """Product layers fused into the single-stage sum kernels, and product layers that write
    a large layer's node flows already rewritten as log f - log m, give bit-identical node
    values, element values, node flows and parameter flows."""
    from pyjuice_b200.model.tensorcircuit import TensorCircuit
    fx = load_fixture(name)
    rng = np.random.default_rng(5)
    ncat = 4 if name != "hclt784" else 256
    x = torch.from_numpy(rng.integers(0, ncat, size=(B, fx["x"].shape[1]))).to(cuda_device)
    saved = (TensorCircuit.fuse_products, TensorCircuit.fuse_products_forward, TensorCircuit.fuse_flow_rewrite)
    out = []
    try:
        for fuse in (False, True):
            TensorCircuit.fuse_products = TensorCircuit.fuse_products_forward = fuse
            TensorCircuit.fuse_flow_rewrite = fuse
            pc = build_fixture_circuit(name, fx).to(cuda_device)
            load_fixture_params(pc, fx)
            if fuse:
                assert pc._fusion_host
            pc.init_param_flows(flows_memory=0.0)
            with torch.no_grad():
                pc(x, **fw)
            pc.backward(inputs=x, allow_modify_flows=True, force_use_fp32=fw.get("force_use_fp32", False))
            torch.cuda.synchronize()
            em = torch.cat([pc._em_view(gi) for gi in pc._fusion_host])
            out.append((pc.node_mars.clone(), em.clone(), pc.node_flows.clone(), pc.param_flows.clone()))
    finally:
        TensorCircuit.fuse_products, TensorCircuit.fuse_products_forward, TensorCircuit.fuse_flow_rewrite = saved
    for a, b in zip(out[0], out[1]):
        assert torch.equal(a, b)


def test_multi_pack_equals_per_layer_packs(cuda_device):
    """One pcb_pack_weights_multi launch writes the same bytes as one pcb_pack_weights per
    tile table (forward and element-flow tables of every sum layer)."""
    from pyjuice_b200.layer.layers import SumLayer
    fx = load_fixture("hclt784")
    pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    saved = SumLayer.pack_short_weights
    try:
        SumLayer.pack_short_weights = True
        jobs = []
        for group in pc.inner_layer_groups:
            if group.is_sum():
                for layer in group:
                    job = layer.forward_pack_job(pc.device, 512, force_use_bf16=True)
                    jobs += ([job] if job is not None else []) + layer.flow_pack_jobs(pc.device, 512)
        assert len(jobs) > 20
        ref = []
        for job in jobs:
            job[2].fill_(7)
            SumLayer._run_pack_job(pc.params, job)
            ref.append(job[2].clone())
            job[2].zero_()
        assert pc._multi_pack(jobs)
        torch.cuda.synchronize()
        for job, r in zip(jobs, ref):
            assert torch.equal(job[2], r)
    finally:
        SumLayer.pack_short_weights = saved


@pytest.mark.parametrize("change", ["torch_write", "em"])
def test_backward_repacks_after_parameter_change(change, cuda_device):
    """The element-flow weights packed by a forward pass are reused by the backward pass only
    while the parameters are unchanged: after an in-place torch write or an EM step between
    the two passes, the backward packs again (same flows as a forced repack)."""
    from pyjuice_b200.layer.layers import SumLayer
    fx = load_fixture("hclt784")
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    saved = SumLayer.pack_short_weights
    try:
        SumLayer.pack_short_weights = True
        out = []
        for force in (False, True):
            pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
            load_fixture_params(pc, fx)
            pc.init_param_flows(flows_memory=0.0)
            with torch.no_grad():
                pc(x, force_use_bf16=True)
            pc.backward(inputs=x, allow_modify_flows=True)
            if change == "em":
                pc.mini_batch_em(step_size=0.5, pseudocount=0.01)
            else:
                with torch.no_grad():
                    pc.params.mul_(torch.linspace(0.5, 1.5, pc.params.numel(), device=cuda_device))
            pc.init_param_flows(flows_memory=0.0)
            if force:
                pc._el_pack_state = None
            pc.backward(inputs=x, allow_modify_flows=True)
            torch.cuda.synchronize()
            out.append(pc.param_flows.clone())
        assert torch.equal(out[0], out[1])
    finally:
        SumLayer.pack_short_weights = saved


def test_deterministic_flows(cuda_device):
    """Parameter flows carry no float atomics on untied circuits: two runs are bit-identical."""
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"]).to(cuda_device)
    _step(pc, x, force_use_fp32=True)
    a = pc.param_flows.clone()
    ai = pc.input_layer_group[0].param_flows.clone()
    _step(pc, x, force_use_fp32=True)
    assert torch.equal(a, pc.param_flows)
    assert torch.equal(ai, pc.input_layer_group[0].param_flows)


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_sampling_bit_exact_vs_oracle(name, cuda_device):
    fx = load_fixture(name)
    pc = build_fixture_circuit(name, fx).to(cuda_device)
    load_fixture_params(pc, fx)
    S, seed = 64, 1234567
    got = juice.queries.sample(pc, S, seed=seed).cpu().numpy()
    lay = orc.layout_from_circuit(pc)
    ref = orc.sample(lay, fx["params0"], fx["in_params0"], S, seed, pc.num_vars)
    assert np.array_equal(got, ref)


def test_sampling_marginals(cuda_device):
    """Empirical single-variable marginals of 20k samples match the exact marginals of the tiny circuit."""
    fx = load_fixture("tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    S = 20000
    s = juice.queries.sample(pc, S, seed=7).cpu().numpy()
    lay = orc.layout_from_circuit(pc)
    allx = np.array(list(itertools.product(range(4), repeat=6)), dtype=np.int64)
    _, _, lls = orc.forward(lay, fx["params0"], fx["in_params0"], allx)
    p = np.exp(lls[:, 0])
    for v in range(6):
        exact = np.array([p[allx[:, v] == k].sum() for k in range(4)])
        emp = np.bincount(s[:, v], minlength=4) / S
        assert np.abs(exact - emp).max() < 0.02


def test_invalid_category_gives_nan_not_fault(cuda_device):
    fx = load_fixture("tiny")
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(fx["x"][:8]).to(cuda_device).clone()
    x[0, 0] = 99
    with torch.no_grad():
        lls = pc(x, force_use_fp32=True)
    assert not torch.isfinite(lls[0, 0])  # NaN or -inf: the bad value never becomes a finite LL
    assert torch.isfinite(lls[1:]).all()


def test_errors_are_raised(cuda_device):
    fx = load_fixture("tiny")
    cpu_pc = build_fixture_circuit("tiny", fx)
    with pytest.raises(RuntimeError):
        cpu_pc(torch.from_numpy(fx["x"][:4]))  # there is no CPU path
    pc = build_fixture_circuit("tiny", fx).to(cuda_device)
    with pytest.raises(RuntimeError):
        pc.mini_batch_em(step_size=0.1)  # no flows yet
    with pytest.raises(ValueError):
        pc.mini_batch_em(step_size=0.0)


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_sampling_matches_reference_draws(name, cuda_device):
    """Bit-exact against the reference's own samples: the reference's queries.sample was run
    with every tl.rand draw of node n in sample s replaced by table[n, s]; the device sampler
    given the same table (``uniforms=``) returns the same 256 samples. The table is the
    SplitMix64 hash of the seeded sampler, so the seeded path must agree too."""
    fx = load_fixture(name)
    sf = load_fixture("samples_" + name)
    pc = build_fixture_circuit(name, fx).to(cuda_device)
    load_fixture_params(pc, fx)
    S, seed = int(sf["num_samples"]), int(sf["uniform_seed"])
    table = torch.from_numpy(orc.uniform_table(seed, pc.num_nodes, S)).to(cuda_device)
    got = juice.queries.sample(pc, S, uniforms=table).cpu().numpy()
    assert np.array_equal(got, sf["samples"])
    assert np.array_equal(juice.queries.sample(pc, S, seed=seed).cpu().numpy(), sf["samples"])
    # a table wider than S (leading dimension > S) reads the same draws
    wide = torch.zeros([pc.num_nodes, S + 13], dtype=torch.float32, device=cuda_device)
    wide[:, :S] = table
    assert np.array_equal(juice.queries.sample(pc, S, uniforms=wide).cpu().numpy(), sf["samples"])


@pytest.mark.parametrize("H", [64, 256, 512])
def test_shared_tied_packs_equal_separate(H, cuda_device):
    """The time steps of a homogeneous HMM (tied transitions) share one packed-weight buffer
    (short packed tiles at 64 hidden states, tcgen05 chunks of long tiles at 256 and 512),
    packed once per pass: log-likelihoods, sum-parameter flows and the sum EM update of two
    split-bf16 steps are bit-identical to separate buffers packed per layer. (The tied
    emission table's flows are summed with atomics, in no fixed order, so the emission
    parameters after the first step are made equal before the second.)"""
    from pyjuice_b200.model.tensorcircuit import TensorCircuit
    saved = TensorCircuit.share_tied_packs
    out = []
    q1 = None
    try:
        for share in (False, True):
            TensorCircuit.share_tied_packs = share
            torch.manual_seed(0)
            pc = juice.compile(juice.structures.HMM(8, H, 50, homogeneous=True)).to(cuda_device)
            x = torch.randint(0, 50, (128, 8), generator=torch.Generator().manual_seed(1)).to(cuda_device)
            res = []
            for step in range(2):
                pc.init_param_flows(flows_memory=0.0)
                lls = pc(x, force_use_bf16=True)
                lls.mean().backward()
                res += [lls.detach().clone(), pc.param_flows.clone()]
                pc.mini_batch_em(step_size=0.1, pseudocount=0.1)
                res.append(pc.params.clone())
                if step == 0:
                    q = pc.input_layer_group[0].params
                    if q1 is None:
                        q1 = q.clone()
                    else:
                        with torch.no_grad():
                            q.copy_(q1)
            if share:
                ptrs = [l._desc(pc.device)["fw_pack"].data_ptr() for g in pc.inner_layer_groups if g.is_sum()
                        for l in g]
                assert len(set(ptrs)) < len(ptrs)
            out.append(res)
    finally:
        TensorCircuit.share_tied_packs = saved
    for a, b in zip(out[0], out[1]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("H,homogeneous", [(64, True), (256, True), (512, True), (256, False)])
def test_tied_set_parameter_flows(H, homogeneous, cuda_device):
    """Parameter flows of a tied set (the time steps of a homogeneous HMM, source included)
    in one launch (pcb_sum_pflows_tc05_tied) against one launch per layer: the same flows up
    to the order of the FP32 sums (split bf16, two backward passes accumulated), and against
    the FP64 oracle within the split-bf16 bound. Without tied transitions nothing changes."""
    from pyjuice_b200.model.tensorcircuit import TensorCircuit
    saved = TensorCircuit.tied_pflows
    out = []
    try:
        for on in (False, True):
            TensorCircuit.tied_pflows = on
            torch.manual_seed(0)
            pc = juice.compile(juice.structures.HMM(8, H, 50, homogeneous=homogeneous)).to(cuda_device)
            x = torch.randint(0, 50, (128, 8), generator=torch.Generator().manual_seed(1)).to(cuda_device)
            pc.init_param_flows(flows_memory=0.0)
            for _ in range(2):
                lls = pc(x, force_use_bf16=True)
                lls.mean().backward()
            if on:
                sets = pc.__dict__.get("_tied_pflow_cache", {})
                assert bool(sum(len(v) for v in sets.values())) == homogeneous
            out.append((pc, x, pc.param_flows.double().clone()))
    finally:
        TensorCircuit.tied_pflows = saved
    a, b = out[0][2], out[1][2]
    assert (a - b).abs().max() <= 1e-5 * a.abs().max()
    pc, x = out[1][0], out[1][1].cpu().numpy()
    lay = orc.layout_from_circuit(pc)
    p0 = pc.params.double().cpu().numpy()
    q0 = pc.input_layer_group[0].params.double().cpu().numpy()
    nm, ems, _ = orc.forward(lay, p0, q0, x)
    _, pf_o, _ = orc.backward(lay, p0, x, nm, ems)
    assert np.abs(b.cpu().numpy() - 2 * pf_o).max() <= 2e-3 * np.abs(2 * pf_o).max()
