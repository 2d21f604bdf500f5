"""The persistent warp-specialised tcgen05 contraction (pcb_lse_contract_tc05_ws) against the
CTA-per-slice kernel (pcb_lse_contract_tc05) through the C ABI: both run the same
arithmetic in the same order (per-sample max, exp, bf16 split, MMAs over 16-term steps,
FP32 accumulators), so their outputs must be bit-identical, for the sum forward (mode 0) and
the element flows (modes 1 and 2), in both precision forms, for ragged tiles (fewer rows and
terms than 128), a partial last sample slice, several tiles per CTA (weights copied again)
and CTAs owning a single unit. Both are also checked against an FP64 evaluation of the
contraction. An oversize tile gives NaN rows and the device status bit, as in the other
kernels."""

import numpy as np
import pytest
import torch

from pyjuice_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _problem(B, device, seed, run):
    """Tiles whose terms come in runs of ``run`` consecutive source rows (random run starts;
    the last run of a tile may be partial)."""
    g = torch.Generator().manual_seed(seed)
    # tiles: (n_rows, k_cnt)
    shapes = [(128, 128), (96, 100), (40, 17), (128, 128), (128, 64), (33, 128), (128, 1)]
    T = len(shapes)
    n_src = 300
    tiles, krow, kw = [], [], []
    for t, (nr, kc) in enumerate(shapes):
        tiles.append([t * 128, nr, len(krow), kc, t * 128 * 128, t * 128, 32, 0])
        for k0 in range(0, kc, run):
            start = int(torch.randint(0, n_src - run + 1, (1,), generator=g))
            krow += [start + j for j in range(min(run, kc - k0))]
        kw += [k * 128 for k in range(kc)]
    src = torch.rand([n_src, B], generator=g) * 6 - 8
    src[7] = -float("inf")                     # a row of -inf terms
    src[:, 3] = -float("inf")                  # a sample whose terms are all -inf
    flows = torch.rand([n_src, B], generator=g)
    flows[11] = 0.0
    aux = torch.rand([T * 128, B], generator=g) * 4 - 5
    params = torch.rand([T * 128 * 128], generator=g) + 0.05
    dev = lambda x: x.to(device)
    return dict(src=dev(src), flows=dev(flows), aux=dev(aux), params=dev(params),
                tiles=dev(torch.tensor(tiles, dtype=torch.int32)), krow=dev(torch.tensor(krow, dtype=torch.int32)),
                kw=dev(torch.tensor(kw, dtype=torch.int32)), shapes=shapes, B=B, T=T, run=run)


def _pack(p, device):
    packed = torch.zeros([p["T"] * 65536], dtype=torch.uint8, device=device)
    nat.call("pcb_pack_weights", nat.ptr(p["params"]), nat.ptr(p["tiles"]), p["T"], 32, nat.ptr(p["kw"]), 1,
             nat.ptr(packed), nat.stream())
    return packed


def _run(p, packed, mode, prec, kernel, bt, arg):
    B, T = p["B"], p["T"]
    src = p["flows"] if mode == 2 else p["src"]
    src2 = p["src"] if mode == 2 else None
    aux = p["aux"] if mode >= 1 else None
    out = torch.full([T * 128, B], 12345.0, device=p["src"].device)
    if kernel == "pcb_lse_contract_tc05":
        nat.call(kernel, nat.ptr(src), nat.ptr(src2), nat.ptr(aux), nat.ptr(out), B, B, nat.ptr(packed),
                 nat.ptr(p["tiles"]), T, nat.ptr(p["krow"]), mode, prec, bt, arg, nat.stream())
    else:
        nat.call(kernel, nat.ptr(src), nat.ptr(src2), nat.ptr(aux), nat.ptr(out), B, B, src.size(0), out.size(0),
                 nat.ptr(packed), nat.ptr(p["tiles"]), T, nat.ptr(p["krow"]), mode, prec, bt, p["run"], arg,
                 nat.stream())
    return out


def _fp64(p, mode):
    """The contraction in FP64 with the FP32 weights (mode 0: log-sum; 1/2: element flows)."""
    B = p["B"]
    src, flows, aux = p["src"].double().cpu(), p["flows"].double().cpu(), p["aux"].double().cpu()
    params = p["params"].double().cpu()
    krow, kw, tiles = p["krow"].cpu(), p["kw"].cpu(), p["tiles"].cpu()
    out = torch.full([p["T"] * 128, B], 12345.0, dtype=torch.float64)
    for t in range(p["T"]):
        o_row, nr, k_off, kc, w_add, a_row, g_str, _ = tiles[t].tolist()
        rows = krow[k_off:k_off + kc].long()
        r = torch.arange(nr)
        wid = kw[k_off:k_off + kc].long()[:, None] + w_add + (r // 32) * g_str + (r % 32)
        W = params[wid]                                    # [k, r]
        if mode == 2:
            v = torch.where(src[rows] == -float("inf"), -float("inf"), torch.log(flows[rows]) - src[rows])
        else:
            v = src[rows]
        m = v.max(dim=0).values
        m0 = torch.where(torch.isfinite(m), m, torch.zeros_like(m))
        acc = W.T @ torch.exp(v - m0)                      # [r, B]
        if mode == 0:
            res = torch.where(torch.isfinite(m), torch.log(acc) + m0, torch.full_like(acc, -float("inf")))
        else:
            res = torch.where(torch.isfinite(m), acc * torch.exp(aux[a_row:a_row + nr] + m0), torch.zeros_like(acc))
        out[o_row:o_row + nr] = res
    return out


@pytest.mark.parametrize("B,run", [(512, 32), (100, 8), (512, 8)])
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("prec", [2, 1])
def test_ws_bit_identical_to_per_slice_kernel(B, run, mode, prec, cuda_device):
    p = _problem(B, cuda_device, seed=B + 10 * mode + prec + run, run=run)
    packed = _pack(p, cuda_device)
    ref64 = _fp64(p, mode)
    for bt in (32, 64):
        base = _run(p, packed, mode, prec, "pcb_lse_contract_tc05", bt, 1)
        for ctas in (0, 3, 1):  # one per SM (mostly one unit each); 3 and 1: many units and tiles per CTA
            got = _run(p, packed, mode, prec, "pcb_lse_contract_tc05_ws", bt, ctas)
            torch.cuda.synchronize()
            assert nat.device_status(clear=True) == 0
            assert torch.equal(got, base), (bt, ctas, (got - base).abs().nan_to_num(0).max())
        # both against FP64 (split form: bf16 hi + lo operands)
        g = base.double().cpu()
        fin = torch.isfinite(ref64)
        assert torch.equal(fin, torch.isfinite(g))
        tol = 1e-4 if prec == 2 else 2e-2
        if mode == 0:
            err = (g[fin] - ref64[fin]).abs().max()
        else:
            err = ((g[fin] - ref64[fin]).abs() / ref64[fin].abs().clamp(min=1e-3)).max()
        assert err <= tol, err


def test_ws_oversize_tile_is_reported(cuda_device):
    B = 64
    src = torch.zeros([256, B], dtype=torch.float32, device=cuda_device)
    out = torch.zeros([128, B], dtype=torch.float32, device=cuda_device)
    krow = torch.zeros([256], dtype=torch.int32, device=cuda_device)
    tiles = torch.tensor([[0, 128, 0, 129, 0, 0, 0, 0]], dtype=torch.int32, device=cuda_device)
    packed = torch.zeros([65536], dtype=torch.uint8, device=cuda_device)
    nat.device_status(clear=True)
    nat.call("pcb_lse_contract_tc05_ws", nat.ptr(src), nat.ptr(None), nat.ptr(None), nat.ptr(out), B, B, 256, 128,
             nat.ptr(packed), nat.ptr(tiles), 1, nat.ptr(krow), 0, 2, 64, 32, 0, nat.stream())
    assert nat.device_status(clear=True) == 2
    assert torch.isnan(out).all()


def test_ws_rejects_unaligned_batch(cuda_device):
    B = 30
    src = torch.zeros([8, 32], dtype=torch.float32, device=cuda_device)
    tiles = torch.tensor([[0, 8, 0, 8, 0, 0, 0, 0]], dtype=torch.int32, device=cuda_device)
    krow = torch.zeros([8], dtype=torch.int32, device=cuda_device)
    packed = torch.zeros([65536], dtype=torch.uint8, device=cuda_device)
    with pytest.raises(RuntimeError, match="B % 4"):
        nat.call("pcb_lse_contract_tc05_ws", nat.ptr(src), nat.ptr(None), nat.ptr(None), nat.ptr(src), 32, B, 8, 8,
                 nat.ptr(packed), nat.ptr(tiles), 1, nat.ptr(krow), 0, 2, 64, 8, 0, nat.stream())


def _pack_fp8(p, device):
    packed = torch.zeros([p["T"] * 65536], dtype=torch.uint8, device=device)
    nat.call("pcb_pack_weights_fp8", nat.ptr(p["params"]), nat.ptr(p["tiles"]), p["T"], 32, nat.ptr(p["kw"]), 1,
             nat.ptr(packed), nat.stream())
    return packed


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("bt", [32, 64])
def test_e4m3_form_vs_fp64(mode, bt, cuda_device):
    """The E4M3 form of the tcgen05 contraction (per-row weight scales, exponentials scaled by
    448, FP32 accumulation) against FP64: log-sums within 0.1 nats, element flows within
    10 % (e4m3 keeps 3 mantissa bits; the errors of 128 positive terms partly average out),
    the same -inf / zero pattern, and clearly less exact than split bf16."""
    p = _problem(512, cuda_device, seed=40 + mode, run=32)
    packed = _pack_fp8(p, cuda_device)
    got = _run(p, packed, mode, 3, "pcb_lse_contract_tc05", bt, 1).double().cpu()
    torch.cuda.synchronize()
    assert nat.device_status(clear=True) == 0
    ref = _fp64(p, mode)
    fin = torch.isfinite(ref)
    assert torch.equal(fin, torch.isfinite(got))
    if mode == 0:
        err = (got[fin] - ref[fin]).abs()
        assert err.max() <= 0.1 and err.mean() <= 0.02, (err.max(), err.mean())
    else:
        big = fin & (ref.abs() > 1e-3 * ref[fin].abs().max())
        rel = ((got[big] - ref[big]).abs() / ref[big].abs())
        assert rel.max() <= 0.1 and rel.mean() <= 0.02, (rel.max(), rel.mean())
        assert torch.all(got[fin & (ref == 0)] == 0)


def test_e4m3_multi_pack_matches_single(cuda_device):
    """Format 1 of pcb_pack_weights_multi writes the same bytes as pcb_pack_weights_fp8."""
    import numpy as np
    from pyjuice_b200.model.tensorcircuit import _PACK_JOB
    p = _problem(64, cuda_device, seed=7, run=8)
    ref = _pack_fp8(p, cuda_device)
    packed = torch.zeros_like(ref)
    rec = np.zeros(1, dtype=_PACK_JOB)
    rec[0] = (p["tiles"].data_ptr(), p["kw"].data_ptr(), packed.data_ptr(), p["T"], 5, 1, 1)
    jobs = torch.from_numpy(rec.view(np.uint8).copy()).to(cuda_device)
    tj = torch.zeros([p["T"]], dtype=torch.int32, device=cuda_device)
    ti = torch.arange(p["T"], dtype=torch.int32, device=cuda_device)
    nat.call("pcb_pack_weights_multi", nat.ptr(p["params"]), nat.ptr(jobs), nat.ptr(tj), nat.ptr(ti), p["T"],
             nat.stream())
    torch.cuda.synchronize()
    per_tile = 16384 + 512
    for t in range(p["T"]):
        assert torch.equal(packed[t * 65536:t * 65536 + per_tile], ref[t * 65536:t * 65536 + per_tile])


def test_e4m3_form_on_hclt784_after_bf16(cuda_device):
    """HCLT-784 at batch 256: a split-bf16 pass, then the E4M3 form on the same circuit (the
    weight packs switch format), then split bf16 again. The E4M3 log-likelihoods (3 mantissa
    bits in the 17 tcgen05 levels) stay within 1.5 nats per sample of the split-bf16 ones,
    0.6 on average (measured: 0.66 and 0.39 at mean LL ~ -2700), and the second split-bf16
    pass reproduces the first bit for bit."""
    from conftest import load_fixture
    from helpers import build_fixture_circuit, load_fixture_params
    from pyjuice_b200.layer.layers import SumLayer
    import numpy as np
    fx = load_fixture("hclt784")
    pc = build_fixture_circuit("hclt784", fx).to(cuda_device)
    load_fixture_params(pc, fx)
    x = torch.from_numpy(np.random.default_rng(21).integers(0, 256, size=(256, 784))).to(cuda_device)
    saved = SumLayer.bf16_form
    try:
        out = []
        for form in (2, 3, 2):
            SumLayer.bf16_form = form
            with torch.no_grad():
                out.append(pc(x, force_use_bf16=True).clone())
            pc.init_param_flows(flows_memory=0.0)
            pc.backward(inputs=x, allow_modify_flows=True)
            assert torch.isfinite(pc.param_flows).all()
    finally:
        SumLayer.bf16_form = saved
    assert torch.equal(out[0], out[2])
    d = (out[1] - out[0]).abs()
    assert torch.isfinite(out[1]).all() and d.max() < 1.5 and d.mean() < 0.6, (d.max(), d.mean())


def _long_problem(B, device, seed):
    """Tiles of 1 .. 400 terms (runs of 32 rows), for the chunked tcgen05 path."""
    g = torch.Generator().manual_seed(seed)
    shapes = [(128, 400), (96, 300), (40, 129), (128, 128), (128, 17), (33, 257)]
    T = len(shapes)
    n_src = 1200
    tiles, krow, kw = [], [], []
    for t, (nr, kc) in enumerate(shapes):
        tiles.append([t * 128, nr, len(krow), kc, t * 128 * 400, t * 128, 32, 0])
        for k0 in range(0, kc, 32):
            start = int(torch.randint(0, n_src - 32 + 1, (1,), generator=g))
            krow += [start + j for j in range(min(32, kc - k0))]
        kw += [k * 128 for k in range(kc)]
    src = torch.rand([n_src, B], generator=g) * 30 - 40
    src[5] = -float("inf")
    flows = torch.rand([n_src, B], generator=g)
    aux = torch.rand([T * 128, B], generator=g) * 4 - 5
    params = torch.rand([T * 128 * 400], generator=g) + 0.05
    dev = lambda x: x.to(device)
    return dict(src=dev(src), flows=dev(flows), aux=dev(aux), params=dev(params),
                tiles=dev(torch.tensor(tiles, dtype=torch.int32)), krow=dev(torch.tensor(krow, dtype=torch.int32)),
                kw=dev(torch.tensor(kw, dtype=torch.int32)), shapes=shapes, B=B, T=T, run=32)


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("prec", [2, 3])
@pytest.mark.parametrize("partials", [False, True])
def test_long_tiles_as_tc05_chunks_vs_fp64(mode, prec, partials, cuda_device):
    """Tiles of up to 400 terms contracted as 128-term chunks on the tcgen05 kernel against
    FP64: one launch per chunk index (first chunk overwrites, later chunks log-add / add), or
    every chunk in one launch into partial rows combined by pcb_chunk_combine. Split bf16
    within 1e-4, E4M3 within the bounds of its single-chunk test."""
    from pyjuice_b200.layer.layers import _chunk_table, _tc05_chunks
    p = _long_problem(256, cuda_device, seed=60 + mode + 3 * prec)
    tab, ranges = _chunk_table(p["tiles"].cpu().numpy().astype("int64"))
    ct = torch.from_numpy(tab).to(torch.int32).to(cuda_device)
    pack = torch.zeros([ct.size(0) * 65536], dtype=torch.uint8, device=cuda_device)
    nat.call("pcb_pack_weights_fp8" if prec == 3 else "pcb_pack_weights", nat.ptr(p["params"]), nat.ptr(ct),
             ct.size(0), 32, nat.ptr(p["kw"]), 1, nat.ptr(pack), nat.stream())
    src = p["flows"] if mode == 2 else p["src"]
    out = torch.full([p["T"] * 128, p["B"]], 12345.0, device=cuda_device)
    _tc05_chunks(src, p["src"] if mode == 2 else None, p["aux"] if mode else None, out, p["B"], p["B"], pack, ct,
                 ranges, p["krow"], mode, prec, nat.stream(), holder=dict() if partials else None, plan_key="plan")
    torch.cuda.synchronize()
    assert nat.device_status(clear=True) == 0
    got = out.double().cpu()
    ref = _fp64(p, mode)
    rows = torch.zeros([p["T"] * 128], dtype=torch.bool)
    for t, (nr, _) in enumerate(p["shapes"]):
        rows[t * 128:t * 128 + nr] = True
    got, ref = got[rows], ref[rows]
    fin = torch.isfinite(ref)
    assert torch.equal(fin, torch.isfinite(got))
    if mode == 0:
        err = (got[fin] - ref[fin]).abs()
        bound = 1e-4 if prec == 2 else 0.1
    else:
        big = fin & (ref.abs() > 1e-3 * ref[fin].abs().max())
        err = (got[big] - ref[big]).abs() / ref[big].abs()
        bound = 1e-4 if prec == 2 else 0.1
    assert err.max() <= bound, err.max()


def test_pd_long_tiles_on_tc05_vs_oracle(cuda_device):
    """A PD circuit whose sum layers have tiles of 256 terms (8x8 grid, 64 latents, block 32,
    four product vectors per sum): the split-bf16 pass runs them as tcgen05 chunks
    (tc05_min_tiles lowered to 1), and its LLs and parameter flows match the FP64 oracle."""
    import numpy as np
    from oracle import pc_oracle as orc
    import pyjuice_b200 as juice
    from pyjuice_b200.layer.layers import SumLayer
    torch.manual_seed(3)
    pc = juice.compile(juice.structures.PD((8, 8), 64, split_intervals=2, block_size=32, max_prod_block_conns=4,
                                           input_dist=juice.distributions.Categorical(num_cats=8))).to(cuda_device)
    saved = SumLayer.tc05_min_tiles
    try:
        SumLayer.tc05_min_tiles = 1
        longs = [l for g in pc.inner_layer_groups if g.is_sum() for l in g if l._desc(cuda_device)["fw_ch"] is not None]
        assert longs and all(l._fw_long(l._desc(cuda_device), 2) for l in longs)
        x = np.random.default_rng(5).integers(0, 8, size=(128, 64))
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            lls = pc(torch.from_numpy(x).to(cuda_device), force_use_bf16=True).double().cpu().numpy()
        pc.backward(inputs=torch.from_numpy(x).to(cuda_device), allow_modify_flows=True)
        pf = pc.param_flows.double().cpu().numpy()
    finally:
        SumLayer.tc05_min_tiles = saved
    lay = orc.layout_from_circuit(pc)
    p0 = pc.params.double().cpu().numpy()
    q0 = pc.input_layer_group[0].params.double().cpu().numpy()
    nm, ems, lls_o = orc.forward(lay, p0, q0, x)
    _, pf_o, _ = orc.backward(lay, p0, x, nm, ems)
    assert np.abs(lls - lls_o).max() <= 1e-3
    assert np.abs(pf - pf_o).max() <= 1e-3 * np.abs(pf_o).max()
