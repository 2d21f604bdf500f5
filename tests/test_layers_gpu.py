"""Layer-level kernels on the GPU, checked with the formulas of the reference's layer tests
(tests/layer/sum_layer_test.py:17-143, tests/layer/prod_layer_test.py:17-91) in FP64 torch."""

import pytest
import torch

import pyjuice_b200 as juice
from pyjuice_b200.nodes import distributions as dists

from circuits import build_layer_test_nodes

pytestmark = pytest.mark.gpu


def _layers(bs):
    ni, nps, nss = build_layer_test_nodes(juice, dists, bs)
    juice.InputLayer(ni, cum_nodes=bs)
    prod = juice.ProdLayer(nps)
    layer = juice.SumLayer(nss, global_nid_start=bs, global_pid_start=bs ** 2, global_pfid_start=0,
                           node2tiednodes=dict())
    return prod, layer


@pytest.mark.parametrize("bs,B,fp32", [(16, 16, True), (16, 16, False), (4, 7, True), (32, 130, True),
                                       (32, 256, False)])
def test_sum_layer_forward_backward(bs, B, fp32, cuda_device):
    torch.manual_seed(63892)
    prod, layer = _layers(bs)
    layer.to(cuda_device)
    em = torch.rand([bs + 3 * 2 * 2 * bs, B]).log().to(cuda_device)
    em[:bs] = -float("inf")
    nm = torch.zeros([bs + bs * 2 * 3, B], device=cuda_device)
    params = torch.rand([bs ** 2 + 3 * 4 * bs * bs], device=cuda_device)
    layer(nm, em, params, force_use_fp32=fp32, force_use_bf16=not fp32)
    tol = 1e-5 if fp32 else 2e-2
    cids, pids = layer.partitioned_cids[0], layer.partitioned_pids[0]
    for j in range(6):
        for i in range(bs):
            ref = (params[pids[j] + i].double()[:, None] * em[cids[j]].double().exp()).sum(0).log()
            assert torch.all((nm[(j + 1) * bs + i].double() - ref).abs() <= tol * ref.abs().clamp(min=1.0))

    nf = torch.rand([bs + bs * 2 * 3, B], device=cuda_device)
    ef = torch.zeros([bs + 3 * 2 * 2 * bs, B], device=cuda_device)
    pf = torch.zeros_like(params)
    nm64 = nm.double()
    layer.backward(nf, ef, nm, em, params, pf, force_use_fp32=fp32)
    chids, parids, parpids = layer.partitioned_chids[0], layer.partitioned_parids[0], layer.partitioned_parpids[0]
    etol = 1e-4 if fp32 else 3e-2
    for j in range(6):
        prow = (parids[j][:, None] + torch.arange(bs, device=cuda_device)[None, :]).reshape(-1)
        for i in range(bs):
            w = (parpids[j][:, None] + i * bs + torch.arange(bs, device=cuda_device)[None, :]).reshape(-1)
            ref = (nf[prow].double() * params[w].double()[:, None] * em[chids[j] + i].double().exp()[None, :]
                   / nm64[prow].exp()).sum(0)
            assert torch.all((ef[chids[j] + i].double() - ref).abs() <= etol * ref.abs().max())
    my_pf = torch.zeros_like(params, dtype=torch.float64)
    for j in range(6):
        for i in range(bs):
            row = (j + 1) * bs + i
            my_pf[layer.partitioned_pfids[0][j] + i] = params[pids[j] + i].double() * (
                nf[row].double()[None, :] * em[cids[j]].double().exp() / nm64[row].exp()[None, :]).sum(1)
    assert torch.all((pf.double() - my_pf).abs() <= 1e-4 * my_pf.abs().max())


def test_sum_layer_unmodified_flows_equal_modified(cuda_device):
    """allow_modify_flows=False (log f - log m computed on the fly) gives the same flows."""
    bs, B = 16, 64
    torch.manual_seed(1)
    prod, layer = _layers(bs)
    layer.to(cuda_device)
    em = torch.rand([bs + 12 * bs, B]).log().to(cuda_device)
    em[:bs] = -float("inf")
    nm = torch.zeros([7 * bs, B], device=cuda_device)
    params = torch.rand([bs ** 2 + 12 * bs * bs], device=cuda_device)
    layer(nm, em, params, force_use_fp32=True)
    nf = torch.rand([7 * bs, B], device=cuda_device)
    ef1, ef2 = torch.zeros_like(em), torch.zeros_like(em)
    pf1, pf2 = torch.zeros_like(params), torch.zeros_like(params)
    layer.backward(nf.clone(), ef1, nm, em, params, pf1, allow_modify_flows=True, force_use_fp32=True)
    layer.backward(nf.clone(), ef2, nm, em, params, pf2, allow_modify_flows=False, force_use_fp32=True)
    assert torch.allclose(ef1, ef2, rtol=1e-5, atol=1e-6)
    assert torch.allclose(pf1, pf2, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("B", [16, 5])
def test_prod_layer_forward_backward(B, cuda_device):
    bs = 16
    torch.manual_seed(2)
    prod, _ = _layers(bs)
    prod.to(cuda_device)
    nm = torch.rand([bs + 4 * 2 * bs, B], device=cuda_device)
    nm[:bs] = 0.0
    em = torch.full([bs + 3 * 2 * bs, B], -float("inf"), device=cuda_device)
    prod(nm, em)
    for nids, cids in zip(prod.partitioned_nids, prod.partitioned_cids):
        for g in range(nids.size(0)):
            for i in range(bs):
                ref = sum(nm[cids[g, j] + i] for j in range(cids.size(1)))
                assert torch.allclose(em[nids[g] + i], ref, atol=1e-6)
    ef = torch.rand_like(em)
    ef[:bs] = 0.0
    nf = torch.zeros_like(nm)
    prod.backward(nf, ef)
    for u, par in zip(prod.partitioned_u_cids, prod.partitioned_parids):
        for g in range(u.size(0)):
            for i in range(bs):
                ref = sum(ef[par[g, q] + i] for q in range(par.size(1)))
                assert torch.allclose(nf[u[g] + i], ref, atol=1e-6)


@pytest.mark.parametrize("path", ["short", "short_packed", "tc05", "tc05_multi"])
@pytest.mark.parametrize("bs,B,form", [(8, 7, 2), (16, 130, 2), (32, 256, 2), (32, 512, 1), (64, 33, 2)])
def test_short_kernels_match_chunked(bs, B, form, path, cuda_device):
    """The single-stage contractions (<= 128 terms: mma.sync or tcgen05) agree with the chunked ones."""
    from pyjuice_b200.layer.layers import SumLayer
    torch.manual_seed(1234 + bs + B)
    prod, layer = _layers(bs)
    layer.to(cuda_device)
    n_el = bs + 3 * 2 * 2 * bs
    n_nd = bs + bs * 2 * 3
    em = (torch.rand([n_el, B]) * 4 - 6).to(cuda_device)
    em[:bs] = -float("inf")
    params = torch.rand([bs ** 2 + 3 * 4 * bs * bs], device=cuda_device)
    nf0 = torch.rand([n_nd, B], device=cuda_device)
    outs = {}
    saved = (SumLayer.short_kernels, SumLayer.bf16_form, SumLayer.tc05_min_tiles, SumLayer.pack_short_weights,
             SumLayer.tc05_slices_per_cta)
    try:
        SumLayer.bf16_form = form
        SumLayer.pack_short_weights = path == "short_packed"
        for short in (False, True):
            SumLayer.short_kernels = short
            SumLayer.tc05_min_tiles = 1 if (short and path in ("tc05", "tc05_multi")) else 1 << 30
            # "tc05": one CTA per sample slice; "tc05_multi": two slices per CTA
            SumLayer.tc05_slices_per_cta = 2 if path == "tc05_multi" else 1
            packed = short and path == "short_packed"
            if packed:  # weights packed ahead of the contractions, as the circuit passes do
                layer.pack_forward_weights(params, B, force_use_bf16=True)
                layer.pack_flow_weights(params, B)
            nm = torch.zeros([n_nd, B], device=cuda_device)
            layer(nm, em, params, force_use_bf16=True, _weights_packed=packed)
            ef = torch.zeros([n_el, B], device=cuda_device)
            pf = torch.zeros_like(params)
            nf = nf0.clone()
            layer.backward(nf, ef, nm, em, params, pf, _weights_packed=packed)
            ef2 = torch.zeros([n_el, B], device=cuda_device)
            nf2 = nf0.clone()
            layer.backward(nf2, ef2, nm, em, params, None, allow_modify_flows=True, _weights_packed=packed)
            outs[short] = (nm[bs:], ef[bs:], ef2[bs:], pf)
    finally:
        (SumLayer.short_kernels, SumLayer.bf16_form, SumLayer.tc05_min_tiles, SumLayer.pack_short_weights,
         SumLayer.tc05_slices_per_cta) = saved
    tol = 2e-5 if form == 2 else 2e-2
    for a, b in zip(outs[False], outs[True]):
        assert torch.isfinite(b).all()
        assert torch.all((a - b).abs() <= tol * a.abs().clamp(min=1.0)), (a - b).abs().max()
