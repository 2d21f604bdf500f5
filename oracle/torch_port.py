"""FP32 PyTorch CPU restatement of one EM step (test and benchmark infrastructure, not
product code).

The reference has no CPU implementation of its compiled-circuit passes (its input layers
raise on CPU, and every pass is a Triton kernel). This module restates the same arithmetic
as ``pc_oracle`` (whose FP64 numpy version is pinned to the reference's outputs) in FP32
with batched torch tensor operations, so that a CPU step uses every host core (intra-op
threads) at the full batch. ``bench.py`` times it as the CPU baseline and as the reference
arm; ``tests/test_oracle_golden.py`` checks it against ``pc_oracle``. The per-partition
tables are converted to tensors once (``TorchLayout``).

Reference formulas restated (paths relative to the reference project root): input
``log theta[x]`` (categorical.py:83-91); product ``sum_j nm[cids[j] + i]``
(prod_layer.py:398-466); sum ``log sum_c theta exp(em_c)`` (sum_layer.py:454-568);
element flows ``sum_n nf theta exp(em - nm)`` and parameter flows
``theta sum_b nf exp(em - nm)`` (sum_layer.py:1572-1730, 2052-2169); EM
``(1 - s) theta + s (f + pc / n) / (sum f + pc)`` (par_update.py:174-256, categorical.py:164-244).
"""

from __future__ import annotations

import numpy as np
import torch

from .pc_oracle import _sum_block_table


def _rows(start: torch.Tensor, bs: int) -> torch.Tensor:
    return (start[:, None] + torch.arange(bs)[None, :]).reshape(-1)


class TorchLayout:
    """Index tables of a ``pc_oracle`` layout as int64 tensors, plus the EM block tables."""

    def __init__(self, layout: dict):
        self.lay = layout
        T = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.long)
        self.groups = []
        for g in layout["groups"]:
            layers = []
            for l in g["layers"]:
                t = dict(kind=l["kind"], bs=l["block_size"], nid_range=tuple(l["nid_range"]))
                for name in ("nids", "cids", "pids", "pfids", "chids", "parids", "parpids", "u_cids"):
                    if name in l:
                        t[name] = [T(a) for a in l[name]]
                if l["kind"] == "sum":
                    t["cs_block_sizes"] = list(l["cs_block_sizes"])
                layers.append(t)
            self.groups.append(dict(kind=g["kind"], layers=layers))
        inp = layout["input"]
        self.in_start = int(inp["nid_start"])
        self.vids, self.s_pids, self.s_pfids = T(inp["vids"]), T(inp["s_pids"]), T(inp["s_pfids"])
        self.ncats = T(inp["ncats"])
        self.in_npf = int(inp["num_param_flows"]) if inp.get("num_param_flows") else \
            int((inp["s_pfids"] + inp["ncats"]).max())
        table = _sum_block_table(layout)
        self.em_blocks = []  # (param base, nch, bs, [flow bases]) grouped by (nch, bs)
        by_shape = {}
        for p0, (nch, bs, f0s) in table.items():
            by_shape.setdefault((nch, bs), []).append((p0, sorted(f0s)))
        for (nch, bs), items in by_shape.items():
            pb = torch.tensor([p for p, _ in items])
            nf = max(len(f) for _, f in items)
            fb = torch.tensor([f + [-1] * (nf - len(f)) for _, f in items])
            self.em_blocks.append((nch, bs, pb, fb))
        K = int(inp["ncats"].max())
        pairs = np.unique(np.stack([inp["s_pids"], inp["s_pfids"], inp["ncats"]], axis=1), axis=0)
        self.in_em = []
        for k in np.unique(pairs[:, 2]):
            sel = pairs[pairs[:, 2] == k]
            self.in_em.append((int(k), T(sel[:, 0]), T(sel[:, 1])))


def forward(tl: TorchLayout, params: torch.Tensor, in_params: torch.Tensor, x: torch.Tensor):
    """node_mars [N, B], element values per product group, lls [B, roots] (FP32)."""
    lay = tl.lay
    B = x.size(0)
    nm = torch.zeros([lay["num_nodes"], B])
    logp = torch.log(in_params)
    nm[tl.in_start:tl.in_start + tl.vids.numel()] = logp[tl.s_pids[:, None] + x[:, tl.vids].T]
    logw = torch.log(params)
    ems = {}
    em = None
    for gi, g in enumerate(tl.groups):
        if g["kind"] == "prod":
            em = torch.full([lay["num_elements"], B], -float("inf"))
            for l in g["layers"]:
                bs = l["bs"]
                for nids, cids in zip(l["nids"], l["cids"]):
                    acc = nm[_rows(cids[:, 0], bs)].clone()
                    for j in range(1, cids.size(1)):
                        acc += nm[_rows(cids[:, j], bs)]
                    em[_rows(nids, bs)] = acc
            ems[gi] = em
            continue
        for l in g["layers"]:
            bs = l["bs"]
            for nids, cids, pids in zip(l["nids"], l["cids"], l["pids"]):
                G, C = cids.shape
                real = (cids != 0)[:, :, None]
                e = torch.where(real, em[cids.reshape(-1)].reshape(G, C, B), -float("inf"))
                w = torch.where(real, torch.exp(logw[pids[:, :, None] + torch.arange(bs)[None, None, :]]), 0.0)
                m = e.amax(dim=1)
                m0 = torch.where(torch.isfinite(m), m, torch.zeros_like(m))
                s = torch.einsum("gci,gcb->gib", w, torch.exp(e - m0[:, None, :]))
                nm[_rows(nids, bs)] = torch.where(torch.isfinite(m)[:, None, :], torch.log(s) + m0[:, None, :],
                                                  torch.full_like(s, -float("inf"))).reshape(G * bs, B)
    r0, r1 = lay["root_range"]
    return nm, ems, nm[r0:r1].T


def backward(tl: TorchLayout, params: torch.Tensor, x: torch.Tensor, nm: torch.Tensor, ems: dict):
    """(param flows, input param flows) with unit root flows (FP32)."""
    lay = tl.lay
    B = x.size(0)
    nf = torch.zeros([lay["num_nodes"], B])
    r0, r1 = lay["root_range"]
    nf[r0:r1] = 1.0
    pf = torch.zeros([lay["num_param_flows"]])
    ef = None
    for gi in range(len(tl.groups) - 1, -1, -1):
        g = tl.groups[gi]
        if g["kind"] == "prod":
            for l in g["layers"]:
                bs = l["bs"]
                for u, par in zip(l["u_cids"], l["parids"]):
                    acc = torch.zeros([u.numel() * bs, B])
                    for q in range(par.size(1)):
                        real = (par[:, q] != 0).repeat_interleave(bs)[:, None]
                        acc += torch.where(real, ef[_rows(par[:, q], bs)], 0.0)
                    nf[_rows(u, bs)] += acc
            continue
        em = ems[gi - 1]
        ef = torch.zeros([lay["num_elements"], B])
        for l in g["layers"]:
            bs = l["bs"]
            ar = torch.arange(bs)
            # log(flow / value) of this layer's nodes only (rows lo .. hi)
            lo, hi = l["nid_range"]
            nmr, nfr = nm[lo:hi], nf[lo:hi]
            fin = torch.isfinite(nmr) & (nfr > 0)
            lr = torch.where(fin, torch.log(nfr) - torch.where(torch.isfinite(nmr), nmr, 0.0), -float("inf"))
            for chids, parids, parpids, cbs in zip(l["chids"], l["parids"], l["parpids"], l["cs_block_sizes"]):
                R, P = parids.shape
                real = (parids != 0).repeat_interleave(bs, dim=1)
                prow = ((parids[:, :, None] + ar).reshape(R, P * bs) - lo).clamp(min=0)
                a = torch.where(real[..., None], lr[prow], -float("inf"))
                m = a.amax(dim=1)
                m = torch.where(torch.isfinite(m), m, torch.zeros_like(m))
                a = torch.exp(a - m[:, None, :])
                wid = parpids[:, None, :, None] + torch.arange(cbs)[None, :, None, None] * bs + ar
                wj = torch.where(real[:, None, :], params[wid.reshape(R, cbs, P * bs)], 0.0)
                acc = torch.einsum("rjk,rkb->rjb", wj, a)
                crow = chids[:, None] + torch.arange(cbs)[None, :]
                ef[crow.reshape(-1)] = (acc * torch.exp(em[crow] + m[:, None, :])).reshape(R * cbs, B)
            for nids, cids, pids, pfids in zip(l["nids"], l["cids"], l["pids"], l["pfids"]):
                R, C = cids.shape
                nrow = nids[:, None] + ar - lo
                a = lr[nrow]
                m = a.amax(dim=1)
                m = torch.where(torch.isfinite(m), m, torch.zeros_like(m))
                a = torch.exp(a - m[:, None, :])
                ce = torch.exp(em[cids] + m[:, None, :])
                s = torch.einsum("rib,rcb->ric", a, ce)
                real = (cids != 0)[:, None, :].expand_as(s)
                slots = (pfids[:, None, :] + ar[None, :, None]).expand_as(s)
                ws = params[pids[:, None, :] + ar[None, :, None]]
                pf.index_add_(0, slots[real], (ws * s)[real])
    in_pf = torch.zeros([tl.in_npf])
    rows = tl.in_start + torch.arange(tl.vids.numel())
    slots = tl.s_pfids[:, None] + x[:, tl.vids].T
    in_pf.index_add_(0, slots.reshape(-1), nf[rows].reshape(-1))
    return pf, in_pf


def em_update(tl: TorchLayout, params: torch.Tensor, pf: torch.Tensor, in_params: torch.Tensor, in_pf: torch.Tensor,
              step_size: float, pseudocount: float):
    """New (params, in_params), FP32 with FP64 normalisers."""
    newp = params.clone()
    for nch, bs, pb, fb in tl.em_blocks:
        idx = (torch.arange(nch * bs)[None, :] + pb[:, None])                 # [n, nch*bs]
        f = torch.zeros(idx.shape, dtype=torch.float64)
        for j in range(fb.size(1)):
            ok = fb[:, j] >= 0
            fi = torch.arange(nch * bs)[None, :] + fb[:, j].clamp(min=0)[:, None]
            f += torch.where(ok[:, None], pf[fi].double(), 0.0)
        f = f.reshape(-1, nch, bs)
        tot = f.sum(dim=1, keepdim=True)
        old = newp[idx].reshape(-1, nch, bs).double()
        newp[idx] = ((1 - step_size) * old + step_size * (f + pseudocount / nch) / (tot + pseudocount)).reshape(
            idx.shape).float()
    new_in = in_params.clone()
    for K, sp, sf in tl.in_em:
        ar = torch.arange(K)
        f = in_pf[sf[:, None] + ar].double()
        # tied input nodes: sum every flow slot of a shared parameter row first
        acc = torch.zeros([new_in.numel()], dtype=torch.float64)
        acc.index_add_(0, (sp[:, None] + ar).reshape(-1), f.reshape(-1))
        rows = torch.unique(sp)[:, None] + ar
        fr = acc[rows]
        new_in[rows] = ((1 - step_size) * new_in[rows].double() + step_size * (fr + pseudocount / K) /
                        (fr.sum(dim=1, keepdim=True) + pseudocount)).float()
    return newp, new_in


def em_step(tl: TorchLayout, params: torch.Tensor, in_params: torch.Tensor, x: torch.Tensor, step_size: float,
            pseudocount: float):
    """One EM step: forward, backward, update. Returns the new parameters and the LLs."""
    nm, ems, lls = forward(tl, params, in_params, x)
    pf, in_pf = backward(tl, params, x, nm, ems)
    p1, q1 = em_update(tl, params, pf, in_params, in_pf, step_size, pseudocount)
    return p1, q1, lls
