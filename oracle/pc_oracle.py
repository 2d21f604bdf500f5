"""CPU oracle of the compiled-circuit passes (test infrastructure, not product code).

Only the test-suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this module, as the checker the CUDA path is compared against; the product never calls
it. It restates the reference's arithmetic in FP64 numpy, driven solely by the compiled
index tables of the reference layout (``partitioned_*`` tensors), so it can run on the
tables of the reference's own compiler (golden fixtures) or of ``pyjuice_b200``.

Reference semantics restated (paths relative to the reference project root):
* input forward   ``log theta[s_pid + x]``           layer/input_layer.py:1016-1054, categorical.py:83-91
* product forward ``sum_j nm[cids[j] + i]``           layer/prod_layer.py:398-466
* sum forward     ``log sum_k theta_k exp(em_k)``     layer/sum_layer.py:454-568, 970-1037
* element flows   ``sum_n nf_n theta_nc em_c / nm_n`` layer/sum_layer.py:1572-1730, 3082-3127
* param flows     ``theta_nc sum_b nf_n em_c / nm_n`` layer/sum_layer.py:2052-2169
* product backward ``nf[u_cid + i] += sum_q ef[parid_q + i]`` layer/prod_layer.py:432-466
* input flows     ``pf[s_pfid + x] += nf``            categorical.py:94-100
* EM              ``(1-s) theta + s (f + pc/n) / (sum f + pc)`` model/backend/par_update.py:174-256,
                  categorical.py:164-244, with tied flow slots summed first
                  (model/backend/parflow_fusing.py:81-99, layer/input_layer.py:1254-1272)
* root flows of ``lls.mean().backward()`` are all 1 (model/tensorcircuit.py:24-37).

Parity is pinned: ``tests/test_oracle_golden.py`` checks this module against the
fixtures that ``tests/golden/make_golden.py`` produced by running the reference itself.
"""

from __future__ import annotations

from typing import Dict, List

import numpy as np


# ----------------------------------------------------------------------------- layout
def layout_from_circuit(pc) -> dict:
    """Reference-layout tables of a ``pyjuice_b200.TensorCircuit`` as numpy arrays."""
    groups = []
    for g in pc.inner_layer_groups:
        layers = []
        for l in g:
            if l.is_sum():
                layers.append(dict(kind="sum", block_size=l.block_size, nid_range=tuple(l._layer_nid_range),
                                   nids=[t.cpu().numpy() for t in l.partitioned_nids],
                                   cids=[t.cpu().numpy() for t in l.partitioned_cids],
                                   pids=[t.cpu().numpy() for t in l.partitioned_pids],
                                   pfids=[t.cpu().numpy() for t in l.partitioned_pfids],
                                   chids=[t.cpu().numpy() for t in l.partitioned_chids],
                                   parids=[t.cpu().numpy() for t in l.partitioned_parids],
                                   parpids=[t.cpu().numpy() for t in l.partitioned_parpids],
                                   cs_block_sizes=list(l.cs_block_sizes)))
            else:
                layers.append(dict(kind="prod", block_size=l.block_size, nid_range=tuple(l._layer_nid_range),
                                   nids=[t.cpu().numpy() for t in l.partitioned_nids],
                                   cids=[t.cpu().numpy() for t in l.partitioned_cids],
                                   u_cids=[t.cpu().numpy() for t in l.partitioned_u_cids],
                                   parids=[t.cpu().numpy() for t in l.partitioned_parids]))
        groups.append(dict(kind=layers[0]["kind"], layers=layers))
    il = pc.input_layer_group[0]
    ncats = il.metadata.cpu()[il.s_mids.cpu()].long().numpy()
    return dict(num_nodes=pc.num_nodes, num_elements=pc.num_elements, root_range=tuple(pc._root_node_range),
                num_sum_params=pc.num_sum_params, num_param_flows=pc.num_param_flows, groups=groups,
                input=dict(nid_start=il._output_ind_range[0], vids=il.vids[:, 0].cpu().numpy(),
                           s_pids=il.s_pids.cpu().numpy(), s_pfids=il.s_pfids.cpu().numpy(), ncats=ncats,
                           num_param_flows=il.num_param_flows))


def layout_from_fixture(fx: Dict[str, np.ndarray], ncats: int) -> dict:
    """Reference-layout tables stored by ``tests/golden/make_golden.py``."""
    groups = []
    gi = 0
    max_prod_bs = 1
    while f"g{gi}_l0_nid_range" in fx:
        layers = []
        li = 0
        while f"g{gi}_l{li}_nid_range" in fx:
            pre = f"g{gi}_l{li}_"
            is_sum = (pre + "pids_count") in fx

            def lst(name):
                return [fx[f"{pre}{name}_{p}"] for p in range(int(fx[pre + name + "_count"]))]

            lo, hi = (int(v) for v in fx[pre + "nid_range"])
            nblocks = sum(x.shape[0] for x in lst("nids"))
            bs = (hi - lo) // max(nblocks, 1)
            if is_sum:
                layers.append(dict(kind="sum", block_size=bs, nid_range=(lo, hi), nids=lst("nids"), cids=lst("cids"),
                                   pids=lst("pids"), pfids=lst("pfids"), chids=lst("chids"), parids=lst("parids"),
                                   parpids=lst("parpids"), cs_block_sizes=[int(v) for v in fx[pre + "cs_block_sizes"]]))
            else:
                max_prod_bs = max(max_prod_bs, bs)
                layers.append(dict(kind="prod", block_size=bs, nid_range=(lo, hi), nids=lst("nids"), cids=lst("cids"),
                                   u_cids=lst("u_cids"), parids=lst("parids")))
            li += 1
        groups.append(dict(kind=layers[0]["kind"], layers=layers))
        gi += 1
    n_in = fx["in_vids"].shape[0]
    return dict(num_nodes=int(fx["num_nodes"]), num_elements=int(fx["num_elements"]),
                root_range=tuple(int(v) for v in fx["root_range"]), num_sum_params=int(fx["num_sum_params"]),
                num_param_flows=int(fx["num_param_flows"]), groups=groups,
                input=dict(nid_start=max_prod_bs, vids=fx["in_vids"][:, 0], s_pids=fx["in_s_pids"],
                           s_pfids=fx["in_s_pfids"], ncats=np.full(n_in, ncats, np.int64),
                           num_param_flows=int(fx["in_param_flows"].shape[0]) if "in_param_flows" in fx else None))


# ----------------------------------------------------------------------------- passes
def _rows(start: np.ndarray, bs: int) -> np.ndarray:
    return (start[:, None] + np.arange(bs)[None, :]).reshape(-1)


def forward(layout: dict, params: np.ndarray, in_params: np.ndarray, x: np.ndarray):
    """Returns (node_mars [N, B], element_mars per inner group index, lls [B])."""
    x = np.asarray(x, dtype=np.int64)
    B = x.shape[0]
    N = layout["num_nodes"]
    nm = np.zeros([N, B], dtype=np.float64)
    inp = layout["input"]
    n_in = inp["vids"].shape[0]
    with np.errstate(divide="ignore"):
        logp = np.log(in_params.astype(np.float64))
        nm[inp["nid_start"]:inp["nid_start"] + n_in] = logp[inp["s_pids"][:, None] + x[:, inp["vids"]].T]
        logw = np.log(params.astype(np.float64))
    ems = {}
    em = None
    for gi, g in enumerate(layout["groups"]):
        if g["kind"] == "prod":
            em = np.full([layout["num_elements"], B], -np.inf)
            for l in g["layers"]:
                bs = l["block_size"]
                for nids, cids in zip(l["nids"], l["cids"]):
                    out = _rows(nids, bs)
                    acc = np.zeros([out.shape[0], B])
                    for j in range(cids.shape[1]):
                        acc += nm[_rows(cids[:, j], bs)]
                    em[out] = acc
            ems[gi] = em
        else:
            for l in g["layers"]:
                bs = l["block_size"]
                for nids, cids, pids in zip(l["nids"], l["cids"], l["pids"]):
                    G, C = cids.shape
                    e = em[cids.reshape(-1)].reshape(G, C, B)                  # [G, C, B]
                    w = logw[pids[:, :, None] + np.arange(bs)[None, None, :]]   # [G, C, bs]
                    w = np.where(cids[:, :, None] == 0, -np.inf, w)
                    t = w.transpose(0, 2, 1)[:, :, :, None] + e[:, None, :, :]  # [G, bs, C, B]
                    m = np.max(t, axis=2, keepdims=True)
                    with np.errstate(invalid="ignore", divide="ignore"):
                        s = np.log(np.sum(np.exp(t - np.where(np.isfinite(m), m, 0.0)), axis=2)) + \
                            np.where(np.isfinite(m[:, :, 0]), m[:, :, 0], 0.0)
                    s = np.where(np.isfinite(m[:, :, 0]), s, -np.inf)
                    nm[_rows(nids, bs)] = s.reshape(G * bs, B)
    r0, r1 = layout["root_range"]
    return nm, ems, nm[r0:r1].T.copy()


def backward(layout: dict, params: np.ndarray, x: np.ndarray, nm: np.ndarray, ems: dict,
             ll_weights: np.ndarray = None):
    """Returns (node_flows [N, B] (unmodified), param_flows, input param_flows) of one batch."""
    x = np.asarray(x, dtype=np.int64)
    B = x.shape[0]
    N = layout["num_nodes"]
    nf = np.zeros([N, B], dtype=np.float64)
    r0, r1 = layout["root_range"]
    nf[r0:r1] = 1.0 if ll_weights is None else ll_weights
    pf = np.zeros([layout["num_param_flows"]], dtype=np.float64)
    w = params.astype(np.float64)
    groups = layout["groups"]
    ef = None
    for gi in range(len(groups) - 1, -1, -1):
        g = groups[gi]
        if g["kind"] == "prod":
            for l in g["layers"]:
                bs = l["block_size"]
                for u, par in zip(l["u_cids"], l["parids"]):
                    tgt = _rows(u, bs)
                    acc = np.zeros([tgt.shape[0], B])
                    for q in range(par.shape[1]):
                        real = np.repeat(par[:, q] != 0, bs)
                        acc += np.where(real[:, None], ef[_rows(par[:, q], bs)], 0.0)
                    nf[tgt] += acc
        else:
            em = ems[gi - 1]
            ef = np.zeros([layout["num_elements"], B])
            # log(flow / mar) of every node; products of huge and tiny factors are formed
            # with a per-sample shift M (max over the nodes involved) to stay in range.
            with np.errstate(divide="ignore", invalid="ignore"):
                lr = np.where(np.isfinite(nm) & (nf > 0), np.log(nf) - np.where(np.isfinite(nm), nm, 0.0), -np.inf)

            def shifted(rows):
                a = lr[rows]
                m = np.max(a, axis=0)
                m = np.where(np.isfinite(m), m, 0.0)
                return np.exp(a - m[None, :]), m

            for l in g["layers"]:
                bs = l["block_size"]
                # element flows
                for chids, parids, parpids, cbs in zip(l["chids"], l["parids"], l["parpids"], l["cs_block_sizes"]):
                    for r in range(chids.shape[0]):
                        npar = int((parids[r] != 0).sum())
                        prow = _rows(parids[r, :npar], bs)                       # parent node rows
                        a, m = shifted(prow)
                        acc = np.zeros([cbs, B])
                        for j in range(cbs):
                            wj = w[(parpids[r, :npar][:, None] + j * bs + np.arange(bs)[None, :]).reshape(-1)]
                            acc[j] = wj @ a
                        crow = chids[r] + np.arange(cbs)
                        ef[crow] = acc * np.exp(em[crow] + m[None, :])
                # parameter flows
                for nids, cids, pids, pfids in zip(l["nids"], l["cids"], l["pids"], l["pfids"]):
                    for r in range(nids.shape[0]):
                        cnt = int((cids[r] != 0).sum())
                        nrow = nids[r] + np.arange(bs)
                        a, m = shifted(nrow)
                        ce = np.exp(em[cids[r, :cnt]] + m[None, :])               # [C, B]
                        s = a @ ce.T                                               # [bs, C]
                        slots = pfids[r, :cnt][None, :] + np.arange(bs)[:, None]
                        ws = w[pids[r, :cnt][None, :] + np.arange(bs)[:, None]]
                        np.add.at(pf, slots.reshape(-1), (ws * s).reshape(-1))
    inp = layout["input"]
    n_in = inp["vids"].shape[0]
    npf = inp["num_param_flows"] if inp.get("num_param_flows") else int(inp["s_pfids"].max() + inp["ncats"].max())
    in_pf = np.zeros([npf], dtype=np.float64)
    rows = inp["nid_start"] + np.arange(n_in)
    slots = inp["s_pfids"][:, None] + x[:, inp["vids"]].T
    np.add.at(in_pf, slots.reshape(-1), nf[rows].reshape(-1))
    return nf, pf, in_pf


def _sum_node_table(layout: dict):
    """(param ids row, flow ids row) of every sum node, one entry per node of every block."""
    out = []
    for g in layout["groups"]:
        if g["kind"] != "sum":
            continue
        for l in g["layers"]:
            bs = l["block_size"]
            for cids, pids, pfids in zip(l["cids"], l["pids"], l["pfids"]):
                for r in range(cids.shape[0]):
                    cnt = int((cids[r] != 0).sum())
                    for i in range(bs):
                        out.append((pids[r, :cnt] + i, pfids[r, :cnt] + i))
    return out


def em_update(layout: dict, params: np.ndarray, pf: np.ndarray, in_params: np.ndarray, in_pf: np.ndarray,
              step_size: float, pseudocount: float):
    """One EM step (keep_zero_params=False); returns new (params, in_params) as float64."""
    newp = params.astype(np.float64).copy()
    groups: Dict[tuple, set] = {}
    for prow, frow in _sum_node_table(layout):
        key = tuple(prow.tolist())
        groups.setdefault(key, set()).add(tuple(frow.tolist()))
    for key, frows in groups.items():
        prow = np.array(key, dtype=np.int64)
        f = np.zeros(prow.shape[0])
        for fr in frows:
            f += pf[np.array(fr, dtype=np.int64)]
        nch = prow.shape[0]
        tot = f.sum()
        newp[prow] = (1 - step_size) * newp[prow] + step_size * (f + pseudocount / nch) / (tot + pseudocount)
    inp = layout["input"]
    new_in = in_params.astype(np.float64).copy()
    by_pid: Dict[int, set] = {}
    for sp, spf, k in zip(inp["s_pids"], inp["s_pfids"], inp["ncats"]):
        by_pid.setdefault((int(sp), int(k)), set()).add(int(spf))
    for (sp, K), spfs in by_pid.items():
        f = np.zeros(K)
        for s in spfs:
            f += in_pf[s:s + K]
        new_in[sp:sp + K] = (1 - step_size) * new_in[sp:sp + K] + step_size * (f + pseudocount / K) / (f.sum() + pseudocount)
    return newp, new_in


# ----------------------------------------------------------------------------- sampling
def uniform(seed: int, node: int, sample: int) -> np.float32:
    """The sampler's uniform draw: top 24 bits of SplitMix64(seed + (counter + 1) * golden)."""
    m = (1 << 64) - 1
    g = 0x9E3779B97F4A7C15
    z = (seed + ((((node << 32) | sample) + 1) * g)) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    z = z ^ (z >> 31)
    return np.float32((z >> 40) * (1.0 / 16777216.0))


def sample(layout: dict, params: np.ndarray, in_params: np.ndarray, num_samples: int, seed: int,
           num_vars: int) -> np.ndarray:
    """Top-down sampling with the device sampler's draw rules (small circuits only)."""
    p32 = params.astype(np.float32)
    ip32 = in_params.astype(np.float32)
    # node id -> (children element ids, param ids) for sum nodes; element id -> child node ids
    sum_ch: Dict[int, tuple] = {}
    prod_ch: Dict[int, List[int]] = {}
    for g in layout["groups"]:
        for l in g["layers"]:
            bs = l["block_size"]
            if l["kind"] == "sum":
                for nids, cids, pids in zip(l["nids"], l["cids"], l["pids"]):
                    for r in range(nids.shape[0]):
                        cnt = int((cids[r] != 0).sum())
                        for i in range(bs):
                            sum_ch[int(nids[r]) + i] = (cids[r, :cnt], pids[r, :cnt] + i)
            else:
                for nids, cids in zip(l["nids"], l["cids"]):
                    for r in range(nids.shape[0]):
                        real = cids[r][cids[r] != 0]
                        for i in range(bs):
                            prod_ch[int(nids[r]) + i] = [int(c) + i for c in real]
    inp = layout["input"]
    in0 = inp["nid_start"]
    out = np.zeros([num_samples, num_vars], dtype=np.int64)
    r0 = layout["root_range"][0]
    for s in range(num_samples):
        stack = [r0]
        while stack:
            n = stack.pop()
            if n in sum_ch:
                ch, pid = sum_ch[n]
                u = uniform(seed, n, s)
                cum = np.float32(0.0)
                pick, last_nz = -1, 0
                for k in range(ch.shape[0]):
                    wk = p32[pid[k]]
                    cum = np.float32(cum + wk)
                    if wk > 0:
                        last_nz = k
                    if u < cum:
                        pick = k
                        break
                if pick < 0:
                    pick = last_nz
                stack.extend(prod_ch[int(ch[pick])])
            else:
                li = n - in0
                K = int(inp["ncats"][li])
                sp = int(inp["s_pids"][li])
                u = uniform(seed, n, s)
                cum = np.float32(0.0)
                pick = 0
                for k in range(K):
                    cum = np.float32(cum + ip32[sp + k])
                    if cum >= u:
                        pick = k
                        break
                out[s, int(inp["vids"][li])] = pick
    return out
