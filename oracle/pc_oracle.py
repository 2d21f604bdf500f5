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


def _mask_rows(layout: dict, missing_mask, B: int) -> np.ndarray:
    """[n_in, B] bool: input node n is summed out in sample b (mask [V] or [B, V])."""
    vids = layout["input"]["vids"]
    m = np.asarray(missing_mask, dtype=bool)
    return np.broadcast_to(m[vids][:, None], (vids.shape[0], B)) if m.ndim == 1 else m[:, vids].T


def input_values(layout: dict, in_params: np.ndarray, x: np.ndarray = None, evidence: np.ndarray = None,
                 missing_mask=None) -> np.ndarray:
    """[n_in, B] log values of the Categorical input nodes: hard evidence ``log theta[x]``
    (categorical.py:83-91), soft evidence ``min(log sum_k E[b, v, k] theta[k], 0)``
    (queries/conditional.py:25-68, 108-111); 0 where ``missing_mask`` marks the variable
    (input_layer.py:1059-1095)."""
    inp = layout["input"]
    theta = in_params.astype(np.float64)
    with np.errstate(divide="ignore"):
        if evidence is None:
            x = np.asarray(x, dtype=np.int64)
            vals = np.log(theta)[inp["s_pids"][:, None] + x[:, inp["vids"]].T]
        else:
            ev = np.asarray(evidence, dtype=np.float64)                            # [B, V, K]
            K = int(inp["ncats"].max())
            th = theta[np.minimum(inp["s_pids"][:, None] + np.arange(K)[None, :], theta.shape[0] - 1)]
            th = np.where(np.arange(K)[None, :] < inp["ncats"][:, None], th, 0.0)  # [n_in, K]
            vals = np.minimum(np.log(np.einsum("nk,bnk->nb", th, ev[:, inp["vids"], :K])), 0.0)
    if missing_mask is not None:
        vals = np.where(_mask_rows(layout, missing_mask, vals.shape[1]), 0.0, vals)
    return vals


def forward(layout: dict, params: np.ndarray, in_params: np.ndarray, x: np.ndarray = None, missing_mask=None,
            evidence: np.ndarray = None):
    """Returns (node_mars [N, B], element_mars per inner group index, lls [B]). Hard
    evidence ``x`` [B, V] or soft evidence ``evidence`` [B, V, K]; variables marked in
    ``missing_mask`` are summed out."""
    vals = input_values(layout, in_params, x, evidence, missing_mask)
    B = vals.shape[1]
    N = layout["num_nodes"]
    nm = np.zeros([N, B], dtype=np.float64)
    inp = layout["input"]
    n_in = inp["vids"].shape[0]
    nm[inp["nid_start"]:inp["nid_start"] + n_in] = vals
    with np.errstate(divide="ignore"):
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
                    e = np.where(cids[:, :, None] == 0, -np.inf, e)
                    w = np.exp(logw[pids[:, :, None] + np.arange(bs)[None, None, :]])   # [G, C, bs]
                    w = np.where(cids[:, :, None] == 0, 0.0, w)
                    m = np.max(e, axis=1)                                       # [G, B]
                    fin = np.isfinite(m)
                    m0 = np.where(fin, m, 0.0)
                    s = np.einsum("gci,gcb->gib", w, np.exp(e - m0[:, None, :]))  # [G, bs, B]
                    with np.errstate(divide="ignore"):
                        s = np.where(fin[:, None, :], np.log(s) + m0[:, None, :], -np.inf)
                    nm[_rows(nids, bs)] = s.reshape(G * bs, B)
    r0, r1 = layout["root_range"]
    return nm, ems, nm[r0:r1].T.copy()


def backward(layout: dict, params: np.ndarray, x: np.ndarray, nm: np.ndarray, ems: dict,
             ll_weights: np.ndarray = None, missing_mask=None, in_params: np.ndarray = None):
    """Returns (node_flows [N, B] (unmodified), param_flows, input param_flows) of one batch.
    Where ``missing_mask`` marks a variable, an input node's flow goes to every category k
    as ``flow * theta[k]`` (categorical.py:102-134; needs ``in_params``). ``x`` None: no
    input flows from observed values (soft evidence)."""
    x = None if x is None else np.asarray(x, dtype=np.int64)
    B = nm.shape[1]
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

            def shifted(rows, real):
                """exp(lr[rows] - M) with M the max over axis 1 (the nodes involved), per sample."""
                a = np.where(real[..., None], lr[rows], -np.inf)               # [R, K, B]
                m = np.max(a, axis=1)
                m = np.where(np.isfinite(m), m, 0.0)
                return np.exp(a - m[:, None, :]), m

            ar = None
            for l in g["layers"]:
                bs = l["block_size"]
                ar = np.arange(bs)
                # element flows: one batched contraction per partition
                for chids, parids, parpids, cbs in zip(l["chids"], l["parids"], l["parpids"], l["cs_block_sizes"]):
                    R, P = parids.shape
                    real = np.repeat(parids != 0, bs, axis=1)                      # [R, P*bs]
                    prow = (parids[:, :, None] + ar).reshape(R, P * bs)
                    a, m = shifted(prow, real)
                    wid = parpids[:, None, :, None] + np.arange(cbs)[None, :, None, None] * bs + ar
                    wj = np.where(real[:, None, :], w[wid.reshape(R, cbs, P * bs)], 0.0)   # [R, cbs, P*bs]
                    acc = np.einsum("rjk,rkb->rjb", wj, a)
                    crow = chids[:, None] + np.arange(cbs)[None, :]                 # [R, cbs]
                    ef[crow.reshape(-1)] = (acc * np.exp(em[crow] + m[:, None, :])).reshape(R * cbs, B)
                # parameter flows: one batched contraction (over the batch) per partition
                for nids, cids, pids, pfids in zip(l["nids"], l["cids"], l["pids"], l["pfids"]):
                    R, C = cids.shape
                    nrow = nids[:, None] + ar                                       # [R, bs]
                    a, m = shifted(nrow, np.ones_like(nrow, dtype=bool))
                    ce = np.exp(em[cids] + m[:, None, :])                           # [R, C, B]
                    s = np.einsum("rib,rcb->ric", a, ce)                            # [R, bs, C]
                    real = np.broadcast_to((cids != 0)[:, None, :], s.shape)
                    slots = pfids[:, None, :] + ar[None, :, None]
                    ws = w[pids[:, None, :] + ar[None, :, None]]
                    np.add.at(pf, slots[real], (ws * s)[real])
    inp = layout["input"]
    n_in = inp["vids"].shape[0]
    npf = inp["num_param_flows"] if inp.get("num_param_flows") else int(inp["s_pfids"].max() + inp["ncats"].max())
    in_pf = np.zeros([npf], dtype=np.float64)
    rows = inp["nid_start"] + np.arange(n_in)
    flows = nf[rows]
    if missing_mask is not None:
        miss = _mask_rows(layout, missing_mask, B)
        theta = in_params.astype(np.float64)
        msum = np.where(miss, flows, 0.0).sum(axis=1)
        for k in range(int(inp["ncats"].max())):
            ok = k < inp["ncats"]
            np.add.at(in_pf, inp["s_pfids"][ok] + k, msum[ok] * theta[inp["s_pids"][ok] + k])
        flows = np.where(miss, 0.0, flows)
    if x is not None:
        slots = inp["s_pfids"][:, None] + x[:, inp["vids"]].T
        np.add.at(in_pf, slots.reshape(-1), flows.reshape(-1))
    return nf, pf, in_pf


def conditional(layout: dict, in_params: np.ndarray, nf: np.ndarray, target_vars=None, scale=None) -> np.ndarray:
    """The conditional query's category distributions ``[B, T, K]``: per target variable,
    ``sum_n nf[n, b] theta[n, k]`` over its input nodes, normalised over k with + 1e-12
    (queries/conditional.py:241-336). ``scale`` ([n_in, B], optional) multiplies the flows
    first and skips the normalisation (the soft-evidence adjoint uses 1 / exp(node_mars))."""
    inp = layout["input"]
    n_in = inp["vids"].shape[0]
    K = int(inp["ncats"].max())
    f = nf[inp["nid_start"]:inp["nid_start"] + n_in]
    if scale is not None:
        f = f * scale
    theta = in_params.astype(np.float64)
    th = theta[np.minimum(inp["s_pids"][:, None] + np.arange(K)[None, :], theta.shape[0] - 1)]
    th = np.where(np.arange(K)[None, :] < inp["ncats"][:, None], th, 0.0)
    tv = range(int(inp["vids"].max()) + 1) if target_vars is None else target_vars
    out = np.stack([np.einsum("nb,nk->bk", f[inp["vids"] == v], th[inp["vids"] == v]) for v in tv], axis=1)
    if scale is None:
        out = out / (out.sum(axis=2, keepdims=True) + 1e-12)
    return out


def forward_alg(layout: dict, params: np.ndarray, in_params: np.ndarray, x: np.ndarray, alg: str = "LL",
                alpha: float = 1.0):
    """Forward pass under a propagation algorithm (layer/sum_layer.py:500-563): "LL"
    (``forward``), "MPE" ``max_c (log w + e_c)``, "GeneralLL"
    ``(log(sum_c w^a exp(a (e_c - m)) + 1e-24) + a m) / a``. Returns (node_mars, ems, lls)."""
    if alg == "LL":
        return forward(layout, params, in_params, x)
    x = np.asarray(x, dtype=np.int64)
    B = x.shape[0]
    nm = np.zeros([layout["num_nodes"], B])
    inp = layout["input"]
    n_in = inp["vids"].shape[0]
    with np.errstate(divide="ignore"):
        nm[inp["nid_start"]:inp["nid_start"] + n_in] = np.log(in_params.astype(np.float64))[
            inp["s_pids"][:, None] + x[:, inp["vids"]].T]
        logw = np.log(params.astype(np.float64))
    ems, em = {}, None
    for gi, g in enumerate(layout["groups"]):
        if g["kind"] == "prod":
            em = np.full([layout["num_elements"], B], -np.inf)
            for l in g["layers"]:
                bs = l["block_size"]
                for nids, cids in zip(l["nids"], l["cids"]):
                    acc = np.zeros([nids.shape[0] * bs, B])
                    for j in range(cids.shape[1]):
                        acc += nm[_rows(cids[:, j], bs)]
                    em[_rows(nids, bs)] = acc
            ems[gi] = em
            continue
        for l in g["layers"]:
            bs = l["block_size"]
            for nids, cids, pids in zip(l["nids"], l["cids"], l["pids"]):
                G, C = cids.shape
                e = np.where(cids[:, :, None] == 0, -np.inf, em[cids.reshape(-1)].reshape(G, C, B))
                lw = np.where(cids[:, :, None] == 0, -np.inf, logw[pids[:, :, None] + np.arange(bs)[None, None, :]])
                if alg == "MPE":
                    s = np.max(lw[:, :, :, None] + e[:, :, None, :], axis=1)         # [G, bs, B]
                else:
                    m = np.max(e, axis=1)
                    fin = np.isfinite(m)
                    m0 = np.where(fin, m, 0.0)
                    t = np.exp(alpha * lw)[:, :, :, None] * np.exp(alpha * (e - m0[:, None, :]))[:, :, None, :]
                    with np.errstate(divide="ignore"):
                        s = np.where(fin[:, None, :], (np.log(t.sum(axis=1) + 1e-24) + alpha * m0[:, None, :]) / alpha,
                                     -np.inf)
                nm[_rows(nids, bs)] = s.reshape(G * bs, B)
    r0, r1 = layout["root_range"]
    return nm, ems, nm[r0:r1].T.copy()


def _lse(a, axis):
    m = np.max(a, axis=axis, keepdims=True)
    m0 = np.where(np.isfinite(m), m, 0.0)
    with np.errstate(divide="ignore"):
        out = np.log(np.exp(a - m0).sum(axis=axis, keepdims=True)) + m0
    return np.squeeze(np.where(np.isfinite(m), out, -np.inf), axis=axis)


def backward_alg(layout: dict, params: np.ndarray, x: np.ndarray, nm: np.ndarray, ems: dict, alg: str = "LL",
                 alpha: float = 1.0, logspace: bool = False, negate: bool = False, ll_weights: np.ndarray = None):
    """Backward pass under a propagation algorithm, in linear or log-space flows, with
    optionally negated parameter flows (sum_layer.py:1572-1730, 2052-2169, 3068-3127;
    prod_layer.py:432-466; categorical.py:94-100). Small circuits only (dense per-edge
    arrays). Returns (node_flows, param_flows, input param_flows).

    Element flows of child c with parents n (weight w, flow f, value m):
      LL  f w exp(e - m);  GeneralLL  f w^a exp(a (e - m));  MPE  f where |log w + e - m| < 1e-6
    summed (log space: log-sum-exp of the logs). Parameter flows of edge (n, c):
      LL / GeneralLL  w sum_b f exp(e - m) (log space: w sum_b exp(f + e - m), exp(f) where
      m = -inf);  MPE  sum_b [|log w + e - m| < 1e-6] f (log space: exp(f)).
    """
    x = np.asarray(x, dtype=np.int64)
    B = x.shape[0]
    N = layout["num_nodes"]
    nf = np.full([N, B], -np.inf if logspace else 0.0)
    r0, r1 = layout["root_range"]
    w_root = np.ones([r1 - r0, B]) if ll_weights is None else np.broadcast_to(ll_weights, (r1 - r0, B))
    with np.errstate(divide="ignore"):
        nf[r0:r1] = np.log(w_root) if logspace else w_root
    pf = np.zeros([layout["num_param_flows"]])
    w = params.astype(np.float64)
    with np.errstate(divide="ignore"):
        lw_all = np.log(w)
    groups = layout["groups"]
    ef = None
    sign = -1.0 if negate else 1.0
    for gi in range(len(groups) - 1, -1, -1):
        g = groups[gi]
        if g["kind"] == "prod":
            for l in g["layers"]:
                bs = l["block_size"]
                for u, par in zip(l["u_cids"], l["parids"]):
                    tgt = _rows(u, bs)
                    cols = [np.where(np.repeat(par[:, q] != 0, bs)[:, None], ef[_rows(par[:, q], bs)],
                                     -np.inf if logspace else 0.0) for q in range(par.shape[1])]
                    if logspace:
                        nf[tgt] = _lse(np.stack([nf[tgt]] + cols), axis=0)
                    else:
                        nf[tgt] += np.sum(cols, axis=0)
            continue
        em = ems[gi - 1]
        ef = np.full([layout["num_elements"], B], -np.inf if logspace else 0.0)
        for l in g["layers"]:
            bs = l["block_size"]
            ar = np.arange(bs)
            for chids, parids, parpids, cbs in zip(l["chids"], l["parids"], l["parpids"], l["cs_block_sizes"]):
                for r in range(chids.shape[0]):
                    pr = parids[r][parids[r] != 0]
                    pp = parpids[r][:pr.shape[0]]
                    nrow = (pr[:, None] + ar).reshape(-1)                        # parents [K]
                    for j in range(cbs):
                        c = int(chids[r]) + j
                        lw = lw_all[(pp[:, None] + j * bs + ar).reshape(-1)]     # [K]
                        f, m, e = nf[nrow], nm[nrow], em[c][None, :]
                        with np.errstate(invalid="ignore", over="ignore"):
                            d = lw[:, None] + e - m
                            if alg == "MPE":
                                hit = np.isfinite(m) & (np.abs(d) < 1e-6)
                                v = _lse(np.where(hit, f, -np.inf), 0) if logspace else np.where(hit, f, 0.0).sum(0)
                            else:
                                xx = np.where(np.isfinite(m), alpha * d if alg == "GeneralLL" else d, -np.inf)
                                v = _lse(f + xx, 0) if logspace else np.where(np.isfinite(xx), f * np.exp(xx), 0.0).sum(0)
                        ef[c] = v
            for nids, cids, pids, pfids in zip(l["nids"], l["cids"], l["pids"], l["pfids"]):
                for r in range(nids.shape[0]):
                    real = cids[r] != 0
                    for i in range(bs):
                        n = int(nids[r]) + i
                        f, m = nf[n][None, :], nm[n][None, :]
                        wv = w[pids[r][real] + i][:, None]
                        e = em[cids[r][real]]
                        with np.errstate(invalid="ignore", over="ignore", divide="ignore"):
                            if alg == "MPE":
                                hit = np.abs(np.log(wv) + e - m) < 1e-6
                                v = np.where(hit, np.exp(f) if logspace else f, 0.0).sum(1)
                            elif logspace:
                                v = wv[:, 0] * np.where(np.isfinite(m), np.exp(f + e - m), np.exp(f)).sum(1)
                            else:
                                v = wv[:, 0] * np.where(np.isfinite(m), f * np.exp(e - m), 0.0).sum(1)
                        np.add.at(pf, pfids[r][real] + i, sign * v)
    inp = layout["input"]
    n_in = inp["vids"].shape[0]
    npf = inp["num_param_flows"] if inp.get("num_param_flows") else int(inp["s_pfids"].max() + inp["ncats"].max())
    in_pf = np.zeros([npf])
    rows = inp["nid_start"] + np.arange(n_in)
    slots = inp["s_pfids"][:, None] + x[:, inp["vids"]].T
    vals = np.exp(nf[rows]) if logspace else nf[rows]
    np.add.at(in_pf, slots.reshape(-1), vals.reshape(-1))
    return nf, pf, in_pf


def _sum_block_table(layout: dict):
    """Per distinct parameter slab: (first param id, #children, block size, set of first flow ids).

    In the compiled layout the weights of a node block are ``pids[r, 0] + k * bs + i`` and
    its flows ``pfids[r, 0] + k * bs + i``; tied node blocks share ``pids[r, 0]`` and may
    own separate flow slots, which EM sums first.
    """
    table: Dict[int, list] = {}
    for g in layout["groups"]:
        if g["kind"] != "sum":
            continue
        for l in g["layers"]:
            bs = l["block_size"]
            for cids, pids, pfids in zip(l["cids"], l["pids"], l["pfids"]):
                cnts = (cids != 0).sum(axis=1)
                for r in range(cids.shape[0]):
                    ent = table.setdefault(int(pids[r, 0]), [int(cnts[r]), bs, set()])
                    ent[2].add(int(pfids[r, 0]))
    return table


def em_update(layout: dict, params: np.ndarray, pf: np.ndarray, in_params: np.ndarray, in_pf: np.ndarray,
              step_size: float, pseudocount: float, keep_zero_params: bool = False):
    """One EM step; returns new (params, in_params) as float64.

    keep_zero_params (par_update.py:199-203, 238-248; categorical.py:180-198): parameters
    below 1e-12 stay zero, and the normaliser is the sum of ``flow + pc / n`` over the
    other entries (no extra pseudocount)."""
    newp = params.astype(np.float64).copy()
    for p0, (nch, bs, f0s) in _sum_block_table(layout).items():
        n = nch * bs
        f = np.zeros(n)
        for f0 in f0s:
            f += pf[f0:f0 + n]
        f = f.reshape(nch, bs)
        old = newp[p0:p0 + n].reshape(nch, bs)
        if keep_zero_params:
            nz = old >= 1e-12
            tot = np.where(nz, f + pseudocount / nch, 0.0).sum(axis=0)
            upd = (1 - step_size) * old + step_size * (f + pseudocount / nch) / tot
            newp[p0:p0 + n] = np.where(nz, upd, 0.0).reshape(-1)
            continue
        tot = f.sum(axis=0)                                    # per node of the block
        newp[p0:p0 + n] = ((1 - step_size) * old + step_size * (f + pseudocount / nch) / (tot + pseudocount)).reshape(-1)
    inp = layout["input"]
    new_in = in_params.astype(np.float64).copy()
    pairs = np.unique(np.stack([inp["s_pids"], inp["s_pfids"], inp["ncats"]], axis=1), axis=0)
    for K in np.unique(pairs[:, 2]):
        sel = pairs[pairs[:, 2] == K]
        ar = np.arange(int(K))
        acc = np.zeros([new_in.shape[0]])
        np.add.at(acc, (sel[:, 0:1] + ar).reshape(-1), in_pf[(sel[:, 1:2] + ar).reshape(-1)])
        sp = np.unique(sel[:, 0])
        rows = sp[:, None] + ar                                # [n, K]
        f = acc[rows]
        if keep_zero_params:
            old = new_in[rows]
            nz = old >= 1e-12
            tot = np.where(nz, f + pseudocount / K, 0.0).sum(axis=1, keepdims=True)
            new_in[rows] = np.where(nz, (1 - step_size) * old + step_size * (f + pseudocount / K) / tot, 0.0)
            continue
        new_in[rows] = (1 - step_size) * new_in[rows] + step_size * (f + pseudocount / K) / (
            f.sum(axis=1, keepdims=True) + pseudocount)
    return newp, new_in


def normalize(layout: dict, params: np.ndarray, pseudocount: float) -> np.ndarray:
    """Sum-to-one normalisation of every node's weights, ``(p + pc / n) / (sum p + pc)``
    (nodes/backend/normalize.py:13-68, model/tensorcircuit.py:1118-1120)."""
    newp = params.astype(np.float64).copy()
    for p0, (nch, bs, _) in _sum_block_table(layout).items():
        w = newp[p0:p0 + nch * bs].reshape(nch, bs)
        newp[p0:p0 + nch * bs] = ((w + pseudocount / nch) / (w.sum(axis=0) + pseudocount)).reshape(-1)
    return newp


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


def uniform_table(seed: int, num_nodes: int, num_samples: int) -> np.ndarray:
    """``[num_nodes, num_samples]`` float32 table of :func:`uniform` (vectorised)."""
    g = np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        ctr = (np.arange(num_nodes, dtype=np.uint64)[:, None] << np.uint64(32)) | \
            np.arange(num_samples, dtype=np.uint64)[None, :]
        z = np.uint64(seed) + (ctr + np.uint64(1)) * g
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return ((z >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)).astype(np.float32)


def sample(layout: dict, params: np.ndarray, in_params: np.ndarray, num_samples: int, seed: int,
           num_vars: int) -> np.ndarray:
    """Top-down sampling with the device sampler's draw rules (small circuits only)."""
    p32 = params.astype(np.float32)
    ip32 = in_params.astype(np.float32)
    # node id -> (children element ids, param ids, product group) for sum nodes;
    # (product group, element id) -> child node ids. Element ids are reused by every
    # product layer group, so they are only meaningful together with their group.
    sum_ch: Dict[int, tuple] = {}
    prod_ch: Dict[tuple, List[int]] = {}
    for gi, g in enumerate(layout["groups"]):
        for l in g["layers"]:
            bs = l["block_size"]
            if l["kind"] == "sum":
                for nids, cids, pids in zip(l["nids"], l["cids"], l["pids"]):
                    for r in range(nids.shape[0]):
                        cnt = int((cids[r] != 0).sum())
                        for i in range(bs):
                            sum_ch[int(nids[r]) + i] = (cids[r, :cnt], pids[r, :cnt] + i, gi - 1)
            else:
                for nids, cids in zip(l["nids"], l["cids"]):
                    for r in range(nids.shape[0]):
                        real = cids[r][cids[r] != 0]
                        for i in range(bs):
                            prod_ch[(gi, int(nids[r]) + i)] = [int(c) + i for c in real]
    inp = layout["input"]
    in0 = inp["nid_start"]
    out = np.zeros([num_samples, num_vars], dtype=np.int64)
    r0 = layout["root_range"][0]
    for s in range(num_samples):
        stack = [r0]
        while stack:
            n = stack.pop()
            if n in sum_ch:
                ch, pid, pg = sum_ch[n]
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
                stack.extend(prod_ch[(pg, int(ch[pick]))])
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
