"""Shared helpers: rebuild fixture circuits with pyjuice_b200 and compare layouts."""

from __future__ import annotations

import numpy as np
import torch

import pyjuice_b200 as juice
from pyjuice_b200.nodes import distributions as dists
from pyjuice_b200.structures import hclt_from_tree

from circuits import build_tiny_dag


def tree_from_fixture(fx):
    seq = [int(v) for v in fx["tree_seq"]]
    off = fx["tree_children_off"]
    flat = fx["tree_children"]
    children = {v: [int(c) for c in flat[off[v]:off[v + 1]]] for v in range(len(seq))}
    return seq, children, int(fx["tree_root"])


def build_fixture_circuit(name: str, fx):
    if name == "tiny":
        root = build_tiny_dag(juice, dists)
        return juice.compile(root, max_tied_ns_per_parflow_block=1)
    seq, children, root_v = tree_from_fixture(fx)
    if name == "hclt64":
        root = hclt_from_tree(seq, children, root_v, 16, input_dist=dists.Categorical(num_cats=4), block_size=16)
    elif name == "hclt784":
        root = hclt_from_tree(seq, children, root_v, 128, input_dist=dists.Categorical(num_cats=256), block_size=32)
    else:
        raise ValueError(name)
    return juice.compile(root)


def layout_mismatches(pc, fx, full: bool = True):
    """Names of index tensors that differ from the fixture (empty list = identical)."""
    import hashlib
    bad = []
    for gi, g in enumerate(pc.inner_layer_groups):
        for li, l in enumerate(g):
            pre = f"g{gi}_l{li}_"
            if (pre + "nid_range") not in fx:
                bad.append(pre + "missing")
                continue
            if tuple(int(v) for v in fx[pre + "nid_range"]) != tuple(l._layer_nid_range):
                bad.append(pre + "nid_range")
            names = ["nids", "cids", "pids", "pfids", "chids", "parids", "parpids"] if l.is_sum() else \
                ["nids", "cids", "u_cids", "parids"]
            for n in names:
                tl = getattr(l, "partitioned_" + n)
                if int(fx[pre + n + "_count"]) != len(tl):
                    bad.append(pre + n + "_count")
                    continue
                for p, t in enumerate(tl):
                    if full:
                        ref = fx[f"{pre}{n}_{p}"]
                        if ref.shape != tuple(t.shape) or not np.array_equal(ref, t.cpu().numpy()):
                            bad.append(f"{pre}{n}_{p}")
                    else:
                        d = hashlib.sha256(t.detach().cpu().long().contiguous().numpy().tobytes()).hexdigest()
                        if str(fx[f"{pre}{n}_{p}_sha"]) != d:
                            bad.append(f"{pre}{n}_{p}")
    if f"g{len(pc.inner_layer_groups)}_l0_nid_range" in fx:
        bad.append("extra groups in fixture")
    for key in ("num_nodes", "num_elements", "num_sum_params", "num_param_flows"):
        if int(fx[key]) != int(getattr(pc, key)):
            bad.append(key)
    return bad


def fixture_params(pc, fx):
    """(sum params, input params) of a fixture: stored, or regenerated from its seed."""
    if "params0" in fx:
        return fx["params0"], fx["in_params0"]
    from circuits import seeded_params
    il = pc.input_layer_group[0]
    ncats = int(il.metadata[0].item())
    return seeded_params(pc._em_pbase.tolist(), pc._em_nch.tolist(), pc._em_bs.tolist(), pc.num_sum_params,
                         il.num_nodes, ncats, seed=int(fx["param_seed"]))


def load_fixture_params(pc, fx):
    p, q = fixture_params(pc, fx)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(p).to(pc.params.device))
        il = pc.input_layer_group[0]
        il.params.copy_(torch.from_numpy(q).to(il.params.device))
