"""Host-side plans of the fused passes, checked on the CPU against the compiled index tensors.

* Product fusion (TensorCircuit._plan_product_fusion): the forward table lists, for every
  term of the sum layer, the child node rows of that term's element; the backward table
  lists every element's child rows, each child row once.
* Flow rewrite (TensorCircuit._rewrite_plan): every row of a rewritten large level has
  exactly one product writer, that writer is not fused away, and its flagged child blocks
  are exactly the blocks inside rewritten levels.
"""

import numpy as np
import pytest
import torch

from conftest import load_fixture
from helpers import build_fixture_circuit

from pyjuice_b200.layer.layers import SumLayer


def _element_children(layer, rows):
    """{element row: sorted child node rows} from partitioned_nids / partitioned_cids."""
    out = dict()
    bs = layer.block_size
    for nids, cids in zip(layer.partitioned_nids, layer.partitioned_cids):
        nids, cids = nids.cpu().numpy(), cids.cpu().numpy()
        for l in range(nids.shape[0]):
            ch = cids[l][cids[l] != 0]
            for i in range(bs):
                out[int(nids[l]) + i] = sorted(int(c) + i for c in ch)
    return out


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_product_fusion_tables(name):
    fx = load_fixture(name)
    pc = build_fixture_circuit(name, fx)
    assert pc._fusion_host
    for gi, tabs in pc._fusion_host.items():
        pl = pc.inner_layer_groups[gi][0]
        sl = pc.inner_layer_groups[gi + 1][0]
        rows = pc._em_region[gi][1]
        ech = _element_children(pl, rows)
        krow = sl._host_desc()["krow"].numpy()
        fw = tabs["fw"].reshape(-1, 4)
        assert fw.shape[0] == krow.shape[0]
        for k, e in enumerate(krow.tolist()):
            assert sorted(int(c) for c in fw[k] if c >= 0) == ech[e]
        if tabs["bw"] is None:
            continue
        bw = tabs["bw"].reshape(-1, 4)
        seen = []
        for e, ch in ech.items():
            assert sorted(int(c) for c in bw[e] if c >= 0) == ch
            seen += ch
        assert len(seen) == len(set(seen)), "a child row with two parent elements"


def test_flow_rewrite_plan():
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx)
    saved = SumLayer.tc05_min_tiles
    try:
        SumLayer.tc05_min_tiles = 1  # every level counts as large
        for fused in (frozenset(), frozenset(g - 1 for g in range(len(pc.inner_layer_groups))
                                             if pc.inner_layer_groups[g].is_sum() and (g - 1) in pc._fusion_host
                                             and pc._fusion_host[g - 1]["bw"] is not None)):
            flags, done = pc._rewrite_plan(fused)
            if not fused:
                assert done and flags  # without product fusion every single-writer level qualifies
            groups = pc.inner_layer_groups
            ranges = [groups[gs][0]._layer_nid_range for gs in done]
            for lo, hi in ranges:
                assert np.all(pc._row_nwriters[lo:hi] == 1)
                assert not set(int(g) for g in np.unique(pc._row_writer[lo:hi])) & set(fused)
            flagged_rows = set()
            for gp, f in flags.items():
                assert gp not in fused
                layer = groups[gp][0]
                brows = layer._host_desc()["bk_row"].numpy()
                for b, on in zip(brows.tolist(), f.cpu().numpy().tolist()):
                    inside = any(lo <= b and b + layer.block_size <= hi for lo, hi in ranges)
                    assert bool(on) == inside
                    if on:
                        flagged_rows.update(range(b, b + layer.block_size))
            want = set()
            for lo, hi in ranges:
                want.update(range(lo, hi))
            assert flagged_rows == want
    finally:
        SumLayer.tc05_min_tiles = saved
