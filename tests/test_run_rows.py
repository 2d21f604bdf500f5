"""Host-side tile planning for the tcgen05 contractions: run detection for the TMA-staged
kernel (a tile table qualifies for boxes of r rows when every tile's terms come in runs of r
consecutive source rows; the last run of a tile may be shorter), and the partial-row plan of
the one-launch long-tile contraction."""

import numpy as np

from helpers import build_fixture_circuit
from conftest import load_fixture

from pyjuice_b200.layer.layers import SumLayer, _run_rows


def _tiles(segments):
    """Tile rows (out_row, n_rows, k_off, k_cnt, ...) for consecutive krow segments."""
    t, off = [], 0
    for n in segments:
        t.append((0, 128, off, n, 0, 0, 0, 0))
        off += n
    return np.asarray(t, np.int64)


def test_runs_of_32_and_8():
    k32 = np.concatenate([np.arange(64, 96), np.arange(0, 32), np.arange(320, 340)])  # last run partial
    assert _run_rows(_tiles([84]), k32) == 32
    k8 = np.concatenate([np.arange(16, 24), np.arange(800, 808), np.arange(40, 45)])
    assert _run_rows(_tiles([21]), k8) == 8
    broken = np.concatenate([np.arange(0, 7), [100]])
    assert _run_rows(_tiles([8]), broken) == 0
    # runs are counted from each tile's first term (a tile shorter than a run is one run)
    two = np.concatenate([np.arange(0, 8), np.arange(50, 58)])
    assert _run_rows(_tiles([8, 8]), two) == 32
    assert _run_rows(_tiles([16]), two) == 8


def test_hclt64_layers_have_block_runs():
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx)
    for g in pc.inner_layer_groups:
        if not g.is_sum():
            continue
        for layer in g.layers:
            d = layer._host_desc()
            if layer.block_size >= 8 and d["fw_tiles"].size(0) >= SumLayer.tc05_min_tiles:
                assert d["fw_run"] in (8, 32)


def test_chunk_plan_remaps_rows_into_partials():
    """The plan of the one-launch long-tile contraction: chunk j of a tile writes its rows at
    j * S + (the rows' index among the S output rows); every output row has as many chunks as
    its tile (at most 128 terms each), all of them written. CPU only."""
    import torch
    from pyjuice_b200.layer.layers import _chunk_plan, _chunk_table
    tiles = np.array([[0, 128, 0, 300, 0, 0, 32, 0], [128, 64, 300, 129, 0, 128, 32, 0],
                      [300, 5, 429, 40, 0, 300, 32, 0]], np.int64)
    tab, ranges = _chunk_table(tiles)
    plan = _chunk_plan(torch.from_numpy(tab).int(), ranges)
    S = plan["S"]
    assert S == 128 + 64 + 5 and plan["nchunks"] == 3
    dst = plan["dst"].numpy()
    assert np.array_equal(dst, np.concatenate([np.arange(0, 192), np.arange(300, 305)]))
    nch = plan["nch"].numpy()
    assert np.array_equal(nch, np.concatenate([np.full(128, 3), np.full(64, 2), np.full(5, 1)]))
    t = plan["table"].numpy()
    written = set()
    for j, (a, n) in enumerate(ranges):
        for row in t[a:a + n]:
            for r in range(int(row[0]), int(row[0]) + int(row[1])):
                assert r // S == j
                written.add(r)
    expect = {j * S + r for r in range(S) for j in range(int(nch[r]))}
    assert written == expect
