"""Host-side run detection for the TMA-staged tcgen05 contraction: a tile table qualifies
for boxes of r rows when every tile's terms come in runs of r consecutive source rows
(the last run of a tile may be shorter)."""

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
