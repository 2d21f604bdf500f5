"""The compiler reproduces the reference's compiled layout exactly (CPU only)."""

import numpy as np
import pytest
import torch

from conftest import load_fixture
from helpers import build_fixture_circuit, layout_mismatches, tree_from_fixture

from pyjuice_b200.structures import chow_liu_tree


@pytest.mark.parametrize("name", ["tiny", "hclt64"])
def test_layout_matches_reference(name):
    fx = load_fixture(name)
    torch.manual_seed(0)
    pc = build_fixture_circuit(name, fx)
    assert layout_mismatches(pc, fx, full=True) == []
    il = pc.input_layer_group[0]
    for n in ("vids", "s_pids", "s_pfids", "s_mids", "nids", "source_nids", "node_id2source_id"):
        assert np.array_equal(fx["in_" + n], getattr(il, n).numpy()), n
    assert tuple(fx["root_range"]) == tuple(pc._root_node_range)


def test_layout_matches_reference_hclt784():
    fx = load_fixture("hclt784")
    pc = build_fixture_circuit("hclt784", fx)
    assert layout_mismatches(pc, fx, full=False) == []
    assert pc.num_nodes == int(fx["num_nodes"])


@pytest.mark.parametrize("name", ["hclt64", "hclt784"])
def test_chow_liu_tree_matches_reference(name):
    fx = load_fixture(name)
    tree = chow_liu_tree(fx["tree_mi"].astype(np.float64))
    root = tree.center()
    seq, children, root_ref = tree_from_fixture(fx)
    assert root == root_ref
    assert tree.dfs_postorder(root) == seq
    ch = tree.bfs_children(root)
    assert all(ch[v] == children[v] for v in range(len(seq)))


def test_layer_test_structure_indices():
    """Exact index assertions of the reference's sum-layer unit test (tests/layer/sum_layer_test.py:49-79)."""
    import pyjuice_b200 as juice
    from pyjuice_b200.nodes import distributions as dists
    from circuits import build_layer_test_nodes

    bs = 16
    ni, nps, nss = build_layer_test_nodes(juice, dists, bs)
    juice.InputLayer(ni, cum_nodes=bs)
    juice.ProdLayer(nps)
    layer = juice.SumLayer(nss, global_nid_start=bs, global_pid_start=bs ** 2, global_pfid_start=0, node2tiednodes=dict())
    nids, cids, pids, pfids = (layer.partitioned_nids[0], layer.partitioned_cids[0], layer.partitioned_pids[0],
                               layer.partitioned_pfids[0])
    assert torch.all(nids == torch.arange(bs, 7 * bs, bs))
    assert torch.all(cids[0:2, 0] == bs) and torch.all(cids[2:4, 0] == 3 * bs) and torch.all(cids[4:6, 0] == 5 * bs)
    assert torch.all(cids[0:2, 1] == bs + 1) and torch.all(cids[2:4, 1] == 3 * bs + 1)
    base = torch.arange(bs, (bs * 2 * 6 + 1) * bs, 2 * bs * bs)
    assert torch.all(pids[:, 0] == base - bs + bs ** 2)
    assert torch.all(pids[:, 1] == base + bs ** 2)
    assert torch.all(pfids[:, 0] == base - bs)
    assert torch.all(pfids[:, 1] == base)
    chids, parids, parpids = layer.partitioned_chids[0], layer.partitioned_parids[0], layer.partitioned_parpids[0]
    assert torch.all(chids == torch.arange(bs, 7 * bs, bs))
    assert torch.all(parids[0:2, 0] == bs) and torch.all(parids[0:2, 1] == 2 * bs)
    assert torch.all(parids[2:4, 0] == 3 * bs) and torch.all(parids[2:4, 1] == 4 * bs)
    assert torch.all(parids[4:6, 0] == 5 * bs) and torch.all(parids[4:6, 1] == 6 * bs)
    expect = [[1, 3], [2, 4], [5, 7], [6, 8], [9, 11], [10, 12]]
    for r in range(6):
        for q in range(2):
            assert int(parpids[r, q]) == expect[r][q] * bs ** 2
