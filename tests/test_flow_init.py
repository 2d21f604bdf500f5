"""The backward pass initialises only the node-flow rows that no product layer overwrites.

CPU: the plan (overwriting vs accumulating product layers, initialised rows) is checked by
replaying the product layers' writes. GPU: on a circuit whose inputs and sums are children
of product vectors in two different product layers, node and parameter flows match the
oracle (which zeroes every row first)."""

import numpy as np
import pytest
import torch

from circuits import build_shared_child_dag, seeded_params
from oracle import pc_oracle as orc

import pyjuice_b200 as juice
from pyjuice_b200.nodes import distributions as dists


def _targets(layer):
    rows = layer._host_desc()["bk_row"].numpy().astype(np.int64)
    return (rows[:, None] + np.arange(layer.block_size)[None, :]).reshape(-1)


def _check_plan(pc):
    state = np.zeros([pc.num_nodes], dtype=bool)  # row holds a defined value
    for a, b in pc._nf_init_ranges:
        state[a:b] = True
    r0, r1 = pc._root_node_range
    state[r0:r1] = True
    for group in reversed(pc.inner_layer_groups):
        if not group.is_prod():
            continue
        for layer in group:
            tgt = _targets(layer)
            if layer.bk_accumulate:
                assert state[tgt].all(), "a layer accumulates into rows nothing initialised"
            state[tgt] = True
    assert state.all()


def test_plan_shared_children():
    pc = juice.compile(build_shared_child_dag(juice, dists))
    acc = [l.bk_accumulate for g in pc.inner_layer_groups if g.is_prod() for l in g]
    assert any(acc) and not all(acc)
    _check_plan(pc)


def test_plan_hclt_overwrites_only():
    from helpers import build_fixture_circuit
    from conftest import load_fixture
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx)
    assert not any(l.bk_accumulate for g in pc.inner_layer_groups if g.is_prod() for l in g)
    assert pc._nf_init_ranges == [(0, pc.num_dummy_nodes)]
    _check_plan(pc)


@pytest.mark.gpu
def test_shared_children_flows_vs_oracle(cuda_device):
    pc = juice.compile(build_shared_child_dag(juice, dists)).to(cuda_device)
    il = pc.input_layer_group[0]
    p, q = seeded_params(pc._em_pbase.tolist(), pc._em_nch.tolist(), pc._em_bs.tolist(), pc.num_sum_params,
                         il.num_nodes, 4, seed=7)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(p).to(cuda_device))
        il.params.copy_(torch.from_numpy(q).to(cuda_device))
    rng = np.random.default_rng(3)
    x = rng.integers(0, 4, size=(37, 4))
    lay = orc.layout_from_circuit(pc)
    nm, ems, _ = orc.forward(lay, p, q, x)
    nf_o, pf_o, ipf_o = orc.backward(lay, p, x, nm, ems)
    xd = torch.from_numpy(x).to(cuda_device)
    for _ in range(2):  # the second pass starts from the first pass's buffers
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            pc(xd, force_use_fp32=True)
        pc.backward(inputs=xd, allow_modify_flows=False, force_use_fp32=True)
        nf = pc.node_flows.double().cpu().numpy()
        real = slice(pc.num_dummy_nodes, pc.num_nodes)
        assert np.abs(nf[real] - nf_o[real]).max() <= 1e-5 * np.abs(nf_o[real]).max()
        pf = pc.param_flows.double().cpu().numpy()
        assert np.abs(pf - pf_o).max() <= 1e-4 * np.abs(pf_o).max()


def test_parentless_elements_are_zeroed_each_pass():
    """A PD structure with max_prod_block_conns = 1 leaves product nodes that no sum block
    selects. The element rows are one buffer reused by every product group, so per product
    group the plan zeroes exactly the rows of its elements that have no parent in the sum
    group above (they would otherwise hold another group's element flows)."""
    import numpy as np
    import torch
    import pyjuice_b200 as juice
    torch.manual_seed(7)
    pc = juice.compile(juice.structures.PD((4, 4), 16, split_intervals=1, max_prod_block_conns=1,
                                           input_dist=juice.distributions.Categorical(num_cats=4)))
    groups = pc.inner_layer_groups
    found = 0
    for gi, group in enumerate(groups):
        if not group.is_prod() or gi + 1 >= len(groups):
            continue
        produced, children = set(), set()
        for layer in group:
            for nids in layer.partitioned_nids:
                for n in nids.tolist():
                    produced.update(range(n, n + layer.block_size))
        for layer in groups[gi + 1]:
            for cids in layer.partitioned_cids:
                children.update(int(c) for c in cids.reshape(-1).tolist() if c != 0)
        orphans = produced - children
        planned = set()
        for a, b in pc._ef_init_ranges.get(gi, ()):
            planned.update(range(a, b))
        assert planned == orphans, gi
        found += len(orphans)
    assert found > 0
