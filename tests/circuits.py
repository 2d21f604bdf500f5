"""Circuit recipes shared by the fixture generator and the tests.

Each recipe only uses the construction API that the reference and ``pyjuice_b200``
have in common (``inputs`` / ``multiply`` / ``summate`` / ``set_block_size`` /
``duplicate``), so the same call builds the same DAG in both packages.
"""

from __future__ import annotations

import torch


def build_tiny_dag(juice, dists):
    """A small DAG exercising the compiler's corner cases.

    * sum vectors with different child counts in one layer (several partitions);
    * a block-sparse sum (explicit ``edge_ids``) and a sparse product (explicit ``edge_ids``);
    * a sum whose children sit at different depths (pass-through insertion);
    * tied sum vectors and tied input vectors;
    * a block-size-1 root.
    """
    with juice.set_block_size(4):
        i = [juice.inputs(v, num_node_blocks=2, dist=dists.Categorical(num_cats=4)) for v in range(5)]
        i.append(i[4].duplicate(5, tie_params=True))
        p01 = juice.multiply(i[0], i[1])
        p01b = juice.multiply(i[0], i[1], edge_ids=torch.tensor([[1, 0], [0, 1]]))
        p23 = juice.multiply(i[2], i[3])
        p45 = juice.multiply(i[4], i[5])
        s01 = juice.summate(p01, p01b, num_node_blocks=3)
        s23 = juice.summate(p23, edge_ids=torch.tensor([[0, 0, 1], [0, 1, 1]]))
        s23t = s23.duplicate(tie_params=True)
        s45 = juice.summate(p45, num_node_blocks=2)
        q = juice.multiply(s01, s23, edge_ids=torch.tensor([[0, 0], [1, 1], [2, 0]]))
        q2 = juice.multiply(s01, s23t, edge_ids=torch.tensor([[2, 1], [0, 0], [1, 0]]))
        p0123 = juice.multiply(i[0], i[1], i[2], i[3])
        r = juice.summate(q, q2, p0123, num_node_blocks=2)
        top = juice.multiply(r, s45)
        root = juice.summate(top, num_node_blocks=1, block_size=1)
    return root


def build_shared_child_dag(juice, dists):
    """Inputs and sums that are children of product vectors in different product layers
    (a sum over two decompositions of the same scope), so that the backward pass writes some
    node flows from two layers: the first writer overwrites, the second accumulates."""
    with juice.set_block_size(4):
        i = [juice.inputs(v, num_node_blocks=2, dist=dists.Categorical(num_cats=4)) for v in range(4)]
        s01 = juice.summate(juice.multiply(i[0], i[1]), num_node_blocks=2)
        s23 = juice.summate(juice.multiply(i[2], i[3]), num_node_blocks=2)
        s012 = juice.summate(juice.multiply(s01, i[2]), num_node_blocks=2)
        a = juice.multiply(s012, i[3])
        b = juice.multiply(s01, s23)
        root = juice.summate(a, b, num_node_blocks=1, block_size=1)
    return root


def seeded_params(em_pbase, em_nch, em_bs, num_sum_params, in_num_nodes, in_ncats, seed: int):
    """Normalised random parameters for a compiled layout, regenerable from a seed.

    Sum weights: each node's weights over its children sum to one (the node-block slab
    ``base + k * bs + i`` of the compiled layout); input nodes: each row of ``in_ncats``
    probabilities sums to one. Used instead of storing large parameter vectors in fixtures.
    """
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros(num_sum_params, dtype=np.float64)
    for base, k, bs in zip(em_pbase, em_nch, em_bs):
        slab = np.exp(-4.0 * rng.random((int(k), int(bs))))
        p[int(base):int(base) + int(k) * int(bs)] = (slab / slab.sum(axis=0, keepdims=True)).reshape(-1)
    q = np.exp(-4.0 * rng.random((in_num_nodes, in_ncats)))
    q /= q.sum(axis=1, keepdims=True)
    return p.astype(np.float32), q.reshape(-1).astype(np.float32)


def build_layer_test_nodes(juice, dists, block_size: int = 16):
    """The node vectors of the reference's sum-layer unit test (tests/layer/sum_layer_test.py:17-48)."""
    with juice.set_block_size(block_size):
        ni = [juice.inputs(v, num_node_blocks=2, dist=dists.Categorical(num_cats=2)) for v in range(4)]
        np0 = juice.multiply(ni[0], ni[1])
        np1 = juice.multiply(ni[2], ni[3])
        np2 = juice.multiply(ni[1], ni[2])
        ns0 = juice.summate(np0, num_node_blocks=2)
        ns1 = juice.summate(np1, num_node_blocks=2)
        ns2 = juice.summate(np2, num_node_blocks=2)
    return ni, [np0, np1, np2], [ns0, ns1, ns2]


def build_dist_dag(juice, dist_factory):
    """Four variables with input vectors of one distribution (``dist_factory()`` per vector),
    two sums over pairs and a block-size-1 root: exercises a non-Categorical input layer."""
    with juice.set_block_size(4):
        i = [juice.inputs(v, num_node_blocks=2, dist=dist_factory()) for v in range(4)]
        s01 = juice.summate(juice.multiply(i[0], i[1]), num_node_blocks=2)
        s23 = juice.summate(juice.multiply(i[2], i[3]), num_node_blocks=2)
        root = juice.summate(juice.multiply(s01, s23), num_node_blocks=1, block_size=1)
    return root
