"""Hidden Markov models as circuits (src/pyjuice/structures/hmm.py:15-86).

For a sequence x_0 .. x_{T-1}: the emission vector of the last step is an input vector over
variable T - 1; walking back from t = T - 2 to 0, the state at step t is a product of the
emission vector of x_t (a duplicate of the first, tied when ``homogeneous``) and a sum over
the previous state vector (the transition, likewise tied), and the root sums the last
product into one node (the initial distribution). ``alpha`` [L, L] (transition), ``beta``
[L, num_emits] (emission) and ``gamma`` [L] (initial) optionally set the parameters.
``var_offset`` shifts the sequence's variables (x_t is variable ``var_offset + t``).

``batched_hmms`` puts several HMMs over disjoint variable ranges into one circuit: a
product of their roots under a one-node sum, so that one compiled circuit evaluates all of
them (its log-likelihood is the sum of theirs, and flows and EM updates stay per HMM). The
layers of every HMM at the same depth then run in the same launches. The reference has no
such builder; it serves batched workloads of uneven HMMs.
"""

from __future__ import annotations

from typing import Callable, Optional

import torch

from ..nodes import inputs, multiply, set_block_size, summate
from ..nodes.distributions import Categorical
from .hclt import _max_cdf_power_of_2


def HMM(seq_length: int, num_latents: int, num_emits: int, homogeneous: bool = True, block_size: Optional[int] = None,
        alpha: Optional[torch.Tensor] = None, beta: Optional[torch.Tensor] = None,
        gamma: Optional[torch.Tensor] = None, sum_edge_ids_constructor: Optional[Callable] = None,
        var_offset: int = 0):
    if seq_length < 2:
        raise ValueError("an HMM needs at least two steps")
    if block_size is None:
        block_size = min(_max_cdf_power_of_2(num_latents), 1024)
    num_node_blocks = num_latents // block_size
    with set_block_size(block_size=block_size):
        emit = inputs(var_offset + seq_length - 1, num_node_blocks=num_node_blocks, dist=Categorical(num_cats=num_emits))
        if beta is not None:
            if tuple(beta.shape) != (num_latents, num_emits):
                raise ValueError("beta must be [num_latents, num_emits]")
            emit.set_params(beta)
        trans = None
        state = emit
        for var in range(seq_length - 2, -1, -1):
            xs = emit.duplicate(var_offset + var, tie_params=homogeneous)
            if trans is None:
                ns = summate(state, num_node_blocks=num_node_blocks, sum_edge_ids_constructor=sum_edge_ids_constructor)
                if alpha is not None:
                    if tuple(alpha.shape) != (num_latents, num_latents):
                        raise ValueError("alpha must be [num_latents, num_latents]")
                    ns.set_params(alpha)
                trans = ns
            else:
                ns = trans.duplicate(state, tie_params=homogeneous)
            state = multiply(xs, ns)
        root = summate(state, num_node_blocks=1, block_size=1, sum_edge_ids_constructor=sum_edge_ids_constructor)
        if gamma is not None:
            if gamma.dim() != 1 or gamma.size(0) != num_latents:
                raise ValueError("gamma must be [num_latents]")
            root.set_params(gamma.unsqueeze(0))
    return root


def batched_hmms(specs, num_emits: int, homogeneous: bool = True, params=None, block_size: Optional[int] = None):
    """One circuit of several HMMs: ``specs`` lists ``(seq_length, num_latents)`` per HMM,
    HMM i covering the variables after those of HMMs 0 .. i-1. ``params`` optionally lists
    ``(alpha, beta, gamma)`` per HMM (see ``HMM``). All HMMs share one block size (default:
    the largest power of two dividing every hidden size, at most 32), because the compiled
    layout keeps the reference's rule of dropping child ids below a layer's first element id
    as dummies, which holds only when the first node id is at least every block size.
    Returns the root: a one-node sum over the product of the HMMs' roots;
    ``offsets[i]`` (attribute of the root) is HMM i's first variable."""
    if block_size is None:
        block_size = 32
        while any(L % block_size for _, L in specs):
            block_size //= 2
    roots, offsets, off = [], [], 0
    for i, (T, L) in enumerate(specs):
        a, b, g = params[i] if params is not None else (None, None, None)
        roots.append(HMM(T, L, num_emits, homogeneous=homogeneous, alpha=a, beta=b, gamma=g, var_offset=off,
                         block_size=block_size))
        offsets.append(off)
        off += T
    with set_block_size(block_size=1):
        prod = multiply(*roots)
        root = summate(prod, num_node_blocks=1, block_size=1)
    root.set_params(torch.ones([1, 1, 1]))
    root.offsets = offsets
    return root
