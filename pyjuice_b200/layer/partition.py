"""Partitioning of node blocks by their number of children.

A layer's node blocks are split into a few partitions; every block of a partition is
padded to the partition's (power-of-2) child count. The split is chosen by the
reference's "dp_with_coalesce" algorithm
(src/pyjuice/layer/backend/node_partition.py:87-226), restated here with numpy:

1. sort the child counts and drop zeros;
2. coalesce: unique counts are grouped while within ``floor((max-min)/1000)`` of the
   group's first value; each group is represented by its last (largest) value and the
   summed multiplicity;
3. weighted DP over the coalesced values: ``dp[i, 1] = v[i] * C[i]`` (``C`` = cumulative
   multiplicities) and ``dp[i, n] = min_j dp[j, n-1] + v[i] * (C[i] - C[j])`` with the
   first minimal ``j`` kept and candidates capped at ``2**31 - 1`` as in the reference;
   the first ``n`` whose cost is within ``ceil(sum * (1 + tol))`` is taken;
4. backtrace. The reference reads the backtrace column of the final partition count at
   every step (node_partition.py:43-47); the same is done here so that the partitions,
   and with them every compiled index tensor, are identical.
"""

from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch

_CAP = 2 ** 31 - 1


def _coalesce(vals: np.ndarray):
    unique_vals, counts = np.unique(vals, return_counts=True)
    tol_range = int(math.floor((unique_vals.max() - unique_vals.min()) / 1000))
    keep_vals, keep_counts = [], []
    start_val, acc = None, 0
    for i in range(unique_vals.shape[0]):
        if start_val is None:
            start_val, acc = unique_vals[i], counts[i]
        elif unique_vals[i] - start_val <= tol_range:
            acc += counts[i]
        else:
            keep_vals.append(unique_vals[i - 1])
            keep_counts.append(acc)
            start_val, acc = unique_vals[i], counts[i]
    if start_val is not None:
        keep_vals.append(unique_vals[-1])
        keep_counts.append(acc)
    return np.array(keep_vals, dtype=np.int64), np.array(keep_counts, dtype=np.int64)


def _weighted_dp(vals: np.ndarray, counts: np.ndarray, max_num_partitions: int, target_overhead: int):
    n = vals.shape[0]
    cum = np.cumsum(counts).astype(np.int64)
    v = vals.astype(np.int64)
    dp = np.zeros([n, max_num_partitions + 1], dtype=np.int64)
    bt = np.zeros([n, max_num_partitions + 1], dtype=np.int64)
    dp[:, 1] = v * cum
    if dp[n - 1, 1] <= target_overhead:
        return 1, bt
    target_n = max_num_partitions
    for npart in range(2, max_num_partitions + 1):
        dp[0, npart] = v[0] * cum[0]
        bt[0, npart] = 0
        for i in range(1, n):
            cands = dp[:i, npart - 1] + v[i] * (cum[i] - cum[:i])
            # first strictly-smaller candidate scanning from the cap == first argmin below the cap
            m = cands.min()
            if m < _CAP:
                dp[i, npart] = m
                bt[i, npart] = int(np.argmax(cands == m))
            else:
                dp[i, npart] = _CAP
                bt[i, npart] = -1
        if dp[n - 1, npart] <= target_overhead:
            target_n = npart
            break
    return target_n, bt


def partition_nodes_by_n_edges(node_n_edges, max_num_partitions: Optional[int] = None,
                               sparsity_tolerance: Optional[float] = None) -> torch.Tensor:
    """Return the sorted maximum child count of each partition (before power-of-2 rounding)."""
    if sparsity_tolerance is not None and sparsity_tolerance < 1e-6:
        sparsity_tolerance = None
        max_num_partitions = 1
    if isinstance(node_n_edges, torch.Tensor):
        node_n_edges = node_n_edges.detach().cpu().numpy()
    node_n_edges = np.asarray(node_n_edges, dtype=np.int64)

    if sparsity_tolerance is not None:
        if not (1e-6 < sparsity_tolerance <= 1.0):
            raise ValueError("sparsity tolerance must be in (1e-6, 1]")
        if max_num_partitions is None:
            max_num_partitions = max(min(np.unique(node_n_edges).shape[0], 16), 1)
    elif max_num_partitions is None:
        max_num_partitions = 1
    elif max_num_partitions < 1:
        raise ValueError("Should provide at least 1 partition.")

    target_overhead = 0 if sparsity_tolerance is None else int(math.ceil(node_n_edges.sum() * (1.0 + sparsity_tolerance)))

    if max_num_partitions == 1:
        return torch.tensor([int(node_n_edges.max())], dtype=torch.long)

    vals = np.sort(node_n_edges)
    vals = vals[vals != 0]
    uvals, counts = _coalesce(vals)
    target_n, bt = _weighted_dp(uvals, counts, max_num_partitions, target_overhead)

    parts = np.zeros([target_n], dtype=np.int64)
    i = uvals.shape[0] - 1
    for npart in range(target_n, 0, -1):
        parts[npart - 1] = i
        i = bt[i, target_n]
    sizes = np.unique(uvals[parts])
    return torch.sort(torch.from_numpy(sizes)).values


def next_power_of_2(x: torch.Tensor) -> torch.Tensor:
    """Elementwise next power of two, computed in float32 like the reference (compilation.py:94-99)."""
    return torch.where(x == 1, 1, 2 ** torch.ceil(torch.log2(x.float())).long())
