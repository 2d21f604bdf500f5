"""Data-parallel EM across processes (one GPU per process).

Each rank runs forward and backward on its own shard of the batch with identical
parameters; parameter flows are additive over samples, so summing them across ranks
before ``mini_batch_em`` gives every rank the update of the union batch, and the
parameters stay identical everywhere. This is the only exchange of the path: one
all-reduce of the sum-parameter flows and one of the input-parameter flows per step
(NCCL over NVLink between GPUs; any torch.distributed backend works).
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def allreduce_param_flows(pc, group=None) -> None:
    """Sum ``pc.param_flows`` and every input layer's ``param_flows`` across ``group``."""
    if not dist.is_available() or not dist.is_initialized():
        return
    if pc.param_flows is not None:
        dist.all_reduce(pc.param_flows, op=dist.ReduceOp.SUM, group=group)
    for layer in pc.input_layer_group:
        if layer.param_flows is not None:
            dist.all_reduce(layer.param_flows, op=dist.ReduceOp.SUM, group=group)


def broadcast_parameters(pc, src: int = 0, group=None) -> None:
    """Make every rank's parameters equal to rank ``src``'s (e.g. after random initialisation)."""
    if not dist.is_available() or not dist.is_initialized():
        return
    with torch.no_grad():
        dist.broadcast(pc.params.data, src=src, group=group)
        for layer in pc.input_layer_group:
            dist.broadcast(layer.params.data, src=src, group=group)
