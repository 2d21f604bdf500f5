"""Conditional probabilities P(x_v = k | evidence) of every (or every target) variable, given
hard evidence ``[B, num_vars]`` (int64, with an optional missing mask) or soft evidence
``[B, num_vars, num_cats]`` (FP32) (src/pyjuice/queries/conditional.py:497-547).

The forward pass evaluates the evidence (``InputLayer.forward`` / ``forward_soft``); the
backward pass computes node flows, and each Categorical input layer turns its nodes' flows
into per-category weights ``sum_n flow[n, b] theta[n, k]`` (``pcb_input_cat_evidence_bwd``),
normalised over k with + 1e-12, as the reference's ``_categorical_backward`` does.

``target_vars`` selects rows of that result. (The reference's own ``target_vars`` path
evaluates a partial set of input nodes and, on a circuit with tied input nodes, returns
values that differ from the same rows of its full result; the rows here are the full
result's.)
"""

from __future__ import annotations

from functools import partial
from typing import Callable, Optional, Sequence, Union

import torch

from .base import query


def _conditional_fw_input_fn(layer, inputs, node_mars, missing_mask=None, **kwargs):
    if layer.dist_signature != "Categorical":
        raise TypeError(f"Unknown/unsupported layer type {layer.dist_signature} for the forward pass. "
                        "Please implement and provide your own `fw_input_fn`.")
    if inputs.dim() == 2:
        if inputs.dtype != torch.long:
            raise ValueError("hard evidence must be int64 [B, num_vars]")
        layer.forward(inputs.permute(1, 0).contiguous(), node_mars, missing_mask=missing_mask)
    elif inputs.dim() == 3:
        if inputs.dtype != torch.float32:
            raise ValueError("soft evidence must be float32 [B, num_vars, num_cats]")
        layer.forward_soft(inputs, node_mars, missing_mask=missing_mask)
    else:
        raise NotImplementedError("Unknown method to compute the forward pass for `Categorical`.")


def _conditional_bk_input_fn(layer, inputs, node_flows, node_mars, outputs=None, target_vars=None, **kwargs):
    if layer.dist_signature != "Categorical":
        raise TypeError(f"Unknown/unsupported layer type {layer.dist_signature} for the backward pass. "
                        "Please implement and provide your own `bk_input_fn`.")
    probs = layer.evidence_backward(node_flows, None, target_vars=target_vars, mode=0)
    probs /= probs.sum(dim=2, keepdim=True) + 1e-12
    outputs.append(probs)


def conditional(pc, data: torch.Tensor, missing_mask: Optional[torch.Tensor] = None,
                target_vars: Optional[Sequence[int]] = None, fw_input_fn: Optional[Union[str, Callable]] = None,
                bk_input_fn: Optional[Union[str, Callable]] = None, **kwargs) -> torch.Tensor:
    """``[B, num_target_vars, num_cats]`` conditional category probabilities."""
    outputs = []
    kwargs["target_vars"] = target_vars
    data = data.to(pc.device)
    query(pc, inputs=data, run_backward=True,
          fw_input_fn=_conditional_fw_input_fn if fw_input_fn is None else fw_input_fn,
          bk_input_fn=partial(_conditional_bk_input_fn, outputs=outputs) if bk_input_fn is None else bk_input_fn,
          missing_mask=missing_mask, **kwargs)
    return outputs[0] if outputs else None
