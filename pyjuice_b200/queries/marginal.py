"""Marginal log-likelihoods log P(e) of partial assignments: the variables set in
``missing_mask`` ([num_vars] or [B, num_vars]) are summed out, which a smooth and
decomposable circuit does exactly by giving their input nodes the value log 1
(src/pyjuice/queries/marginal.py:16-37)."""

from __future__ import annotations

from typing import Callable, Optional, Union

import torch

from .base import query
from .conditional import _conditional_fw_input_fn


def marginal(pc, data: torch.Tensor, missing_mask: Optional[torch.Tensor] = None,
             fw_input_fn: Optional[Union[str, Callable]] = None, **kwargs) -> torch.Tensor:
    """``[B, num_root_nodes]`` log-likelihoods of ``data`` with the masked variables summed out."""
    return query(pc, inputs=data.to(pc.device), run_backward=False,
                 fw_input_fn=_conditional_fw_input_fn if fw_input_fn is None else fw_input_fn,
                 missing_mask=missing_mask, **kwargs)
