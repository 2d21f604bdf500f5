"""The query driver shared by ``marginal`` and ``conditional`` (src/pyjuice/queries/base.py:9-27):
a forward pass with a custom input-layer function, then optionally a backward pass
without parameter flows whose input-layer function collects per-category results."""

from __future__ import annotations

from typing import Callable, Optional, Union

import torch


def query(pc, inputs: torch.Tensor, run_backward: bool = True, fw_input_fn: Optional[Union[str, Callable]] = None,
          bk_input_fn: Optional[Union[str, Callable]] = None, fw_output_fn: Optional[Callable] = None, **kwargs):
    with torch.no_grad():
        lls = pc.forward(inputs, input_layer_fn=fw_input_fn, **kwargs)
    if fw_output_fn is not None:
        return fw_output_fn(pc)
    if not run_backward:
        return lls
    if bk_input_fn is None:
        raise ValueError("a backward query needs `bk_input_fn`")
    pc.backward(inputs, input_layer_fn=bk_input_fn, compute_param_flows=False, **kwargs)
    return None
