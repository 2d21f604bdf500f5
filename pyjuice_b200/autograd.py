"""Differentiable log-likelihood of soft evidence: a ``torch.autograd.Function`` whose
backward pass is the circuit's own flow computation on the device.

``circuit_ll(pc, sum_logits, evidence)`` returns ``lls [B, 1]`` of a circuit whose sum
weights are ``softmax(sum_logits)`` over each node's children, evaluated on soft evidence
``E [B, num_vars, num_cats]`` (input node values ``min(log sum_k E theta, 0)``). Its
backward pass, for upstream gradients ``g [B, 1]``:

* runs the circuit's backward pass with root weights ``g`` (node flows and parameter flows;
  signs are handled by running with ``|g|`` when all weights share a sign, and with the
  signed-flow kernels otherwise);
* d/d sum_logits = ``pf - theta * sum_children pf`` per node (``pcb_sum_logit_grad``);
* d/dE[b, v, k] = ``sum_{n in v} flow[n, b] theta[n, k] / exp(node_mars[n, b])``
  (``pcb_input_cat_evidence_bwd`` mode 1).

The reference offers no such adjoint (its parameters carry no autograd and its
``_categorical_backward`` returns normalised category weights, queries/conditional.py:241-336);
the test suite checks these gradients against FP64 central differences of the oracle.
The backward pass reads the node values of the forward pass, so the circuit must not run
another forward pass between the two.
"""

from __future__ import annotations

from typing import Optional

import torch


def _soft_fw(layer, inputs, node_mars, missing_mask=None, **kwargs):
    layer.forward_soft(inputs, node_mars, missing_mask=missing_mask)


class _CircuitLL(torch.autograd.Function):

    @staticmethod
    def forward(ctx, pc, sum_logits, evidence, missing_mask, force_use_fp32):
        with torch.no_grad():
            pc.set_params_from_logits(sum_logits.detach())
            lls = pc.forward(evidence.detach(), input_layer_fn=_soft_fw, missing_mask=missing_mask,
                             force_use_fp32=force_use_fp32)
        ctx.pc = pc
        ctx.force_use_fp32 = force_use_fp32
        ctx.missing_mask = missing_mask
        ctx.save_for_backward(evidence)
        return lls.detach()

    @staticmethod
    def backward(ctx, grad):
        pc = ctx.pc
        (evidence,) = ctx.saved_tensors
        w = grad.detach().permute(1, 0).contiguous().float()
        sign = 1.0
        mixed = bool((w < 0).any()) and bool((w > 0).any())
        if not mixed and bool((w < 0).any()):
            w, sign = -w, -1.0
        ev_grad = []

        def bk(layer, inputs, node_flows, node_mars, **kw):
            ev_grad.append(layer.evidence_backward(node_flows, node_mars, None, mode=1))

        pc.init_param_flows(flows_memory=0.0)
        pc.backward(evidence, ll_weights=w, compute_param_flows=True, flows_memory=0.0, input_layer_fn=bk,
                    allow_modify_flows=not mixed, allow_neg_flows=mixed, force_use_fp32=ctx.force_use_fp32,
                    missing_mask=ctx.missing_mask)
        g_logits = pc.sum_logit_grad(scale=sign) if ctx.needs_input_grad[1] else None
        g_ev = None
        if ctx.needs_input_grad[2]:
            g_ev = ev_grad[0] * sign
            if g_ev.size(2) != evidence.size(2):
                g_ev = torch.nn.functional.pad(g_ev, (0, evidence.size(2) - g_ev.size(2)))
            if ctx.missing_mask is not None:  # summed-out variables do not depend on the evidence
                m = ctx.missing_mask.to(g_ev.device, torch.bool)
                g_ev = g_ev.masked_fill(m[None, :, None] if m.dim() == 1 else m[:, :, None], 0.0)
        return None, g_logits, g_ev, None, None


def circuit_ll(pc, sum_logits: torch.Tensor, evidence: torch.Tensor, missing_mask: Optional[torch.Tensor] = None,
               force_use_fp32: bool = True) -> torch.Tensor:
    """Log-likelihoods ``[B, 1]`` of soft evidence, differentiable with respect to
    ``sum_logits`` (shaped like ``pc.params``) and ``evidence`` ``[B, num_vars, num_cats]``."""
    return _CircuitLL.apply(pc, sum_logits, evidence, missing_mask, force_use_fp32)
