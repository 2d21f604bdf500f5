"""Top-down probabilities: the probability that a top-down (ancestral) walk from the root
reaches each node, and the parameter flows of that walk (src/pyjuice/model/backend/top_down_prob.py:290-402).

They are the node flows of one evidence-free pass: every variable summed out, root flow 1.
Here that pass runs on the circuit's own kernels over private single-sample buffers: a
forward pass with all variables missing (input values log 1; node values log Z_n, which is
0 for a normalised circuit, so the same pass also covers unnormalised ones, where the
reference multiplies each weight by exp(Z_child - Z_node)), then a backward pass from
root weight 1 (node flows = top-down probabilities) and, if parameter flows are wanted,
from root weight ``scale`` with the parameter flows accumulated (sum weights
``scale * theta * tdp``; input categories ``scale * tdp * theta_k``, as the reference's
``add_missing_flows``). The circuit's batch buffers and its running flow total are left as
they were.
"""

from __future__ import annotations

import contextlib

import torch

_BUFFERS = ("node_mars", "element_mars", "_em_resident", "node_flows", "element_flows")


@contextlib.contextmanager
def _private_buffers(pc, key: str):
    saved = {n: pc.__dict__.get(n) for n in _BUFFERS}
    store = pc.__dict__.setdefault("_private_buffer_sets", {}).setdefault(key, {})
    for n in _BUFFERS:
        pc.__dict__[n] = store.get(n)
    cum = pc._cum_flow_dev
    try:
        yield
    finally:
        for n in _BUFFERS:
            store[n] = pc.__dict__.get(n)
            pc.__dict__[n] = saved[n]
        pc._cum_flow_dev = cum


def eval_top_down_probs(pc, update_pflow: bool = True, scale: float = 1.0, pc_is_normalized: bool = True,
                        use_cudagraph: bool = True):
    """Top-down probability of every node into ``pc._single_node_flows`` ``[num_nodes]``; with
    ``update_pflow`` adds ``scale`` times the walk's parameter flows to the parameter flows.
    ``pc_is_normalized`` is accepted for the reference's signature; the pass is exact either
    way."""
    dev = pc.device
    x = torch.zeros([1, pc.num_vars], dtype=torch.long, device=dev)
    miss = torch.ones([pc.num_vars], dtype=torch.bool, device=dev)
    with _private_buffers(pc, "top_down"), torch.no_grad():
        pc.forward(x, missing_mask=miss, force_use_fp32=True)
        pc.backward(inputs=x, compute_param_flows=False, allow_modify_flows=False, force_use_fp32=True,
                    missing_mask=miss, input_layer_fn=lambda *a, **k: None)
        pc._single_node_flows = pc.node_flows[:, 0].clone()
        if update_pflow:
            if pc.param_flows is None:
                pc.init_param_flows(flows_memory=0.0)
            w = torch.full([1, 1], float(scale), dtype=torch.float32, device=dev)
            pc.backward(inputs=x, ll_weights=w, compute_param_flows=True, flows_memory=1.0, allow_modify_flows=False,
                        force_use_fp32=True, missing_mask=miss)
    return None
