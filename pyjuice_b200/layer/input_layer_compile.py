"""Input-layer compilation (reference: src/pyjuice/layer/input_layer.py:33-255, 968-996).

Produces the reference's per-node tables: ``vids [n, 1]``, ``s_pids``, ``s_pfids``,
``metadata`` / ``s_mids``, ``nids`` (index among the nodes of the same variable),
``source_nids``, ``node_id2source_id`` and the tied-flow table ``tied2source_nids``.
"""

from __future__ import annotations

from copy import deepcopy
from typing import Sequence

import torch


def reorder_input_nodes(nodes):
    """Untied vectors first (in order), tied ones after, pulling a tied vector's source forward."""
    node_set = set(nodes)
    untied, tied, added = [], [], set()
    for ns in nodes:
        if ns in added:
            continue
        if not ns.is_tied():
            untied.append(ns)
            added.add(ns)
        else:
            src = ns.get_source_ns()
            if src in added:
                tied.append(ns)
                added.add(ns)
            elif src in node_set:
                untied.append(src)
                tied.append(ns)
                added.add(ns)
                added.add(src)
            else:
                raise ValueError("A tied `InputNodes` should be in the same layer with its source nodes.")
    out = untied + tied
    if len(out) != len(nodes):
        raise RuntimeError("Total node length should not change after reordering.")
    return out


def compile_input_layer(nodes: Sequence, cum_nodes: int, max_tied_ns_per_parflow_block: int):
    nodes = reorder_input_nodes(list(nodes))
    signature = nodes[0].dist.get_signature()
    layer_num_nodes = 0
    cum_params = 0
    cum_param_flows = 0
    cum_source = 0
    node2tied = dict()
    node_vars, metadata_per_ns = [], []
    start = cum_nodes
    for ns in nodes:
        if ns.dist.get_signature() != signature:
            raise ValueError("Nodes of an InputLayer must have the same distribution type.")
        node_vars.append(ns.scope.to_list())
        metadata_per_ns.append(ns.dist.get_metadata())
        ns._output_ind_range = (cum_nodes, cum_nodes + ns.num_nodes)
        cum_nodes += ns.num_nodes
        layer_num_nodes += ns.num_nodes
        npar = ns.num_nodes * ns.dist.num_parameters()
        npf = ns.num_nodes * ns.dist.num_param_flows()
        if not ns.is_tied():
            ns._param_range = (cum_params, cum_params + npar)
            cum_params += npar
            ns._param_flow_range = (cum_param_flows, cum_param_flows + npf)
            cum_param_flows += npf
            cum_source += ns.num_nodes
        else:
            src = ns.get_source_ns()
            ns._param_range = deepcopy(src._param_range)
            if src not in node2tied:
                node2tied[src] = [[src], 1, src._param_flow_range]
            if node2tied[src][1] >= max_tied_ns_per_parflow_block:
                ns._param_flow_range = (cum_param_flows, cum_param_flows + npf)
                cum_param_flows += npf
                node2tied[src][2] = ns._param_flow_range
                node2tied[src][0].append(ns)
                node2tied[src][1] = 1
            else:
                ns._param_flow_range = deepcopy(node2tied[src][2])
                node2tied[src][1] += 1

    nvars = len(node_vars[0])
    vids = torch.empty([layer_num_nodes, nvars], dtype=torch.long)
    s_pids = torch.empty([layer_num_nodes], dtype=torch.long)
    s_pfids = torch.empty([layer_num_nodes], dtype=torch.long)
    s_mids = torch.empty([layer_num_nodes], dtype=torch.long)
    nids = torch.empty([layer_num_nodes], dtype=torch.long)
    source_nids = torch.empty([cum_source], dtype=torch.long)
    node_id2source_id = torch.empty([layer_num_nodes], dtype=torch.long)
    metadata = []
    n0 = 0
    src0 = 0
    var2count = dict()
    ns2range = dict()
    for i, ns in enumerate(nodes):
        n1 = n0 + ns.num_nodes
        ns2range[ns] = (n0, n1)
        if len(node_vars[i]) != nvars:
            raise ValueError("all input nodes of a layer need the same number of variables")
        vids[n0:n1, :] = torch.tensor(node_vars[i]).view(1, -1)
        k = ns.dist.num_parameters()
        s_pids[n0:n1] = ns._param_range[0] + torch.arange(0, ns.num_nodes * k, k) if k > 0 else 0
        kf = ns.dist.num_param_flows()
        s_pfids[n0:n1] = ns._param_flow_range[0] + torch.arange(0, ns.num_nodes * kf, kf) if kf > 0 else 0
        if not ns.is_tied():
            source_nids[src0:src0 + ns.num_nodes] = torch.arange(n0, n1)
            src0 += ns.num_nodes
            node_id2source_id[n0:n1] = -1
        else:
            t0, t1 = ns2range[ns.get_source_ns()]
            node_id2source_id[n0:n1] = torch.arange(t0, t1)
        s_mids[n0:n1] = len(metadata)
        metadata.extend(metadata_per_ns[i])
        if nvars == 1:
            v = node_vars[i][0]
            c = var2count.get(v, 0)
            nids[n0:n1] = torch.arange(0, n1 - n0) + c
            var2count[v] = c + n1 - n0
        n0 = n1

    tied2source = []
    for src, item in node2tied.items():
        if len(item[0]) > 1:
            npf = src._param_flow_range[1] - src._param_flow_range[0]
            ch = torch.tensor([c._param_flow_range[0] for c in item[0]], dtype=torch.long)
            tied2source.append([src._param_flow_range[0], npf, ch])

    return dict(nodes=nodes, nid_range=(start, start + layer_num_nodes), num_nodes=layer_num_nodes,
                num_parameters=cum_params, num_param_flows=cum_param_flows, signature=signature,
                vids=vids, s_pids=s_pids, s_pfids=s_pfids, metadata=torch.tensor(metadata).float(),
                s_mids=s_mids, nids=nids, source_nids=source_nids, node_id2source_id=node_id2source_id,
                tied2source_nids=tied2source, num_vars_per_node=nvars)
