"""Layer compilation: circuit node vectors -> partitioned index tensors.

These functions produce exactly the index tensors the reference compiler produces
(src/pyjuice/layer/compilation.py), so that ``partitioned_*`` tensors, parameter
offsets and node / element numbering are interchangeable with the reference's. The
index arithmetic is restated with vectorised numpy per node vector instead of the
reference's per-edge Triton/numba kernels.

Sum layer, forward tables (compilation.py:262-595), for node block ``g`` of a layer:
  ``nids[p][l]``      first node id of the block,
  ``cids[p][l, k]``   element id of its k-th child node (edge order, zero padded),
  ``pids[p][l, k]``   parameter id of (child k, node 0); node i of the block uses ``+ i``,
  ``pfids[p][l, k]``  the same for parameter flows.
Sum layer, backward tables (compilation.py:697-901), for child block ``c``:
  ``chids[p][l]``       first element id of the child block,
  ``parids[p][l, q]``   first node id of its q-th parent block,
  ``parpids[p][l, q]``  first parameter id of the [ch_block_size, block_size] edge block.
Product layer (compilation.py:878-1185):
  ``nids[p][l]`` first element id, ``cids[p][l, j]`` first node id of child j,
  ``u_cids[p][l]`` child node ids with a parent, ``parids[p][l, q]`` their parents.
"""

from __future__ import annotations

from copy import deepcopy
from typing import Dict, List, Sequence

import numpy as np
import torch

from .partition import next_power_of_2, partition_nodes_by_n_edges


def _group_offsets(keys: np.ndarray, num_keys: int) -> np.ndarray:
    """For each position i, how many earlier positions share ``keys[i]`` (a running count)."""
    order = np.argsort(keys, kind="stable")
    sorted_keys = keys[order]
    counts = np.bincount(keys, minlength=num_keys)
    starts = np.zeros(num_keys, dtype=np.int64)
    starts[1:] = np.cumsum(counts)[:-1]
    ranks_sorted = np.arange(keys.shape[0], dtype=np.int64) - starts[sorted_keys]
    out = np.empty_like(ranks_sorted)
    out[order] = ranks_sorted
    return out


def _assign_partitions(counts: torch.Tensor, max_chs: torch.Tensor, min_start: int):
    """Partition id / index-in-partition / partition sizes for blocks with child counts ``counts``."""
    num = counts.size(0)
    part_ids = torch.zeros([num], dtype=torch.long)
    local_ids = torch.zeros([num], dtype=torch.long)
    sizes = torch.zeros([max_chs.size(0)], dtype=torch.long)
    lo = min_start
    for p, hi in enumerate(max_chs.tolist()):
        crit = (counts >= lo) & (counts <= hi)
        size = int(crit.sum().item())
        part_ids[crit] = p
        local_ids[crit] = torch.arange(size)
        sizes[p] = size
        lo = hi + 1
    return part_ids, local_ids, sizes


def _partition_max(counts: torch.Tensor, layer_sparsity_tol, max_num_partitions) -> torch.Tensor:
    m = partition_nodes_by_n_edges(counts, sparsity_tolerance=layer_sparsity_tol, max_num_partitions=max_num_partitions)
    return torch.unique(next_power_of_2(m))


def compile_sum_layer(nodes: Sequence, global_nid_start: int, global_pid_start: int, global_pfid_start: int,
                      node2tiednodes: dict, layer_sparsity_tol, max_num_partitions, max_tied_ns_per_parflow_block: int):
    """Compile one sum layer. Returns a dict of tensors and ranges (see module docstring)."""
    block_size = nodes[0].block_size
    layer_nid_start, layer_pid_start, layer_pfid_start = global_nid_start, global_pid_start, global_pfid_start

    # ---- forward statistics (compilation.py:107-128) ----
    layer_num_nblocks = sum(ns.num_node_blocks for ns in nodes)
    n_chs = torch.zeros([layer_num_nblocks], dtype=torch.long)
    nid = global_nid_start
    s = 0
    num_edges = 0
    for ns in nodes:
        cnt = torch.bincount(ns.edge_ids[0, :], minlength=ns.num_node_blocks) * ns.ch_block_size
        n_chs[s:s + ns.num_node_blocks] = cnt
        ns._output_ind_range = (nid, nid + ns.num_nodes)
        nid += ns.num_nodes
        num_edges += ns.num_edges
        s += ns.num_node_blocks
    num_nodes = layer_num_nblocks * block_size

    fw_max = _partition_max(n_chs, layer_sparsity_tol, max_num_partitions)
    fw_part, fw_local, fw_sizes = _assign_partitions(n_chs, fw_max, 1)
    fw_part_np, fw_local_np = fw_part.numpy(), fw_local.numpy()

    nparts = fw_max.size(0)
    nids = [np.zeros([int(fw_sizes[p])], dtype=np.int64) for p in range(nparts)]
    cids = [np.zeros([int(fw_sizes[p]), int(fw_max[p])], dtype=np.int64) for p in range(nparts)]
    pids = [np.zeros([int(fw_sizes[p]), int(fw_max[p])], dtype=np.int64) for p in range(nparts)]
    pfids = [np.zeros([int(fw_sizes[p]), int(fw_max[p])], dtype=np.int64) for p in range(nparts)]

    all_param_ids: Dict[int, np.ndarray] = {}
    all_param_flow_ids: Dict[int, np.ndarray] = {}
    original_param_nids = []
    node2tiedcounts = dict()

    nblock_start = 0
    for ns_idx, ns in enumerate(nodes):
        # ---- parameter / parameter-flow ranges, tying (compilation.py:369-447) ----
        if not ns.is_tied():
            if not ns.provided("_param_range"):
                ns._param_range = (global_pid_start, global_pid_start + ns.num_edges)
                global_pid_start += ns.num_edges
                ns._param_flow_range = (global_pfid_start, global_pfid_start + ns.num_edges)
                global_pfid_start += ns.num_edges
                add_params, add_pflows = True, True
            else:
                add_params, add_pflows = False, False
            original_param_nids.append(ns_idx)
            ns_pid_start = ns._param_range[0]
            ns_pfid_start = ns._param_flow_range[0]
        else:
            source_ns = ns.get_source_ns()
            if not source_ns.provided("_param_range"):
                ns._param_range = (global_pid_start, global_pid_start + ns.num_edges)
                ns._param_flow_range = (global_pfid_start, global_pfid_start + ns.num_edges)
                source_ns._param_range = ns._param_range
                source_ns._param_flow_range = ns._param_flow_range
                global_pid_start += ns.num_edges
                global_pfid_start += ns.num_edges
                add_params, add_pflows = True, True
            else:
                ns._param_range = deepcopy(source_ns._param_range)
                add_params, add_pflows = False, False
            if source_ns not in node2tiednodes:
                node2tiednodes[source_ns] = [[source_ns], [source_ns._param_flow_range]]
                node2tiedcounts[source_ns] = [1]
            elif source_ns not in node2tiedcounts:
                node2tiedcounts[source_ns] = [0 for _ in range(len(node2tiednodes[source_ns][0]))]
            if not ns.provided("_param_flow_range"):
                counts = node2tiedcounts[source_ns]
                if all(c >= max_tied_ns_per_parflow_block for c in counts):
                    ns._param_flow_range = (global_pfid_start, global_pfid_start + ns.num_edges)
                    global_pfid_start += ns.num_edges
                    node2tiednodes[source_ns][1].append(ns._param_flow_range)
                    node2tiednodes[source_ns][0].append(ns)
                    counts.append(1)
                    add_pflows = True
                else:
                    target = min(range(len(counts)), key=lambda i: counts[i])
                    ns._param_flow_range = deepcopy(node2tiednodes[source_ns][1][target])
                    counts[target] += 1
                    add_pflows = False
            ns_pid_start = source_ns._param_range[0]
            ns_pfid_start = ns._param_flow_range[0]

        # ---- flattened edges: one per (node block, child node) ----
        cbs = ns.ch_block_size
        e = ns.edge_ids.numpy()
        e0 = np.repeat(e[0], cbs)
        e1 = (e[1][:, None] * cbs + np.arange(cbs)[None, :]).reshape(-1)
        chs_off = _group_offsets(e0, ns.num_node_blocks)
        ns_nchs = np.bincount(e0, minlength=ns.num_node_blocks)
        cum_n_chs = np.zeros(ns.num_node_blocks, dtype=np.int64)
        cum_n_chs[1:] = np.cumsum(ns_nchs)[:-1]

        cs_cum = np.zeros(ns.num_chs, dtype=np.int64)
        cs_start = np.zeros(ns.num_chs, dtype=np.int64)
        acc = 0
        for i, cs in enumerate(ns.chs):
            cs_cum[i] = acc
            cs_start[i] = cs._output_ind_range[0]
            acc += cs.num_nodes
        which_cs = np.searchsorted(cs_cum, e1, side="right") - 1
        global_cid = cs_start[which_cs] + e1 - cs_cum[which_cs]

        gblock = nblock_start + e0
        part = fw_part_np[gblock]
        local = fw_local_np[gblock]
        global_nid = global_nid_start + gblock * block_size
        global_pid = ns_pid_start + (cum_n_chs[e0] + chs_off) * block_size
        global_pfid = ns_pfid_start + (cum_n_chs[e0] + chs_off) * block_size
        for p in np.unique(part):
            m = part == p
            nids[p][local[m]] = global_nid[m]
            cids[p][local[m], chs_off[m]] = global_cid[m]
            pids[p][local[m], chs_off[m]] = global_pid[m]
            pfids[p][local[m], chs_off[m]] = global_pfid[m]
        if add_params:
            all_param_ids[ns_idx] = global_pid
        if add_pflows:
            all_param_flow_ids[ns_idx] = global_pfid
        nblock_start += ns.num_node_blocks

    for ns_idx, pids_e in all_param_ids.items():
        ns = nodes[ns_idx]
        if ns.is_tied():
            ns = ns.get_source_ns()
        ns._param_ids = torch.from_numpy(pids_e[0::ns.ch_block_size].copy())
    for ns_idx, pfids_e in all_param_flow_ids.items():
        ns = nodes[ns_idx]
        ns._param_flow_ids = torch.from_numpy(pfids_e[0::ns.ch_block_size].copy())
    for ns_idx in original_param_nids:
        ns = nodes[ns_idx]
        ns._inverse_param_ids = torch.argsort(ns._param_ids)

    out = dict(
        num_nodes=num_nodes, num_edges=num_edges, block_size=block_size,
        nid_range=(layer_nid_start, layer_nid_start + num_nodes),
        pid_range=(layer_pid_start, global_pid_start), pfid_range=(layer_pfid_start, global_pfid_start),
        nids=[torch.from_numpy(x) for x in nids], cids=[torch.from_numpy(x) for x in cids],
        pids=[torch.from_numpy(x) for x in pids], pfids=[torch.from_numpy(x) for x in pfids],
    )

    # ---- backward statistics (compilation.py:131-173) ----
    gsize2cs: Dict[int, List] = {}
    gsize2nblocks: Dict[int, int] = {}
    cs2parns: Dict = {}
    for ns in nodes:
        for cs in ns.chs:
            g = cs.block_size
            if g not in gsize2cs:
                gsize2cs[g] = []
                gsize2nblocks[g] = 0
            if not any(c is cs for c in gsize2cs[g]):
                gsize2cs[g].append(cs)
                gsize2nblocks[g] += cs.num_node_blocks
            if cs not in cs2parns:
                cs2parns[cs] = []
            if not any(n is ns for n in cs2parns[cs]):
                cs2parns[cs].append(ns)

    ns2cum_n_chs = {}
    ns2chs_off = {}

    def _ns_tables(ns):
        if ns not in ns2cum_n_chs:
            e0 = ns.edge_ids[0].numpy()
            ns2chs_off[ns] = _group_offsets(e0, ns.num_node_blocks)
            nch = np.bincount(e0, minlength=ns.num_node_blocks)
            c = np.zeros(ns.num_node_blocks, dtype=np.int64)
            c[1:] = np.cumsum(nch)[:-1]
            ns2cum_n_chs[ns] = c
        return ns2cum_n_chs[ns], ns2chs_off[ns]

    chids_all, parids_all, parpids_all, cs_block_sizes = [], [], [], []
    for g, cs_list in gsize2cs.items():
        # number of parent edge blocks per child node block
        n_pargs = []
        per_cs_edges = []
        for cs in cs_list:
            cnt = np.zeros(cs.num_node_blocks, dtype=np.int64)
            edges = []
            for ns in cs2parns[cs]:
                cs_id = next(i for i, c in enumerate(ns.chs) if c is cs)
                esid = sum(c.num_node_blocks for c in ns.chs[:cs_id])
                eeid = esid + cs.num_node_blocks
                e = ns.edge_ids.numpy()
                crit = (e[1] >= esid) & (e[1] < eeid)
                cnt += np.bincount(e[1][crit] - esid, minlength=cs.num_node_blocks)
                edges.append((ns, e[0][crit], e[1][crit] - esid, crit))
            n_pargs.append(cnt)
            per_cs_edges.append(edges)
        n_pargs = torch.from_numpy(np.concatenate(n_pargs))

        bk_max = _partition_max(n_pargs, layer_sparsity_tol, max_num_partitions)
        bk_part, bk_local, bk_sizes = _assign_partitions(n_pargs, bk_max, 1)
        bk_part_np, bk_local_np = bk_part.numpy(), bk_local.numpy()
        nbp = bk_max.size(0)
        chids = [np.zeros([int(bk_sizes[p])], dtype=np.int64) for p in range(nbp)]
        parids = [np.zeros([int(bk_sizes[p]), int(bk_max[p])], dtype=np.int64) for p in range(nbp)]
        parpids = [np.zeros([int(bk_sizes[p]), int(bk_max[p])], dtype=np.int64) for p in range(nbp)]

        cs_nblock_start = 0
        for cs, edges in zip(cs_list, per_cs_edges):
            cid_all = np.concatenate([x[2] for x in edges]) if edges else np.zeros([0], dtype=np.int64)
            pars_off_all = _group_offsets(cid_all, cs.num_node_blocks)
            pos = 0
            for ns, nid_e, cid_e, crit in edges:
                n_e = nid_e.shape[0]
                pars_off = pars_off_all[pos:pos + n_e]
                pos += n_e
                ns_pid_start = ns.get_source_ns()._param_range[0] if ns.is_tied() else ns._param_range[0]
                cum_n_chs, chs_off_full = _ns_tables(ns)
                chs_off = chs_off_full[crit]
                gb = cs_nblock_start + cid_e
                part = bk_part_np[gb]
                local = bk_local_np[gb]
                gchid = cs._output_ind_range[0] + cid_e * cs.block_size
                gparid = ns._output_ind_range[0] + nid_e * ns.block_size
                gpid = ns_pid_start + (cum_n_chs[nid_e] + chs_off) * ns.block_size * cs.block_size
                for p in np.unique(part):
                    m = part == p
                    chids[p][local[m]] = gchid[m]
                    parids[p][local[m], pars_off[m]] = gparid[m]
                    parpids[p][local[m], pars_off[m]] = gpid[m]
            cs_nblock_start += cs.num_node_blocks

        chids_all.extend(torch.from_numpy(x) for x in chids)
        parids_all.extend(torch.from_numpy(x) for x in parids)
        parpids_all.extend(torch.from_numpy(x) for x in parpids)
        cs_block_sizes.extend([g] * nbp)

    out.update(chids=chids_all, parids=parids_all, parpids=parpids_all, cs_block_sizes=cs_block_sizes)
    return out


def compile_prod_layer(nodes: Sequence, global_nid_start: int, layer_sparsity_tol, max_num_partitions):
    """Compile one product layer (prod_layer.py:30-158 with compilation.py:878-1185)."""
    use_block_sparse = all(ns.is_block_sparse() and ns.block_size == nodes[0].block_size for ns in nodes)
    block_size = nodes[0].block_size if use_block_sparse else 1

    if use_block_sparse:
        nblock = sum(ns.num_node_blocks for ns in nodes)
    else:
        nblock = sum(ns.num_nodes for ns in nodes)
    n_chgs = torch.zeros([nblock], dtype=torch.long)
    s = 0
    nid = global_nid_start
    num_edges = 0
    for ns in nodes:
        k = ns.num_node_blocks if use_block_sparse else ns.num_nodes
        n_chgs[s:s + k] = ns.num_chs
        num_edges += ns.num_nodes * ns.num_chs
        ns._output_ind_range = (nid, nid + ns.num_nodes)
        nid += ns.num_nodes
        s += k
    num_nodes = nblock * block_size

    fw_max = _partition_max(n_chgs, layer_sparsity_tol, max_num_partitions)
    nparts = fw_max.size(0)
    part_of_ns, local_of_ns = [], []
    sizes = [0] * nparts
    for ns in nodes:
        p = int((ns.num_chs > fw_max).sum().item())
        part_of_ns.append(p)
        local_of_ns.append(sizes[p])
        sizes[p] += ns.num_node_blocks if use_block_sparse else ns.num_nodes

    nids = [torch.zeros([sizes[p]], dtype=torch.long) for p in range(nparts)]
    cids = [torch.zeros([sizes[p], int(fw_max[p])], dtype=torch.long) for p in range(nparts)]
    for ns, p, ls in zip(nodes, part_of_ns, local_of_ns):
        n_sid = ns._output_ind_range[0]
        if use_block_sparse:
            le = ls + ns.num_node_blocks
            nids[p][ls:le] = torch.arange(0, ns.num_nodes, block_size) + n_sid
            for j, cs in enumerate(ns.chs):
                cids[p][ls:le, j] = ns.edge_ids[:, j] * block_size + cs._output_ind_range[0]
        else:
            le = ls + ns.num_nodes
            nids[p][ls:le] = torch.arange(0, ns.num_nodes) + n_sid
            if ns.is_sparse():
                for j, cs in enumerate(ns.chs):
                    cids[p][ls:le, j] = ns.edge_ids[:, j] + cs._output_ind_range[0]
            else:
                e = (ns.edge_ids[:, None, :].repeat(1, ns.block_size, 1) * ns.block_size
                     + torch.arange(0, ns.block_size)[None, :, None]).flatten(0, 1)
                for j, cs in enumerate(ns.chs):
                    cids[p][ls:le, j] = e[:, j] + cs._output_ind_range[0]

    # ---- backward: parents of every used child block (compilation.py:975-1185) ----
    flat_cids = torch.cat([c.reshape(-1) for c in cids])
    flat_cid2nid = torch.cat([n.unsqueeze(1).repeat(1, c.size(1)).reshape(-1) for n, c in zip(nids, cids)])
    u_cids, par_counts = torch.unique(flat_cids, sorted=True, return_counts=True)
    below = torch.arange(0, u_cids.size(0))[u_cids < global_nid_start]
    if below.numel() > 0:
        cut = int(below.max().item()) + 1
        u_cids = u_cids[cut:]
        par_counts = par_counts[cut:]

    bk_max = _partition_max(par_counts, layer_sparsity_tol, max_num_partitions)
    bk_part, bk_local, bk_sizes = _assign_partitions(par_counts, bk_max, 0)
    nbp = bk_max.size(0)
    out_u = [torch.zeros([int(bk_sizes[p])], dtype=torch.long) for p in range(nbp)]
    out_par = [torch.zeros([int(bk_sizes[p]), int(bk_max[p])], dtype=torch.long) for p in range(nbp)]

    fc = flat_cids.numpy()
    fn = flat_cid2nid.numpy()
    order = np.argsort(fc, kind="stable")
    sfc, sfn = fc[order], fn[order]
    starts = np.searchsorted(sfc, u_cids.numpy(), side="left")
    ends = np.searchsorted(sfc, u_cids.numpy(), side="right")
    bp, bl = bk_part.numpy(), bk_local.numpy()
    for i in range(u_cids.size(0)):
        p, l = bp[i], bl[i]
        out_u[p][l] = u_cids[i]
        pars = sfn[starts[i]:ends[i]]
        out_par[p][l, :pars.shape[0]] = torch.from_numpy(pars)

    return dict(num_nodes=num_nodes, num_edges=num_edges, block_size=block_size, use_block_sparse=use_block_sparse,
                nid_range=(global_nid_start, global_nid_start + num_nodes),
                nids=nids, cids=cids, u_cids=out_u, parids=out_par)
