"""``TensorCircuit``: a compiled circuit whose passes run on the sm_100a kernels.

Drop-in for the reference's ``TensorCircuit`` (src/pyjuice/model/tensorcircuit.py:94-1261):
same constructor arguments, buffers (``node_mars``, ``element_mars``, ``node_flows``,
``element_flows``, ``params``, ``param_flows``), layer groups, ``forward`` /
``backward`` / ``mini_batch_em`` semantics, the autograd hook that turns
``lls.mean().backward()`` into a circuit backward pass, and the accessors
(``get_node_mars``, ``get_node_flows``, ``update_parameters``, ...).

Differences that are deliberate:
* buffers are only initialised where a kernel reads them before writing (dummy rows;
  ``node_flows`` which is accumulated), instead of full re-initialisation each pass;
* the running total of root flows (``_cum_flow``) is kept on the device, so
  ``backward`` does not synchronise with the host;
* EM and normalisation accumulate in FP64 per node block (``pcb_sum_em``), without
  atomics.
"""

from __future__ import annotations

import hashlib
from functools import partial
from typing import Callable, Optional, Sequence, Union

import numpy as np
import torch
import torch.nn as nn

from .. import _native as nat
from ..layer.layers import InputLayer, LayerGroup, ProdLayer, SumLayer, _ch_pack, _mma, _num_sms
from ..nodes import CircuitNodes, multiply, summate


def _pc_model_backward_hook(grad, pc, inputs, record_cudagraph, apply_cudagraph, propagation_alg, **kwargs):
    """Gradient hook on the returned log-likelihoods (tensorcircuit.py:24-37).

    The weights are normalised to sum to the batch size, so ``lls.mean()`` and
    ``lls.sum()`` produce the same flows, as in the reference.
    """
    grad = grad.permute(1, 0)
    pc.backward(inputs=inputs, ll_weights=grad / grad.sum() * grad.size(1),
                compute_param_flows=pc._optim_hyperparams["compute_param_flows"],
                flows_memory=pc._optim_hyperparams["flows_memory"], record_cudagraph=record_cudagraph,
                apply_cudagraph=apply_cudagraph, propagation_alg=propagation_alg, **kwargs)
    return None


# One PcbShortLevel record (include/pcb200.h): two pointers and eight int32 fields.
_SHORT_LEVEL = np.dtype([("packed", "<u8"), ("element_out", "<u8"), ("tile0", "<i4"), ("num_tiles", "<i4"),
                         ("rpb_log2", "<i4"), ("w_stride", "<i4"), ("row_splits", "<i4"), ("need", "<i4"),
                         ("wvec", "<i4"), ("item0", "<i4")])

# One PcbPackJob record (include/pcb200.h): three pointers and four int32 fields.
_PACK_JOB = np.dtype([("tiles", "<u8"), ("kw", "<u8"), ("packed", "<u8"), ("num_tiles", "<i4"),
                      ("rpb_log2", "<i4"), ("w_stride", "<i4"), ("format", "<i4")])


class TensorCircuit(nn.Module):
    # Side streams that the backward pass spreads the parameter-flow launches over.
    pflow_streams = 4
    # Fuse product layers into the single-stage kernels of the sum layers next to them
    # (where _plan_product_fusion shows that the result is the same): in the backward pass
    # (element flows written straight to the children's node flows) and, separately, in the
    # forward pass (terms staged as sums of child node rows). The forward fusion is off by
    # default: on HCLT-784 (B = 512) staging up to four child rows per term cost more than
    # the product launch it saves (forward 0.87 -> 0.93 ms), while the backward fusion saves
    # 0.07 ms.
    fuse_products = True
    fuse_products_forward = False
    # Let the product layer that alone writes a large sum layer's node flows write them as
    # log f - log m directly (the rewrite that layer's backward would otherwise launch).
    fuse_flow_rewrite = True

    def __init__(self, root_ns: CircuitNodes, layer_sparsity_tol: float = 0.5,
                 max_num_partitions: Optional[int] = None, disable_gpu_compilation: bool = False,
                 force_gpu_compilation: bool = False, max_tied_ns_per_parflow_block: int = 8,
                 device: Optional[Union[int, torch.device]] = None, verbose: bool = False) -> None:
        super().__init__()
        if not isinstance(root_ns, CircuitNodes):
            raise TypeError("`root_ns` should be an instance of `CircuitNodes`.")
        self.root_ns = root_ns
        self.device = torch.device("cpu")
        self.num_vars = max(root_ns.scope.to_list()) + 1
        self.node_mars = None
        self.element_mars = None
        self.node_flows = None
        self.element_flows = None
        self.param_flows = None
        self.param_flows_f64 = None
        self._init_layers(layer_sparsity_tol=layer_sparsity_tol, max_num_partitions=max_num_partitions,
                          max_tied_ns_per_parflow_block=max_tied_ns_per_parflow_block)
        self._optim_hyperparams = {"compute_param_flows": True, "flows_memory": 1.0}
        self._recorded_cuda_graphs = dict()
        self.default_propagation_alg = "LL"
        self.propagation_alg_kwargs = dict()
        self._run_params = dict()
        self._cum_flow_dev = None
        self._side_streams = dict()
        # False (default): every product layer group keeps its element values resident for
        # the backward pass. True: they share element_mars (as in the reference) and the
        # backward pass recomputes each group's element values from the kept node values
        # right before the sum group above it, saving the resident buffer
        # (num_elements of all groups x batch x 4 bytes).
        self.recompute_element_values = False
        self._level_runs = dict()
        self._dev_tables = {}
        self._pack_tables = {}
        self._param_epoch = 0      # bumped by every in-library write of the sum parameters
        self._fw_partial_eval_enabled = False
        self._bk_partial_eval_enabled = False
        self._partial_epoch = 0    # bumped whenever partial evaluation is switched
        self._el_pack_state = None  # parameters and pass settings the element-flow packs were made for
        if device is not None:
            self.to(device)

    # ------------------------------------------------------------------ compile
    def _create_node_layers(self):
        """Depth assignment with pass-through insertion (tensorcircuit.py:1122-1191)."""
        depth2nodes = dict()
        nodes2depth = dict()
        num_layers = 1
        max_node_bs = 0
        max_ele_bs = 0
        order = list(self.root_ns)  # post-order: children first
        for ns in order:
            if ns in nodes2depth:
                continue
            if ns.is_input():
                nodes2depth[ns] = 0
                depth2nodes.setdefault(0, {"input": []})["input"].append(ns)
                continue
            depth = max(nodes2depth[cs] for cs in ns.chs) + (1 if ns.is_prod() else 0)
            num_layers = max(depth + 1, num_layers)
            nodes2depth[ns] = depth
            if depth not in depth2nodes:
                depth2nodes[depth] = {"sum": [], "prod": []}
            if ns.is_sum():
                for idx, cs in enumerate(ns.chs):
                    cs_depth = nodes2depth[cs]
                    if cs_depth < depth:
                        pass_sum = summate(cs, num_node_blocks=cs.num_node_blocks, block_size=cs.block_size,
                                           edge_ids=torch.arange(0, cs.num_node_blocks)[None, :].repeat(2, 1),
                                           params=torch.eye(cs.block_size)[None, :, :].repeat(cs.num_node_blocks, 1, 1))
                        pass_prod = multiply(pass_sum)
                        ns.chs[idx] = pass_prod
                        depth2nodes[cs_depth]["sum"].append(pass_sum)
                        nodes2depth[pass_sum] = cs_depth
                        nodes2depth[pass_prod] = depth
                depth2nodes[depth]["sum"].append(ns)
                max_node_bs = max(max_node_bs, ns.block_size)
            else:
                max_ele_bs = max(max_ele_bs, ns.block_size)
        pns2layer = dict()
        for layer in range(1, len(depth2nodes)):
            for ns in depth2nodes[layer]["sum"]:
                for cs in ns.chs:
                    if cs.is_prod():
                        if id(cs) in pns2layer:
                            if pns2layer[id(cs)] != layer:
                                raise ValueError("a product node is requested by sum nodes at different layers")
                        else:
                            depth2nodes[layer]["prod"].append(cs)
                            pns2layer[id(cs)] = layer
        return depth2nodes, num_layers, max_node_bs, max_ele_bs

    def _init_layers(self, layer_sparsity_tol, max_num_partitions, max_tied_ns_per_parflow_block):
        """Layer construction and global numbering (tensorcircuit.py:920-1092)."""
        self.root_ns._clear_tensor_circuit_hooks()
        depth2nodes, num_layers, max_node_bs, max_ele_bs = self._create_node_layers()
        self.num_dummy_nodes = max_ele_bs
        self.num_dummy_eles = max_node_bs
        self.num_dummy_params = max_node_bs * max_ele_bs
        num_nodes = self.num_dummy_nodes
        num_edges = 0
        num_elements = self.num_dummy_eles
        num_parameters = self.num_dummy_params
        num_param_flows = 0
        node2tiednodes = dict()
        self.inner_layer_groups = []
        em_regions = []
        self.input_layer_group = None
        input_layers = []
        for depth in range(num_layers):
            if depth == 0:
                sig2nodes = dict()
                for ns in depth2nodes[0]["input"]:
                    sig2nodes.setdefault(ns.dist.get_signature(), []).append(ns)
                for sig, nodes in sig2nodes.items():
                    layer = InputLayer(nodes, cum_nodes=num_nodes, pc_num_vars=self.num_vars,
                                       max_tied_ns_per_parflow_block=max_tied_ns_per_parflow_block)
                    input_layers.append(layer)
                    num_nodes += layer.num_nodes
                self.input_layer_group = LayerGroup(input_layers)
                self.input_layers = nn.ModuleList(input_layers)
                continue
            if not depth2nodes[depth]["prod"] or not depth2nodes[depth]["sum"]:
                raise ValueError(f"depth {depth} has no product or no sum nodes")
            gsize2prod = dict()
            for ns in depth2nodes[depth]["prod"]:
                gsize2prod.setdefault(ns.block_size, []).append(ns)
            layer_num_elements = max_node_bs
            prod_layers = []
            for _, nodes in gsize2prod.items():
                pl = ProdLayer(nodes, global_nid_start=layer_num_elements, layer_sparsity_tol=layer_sparsity_tol,
                               max_num_partitions=max_num_partitions)
                layer_num_elements += pl.num_nodes
                num_edges += pl.num_edges
                prod_layers.append(pl)
            self.inner_layer_groups.append(LayerGroup(prod_layers))
            em_regions.append((len(self.inner_layer_groups) - 1, layer_num_elements))
            num_elements = max(num_elements, layer_num_elements)
            gsize2sum = dict()
            for ns in depth2nodes[depth]["sum"]:
                gsize2sum.setdefault(ns.block_size, []).append(ns)
            sum_layers = []
            for _, nodes in gsize2sum.items():
                sl = SumLayer(nodes, global_nid_start=num_nodes, global_pid_start=num_parameters,
                              global_pfid_start=num_param_flows, node2tiednodes=node2tiednodes,
                              layer_sparsity_tol=layer_sparsity_tol, max_num_partitions=max_num_partitions,
                              max_tied_ns_per_parflow_block=max_tied_ns_per_parflow_block)
                num_nodes += sl.num_nodes
                num_edges += sl.num_edges
                num_parameters += sl.num_parameters
                num_param_flows += sl.num_param_flows
                sum_layers.append(sl)
            self.inner_layer_groups.append(LayerGroup(sum_layers))

        self.num_nodes = num_nodes
        self.num_edges = num_edges
        self.num_elements = num_elements
        # Every product layer group keeps its element values in its own row region of one
        # resident buffer, so the backward pass reads them instead of recomputing them.
        self._em_region = dict()
        off = 0
        for gi, rows in em_regions:
            self._em_region[gi] = (off, rows)
            off += rows
        self._em_rows = off
        self.num_sum_params = num_parameters
        self.num_param_flows = num_param_flows
        self.num_root_nodes = self.root_ns.num_nodes
        self._root_node_range = (self.num_nodes - self.num_root_nodes, self.num_nodes)
        self._node2tiednodes = node2tiednodes
        # The source of a tied set shares its parameter-flow slots with up to
        # max_tied_ns_per_parflow_block - 1 tied vectors in other layers, whose parameter
        # flows may run at the same time on other streams: its layer adds with atomics too.
        sources = {id(ns.get_source_ns()) for group in self.inner_layer_groups if group.is_sum()
                   for layer in group for ns in layer.nodes if ns.is_tied()}
        for group in self.inner_layer_groups:
            if group.is_sum():
                for layer in group:
                    if any(id(ns) in sources for ns in layer.nodes):
                        layer._has_tied = True
        self._build_em_tables()
        self._plan_node_flow_init()
        self._plan_product_fusion()
        self._init_parameters()

    def _plan_product_fusion(self):
        """Product layers that a single-stage sum kernel can absorb (host tables, once).

        For product group ``gi`` with one layer, feeding sum group ``gi + 1`` with one layer,
        and elements of at most four children:
          * forward: the sum layer's terms are element rows of this group; the kernel can
            stage their children's node rows and add them (``fw``: per term, four node rows);
          * backward, when additionally the product layer overwrites its child rows (see
            _plan_node_flow_init), every child node has exactly one parent element, and the
            sum layer's element-flow tiles cover every element: the element-flow kernel can
            write each element's flow to its children's rows (``bw``: per element, four node
            rows). The product layer's own launch is then skipped.
        """
        self._fusion_host, self._fusion_dev = dict(), dict()
        groups = self.inner_layer_groups
        for gi in range(len(groups) - 1):
            if not (groups[gi].is_prod() and groups[gi + 1].is_sum()):
                continue
            if len(groups[gi]) != 1 or len(groups[gi + 1]) != 1:
                continue
            pl, sl = groups[gi][0], groups[gi + 1][0]
            pd, sd = pl._host_desc(), sl._host_desc()
            fr, fo = pd["fw_row"].numpy().astype(np.int64), pd["fw_off"].numpy().astype(np.int64)
            fc, fch = pd["fw_cnt"].numpy().astype(np.int64), pd["fw_chs"].numpy().astype(np.int64)
            if fr.size == 0 or fc.min() < 1 or fc.max() > 4:
                continue
            rows = self._em_region[gi][1]
            bs = pl.block_size
            ech = np.full([rows, 4], -1, np.int64)
            written = np.zeros([rows], dtype=bool)
            ar = np.arange(bs)
            for g in range(fr.size):
                written[fr[g]:fr[g] + bs] = True
                for j in range(int(fc[g])):
                    ech[fr[g]:fr[g] + bs, j] = fch[fo[g] + j] + ar
            krow = sd["krow"].numpy().astype(np.int64)
            if krow.size == 0 or krow.max() >= rows or not written[krow].all():
                continue
            fw = ech[krow].astype(np.int32).reshape(-1)
            bw = None
            if not pl.bk_accumulate and np.all(pd["bk_cnt"].numpy() == 1):
                covered = np.zeros([rows], dtype=bool)
                for eg in sd["el_groups"]:
                    for t in eg["tiles"].numpy():
                        covered[t[0]:t[0] + t[1]] = True
                if covered[written].all():
                    bw = ech.astype(np.int32).reshape(-1)
            self._fusion_host[gi] = dict(fw=fw, bw=bw)

    def _rewrite_plan(self, fused_prod=frozenset()):
        """Large sum layers whose node flows the product layers write already rewritten as
        log f - log m: every row written by exactly one overwriting single-layer product
        group that is not fused into an element-flow kernel in this pass (``fused_prod``).
        Returns ({product group: device flags per child block}, {rewritten sum groups});
        cached per device, large-layer threshold and fused set."""
        fused_prod = frozenset(fused_prod)
        key = (self.device.type, self.device.index, SumLayer.tc05_min_tiles, fused_prod)
        plan = self._rewrite_plans.get(key)
        if plan is not None:
            return plan
        groups = self.inner_layer_groups
        nw, wr = self._row_nwriters, self._row_writer
        ranges, done = [], set()
        for gs, group in enumerate(groups):
            if not group.is_sum() or len(group) != 1:
                continue
            layer = group[0]
            if layer._host_desc()["fw_tiles"].size(0) < SumLayer.tc05_min_tiles:
                continue
            lo, hi = layer._layer_nid_range
            if hi <= lo or not np.all(nw[lo:hi] == 1):
                continue
            gps = np.unique(wr[lo:hi])
            if np.any(gps < 0) or any(groups[int(g)][0].bk_accumulate or int(g) in fused_prod for g in gps):
                continue
            ranges.append((int(lo), int(hi)))
            done.add(gs)
        flags = dict()
        if ranges:
            for gp, group in enumerate(groups):
                if not group.is_prod() or len(group) != 1 or gp in fused_prod:
                    continue
                layer = group[0]
                rows = layer._host_desc()["bk_row"].numpy().astype(np.int64)
                inside = np.zeros(rows.shape[0], dtype=bool)
                for lo, hi in ranges:
                    inside |= (rows >= lo) & (rows + layer.block_size <= hi)
                if inside.any():
                    flags[gp] = torch.from_numpy(inside.astype(np.int32)).to(self.device)
        plan = (flags, done)
        self._rewrite_plans[key] = plan
        return plan

    def _fusion_tables(self, gi: int, kind: str):
        """Device table ``kind`` ("fw" or "bw") of product group ``gi`` (None if not fusable)."""
        h = self._fusion_host.get(gi)
        if h is None or h[kind] is None or not TensorCircuit.fuse_products:
            return None
        if kind == "fw" and not TensorCircuit.fuse_products_forward:
            return None
        key = (self.device.type, self.device.index, gi, kind)
        t = self._fusion_dev.get(key)
        if t is None:
            t = torch.from_numpy(h[kind]).to(self.device)
            self._fusion_dev[key] = t
        return t

    def _plan_node_flow_init(self):
        """Which node-flow rows the backward pass must initialise.

        Product layers write the flows of their child nodes. Visited in backward order, a
        layer none of whose target rows has been written yet overwrites them (no prior
        zeroing needed); a layer that meets rows written before accumulates into them. Only
        the rows that are accumulated into without an earlier writer, and the rows that no
        product layer writes (dummy rows), are initialised by ``backward`` (the root rows
        are set there explicitly). Results are the same as zeroing every row first.
        """
        written = np.zeros([self.num_nodes], dtype=bool)
        need = np.zeros([self.num_nodes], dtype=bool)
        nwriters = np.zeros([self.num_nodes], dtype=np.int64)
        writer = np.full([self.num_nodes], -1, dtype=np.int64)
        for gi in range(len(self.inner_layer_groups) - 1, -1, -1):
            group = self.inner_layer_groups[gi]
            if not group.is_prod():
                continue
            for layer in group:
                rows = layer._host_desc()["bk_row"].numpy().astype(np.int64)
                tgt = (rows[:, None] + np.arange(layer.block_size)[None, :]).reshape(-1)
                if written[tgt].any():
                    layer.bk_accumulate = True
                    need[tgt[~written[tgt]]] = True
                else:
                    layer.bk_accumulate = False
                written[tgt] = True
                nwriters[tgt] += 1
                writer[tgt] = gi if len(group) == 1 else -2
        # kept for _rewrite_plan: how many product layers write each row, and which group
        # (-2: a group of several layers)
        self._row_nwriters, self._row_writer = nwriters, writer
        self._rewrite_plans = dict()
        r0, r1 = self._root_node_range
        need |= ~written
        need[r0:r1] = False
        idx = np.flatnonzero(need)
        ranges = []
        if idx.size:
            cuts = np.flatnonzero(np.diff(idx) != 1)
            starts = np.concatenate([[idx[0]], idx[cuts + 1]])
            ends = np.concatenate([idx[cuts] + 1, [idx[-1] + 1]])
            ranges = [(int(a), int(b)) for a, b in zip(starts, ends)]
        self._nf_init_ranges = ranges
        self._ef_init_ranges = self._plan_element_flow_init()

    def _plan_element_flow_init(self):
        """Per product layer group: the element-flow rows it reads that the sum group right
        above it does not write.

        As in the reference, the element rows are one buffer that every product layer group
        reuses: the sum group above a product group writes the flows of that group's
        elements, which the product layers then read. An element without a parent sum node (a
        product that no sum block selected, as in PD structures with
        ``max_prod_block_conns``) is not written there, and its rows would still hold the
        flows of another group's elements; those rows are zeroed before the product group's
        backward pass (the reference zeroes the whole buffer, tensorcircuit.py:394-395)."""
        plan = dict()
        groups = self.inner_layer_groups
        for gi, group in enumerate(groups):
            if not group.is_prod() or gi + 1 >= len(groups):
                continue
            read = np.zeros([self.num_elements], dtype=bool)
            for layer in group:
                chs = layer._host_desc()["bk_chs"].numpy().astype(np.int64)
                read[(chs[:, None] + np.arange(layer.block_size)[None, :]).reshape(-1)] = True
            written = np.zeros([self.num_elements], dtype=bool)
            for layer in groups[gi + 1]:
                for eg in layer._host_desc()["el_groups"]:
                    for t in eg["tiles"].numpy():
                        written[int(t[0]):int(t[0]) + int(t[1])] = True
            need = read & ~written
            need[:self.num_dummy_eles] = False  # filled at the start of the pass
            idx = np.flatnonzero(need)
            if not idx.size:
                continue
            cuts = np.flatnonzero(np.diff(idx) != 1)
            starts = np.concatenate([[idx[0]], idx[cuts + 1]])
            ends = np.concatenate([idx[cuts] + 1, [idx[-1] + 1]])
            plan[gi] = [(int(a), int(b)) for a, b in zip(starts, ends)]
        return plan

    def _build_em_tables(self):
        """Per sum node block: parameter / flow base, #children, block size (untied vectors only).

        The reference enumerates the same (node, child) parameters per row of at most 32
        children (par_update.py:15-171); here one entry covers a whole node block, whose
        parameters are the contiguous [nch x block_size] slab ``base + k * bs + i``.
        """
        pb, fb, nch, bsz = [], [], [], []
        for ns in self.root_ns:
            if not ns.is_sum() or ns.is_tied():
                continue
            e0 = ns.edge_ids[0].numpy()
            cnt = np.bincount(e0, minlength=ns.num_node_blocks) * ns.ch_block_size
            cum = np.zeros(ns.num_node_blocks, np.int64)
            cum[1:] = np.cumsum(cnt)[:-1]
            pb.append(ns._param_range[0] + cum * ns.block_size)
            fb.append(ns._param_flow_range[0] + cum * ns.block_size)
            nch.append(cnt)
            bsz.append(np.full(ns.num_node_blocks, ns.block_size, np.int64))
        cat = lambda xs: np.concatenate(xs) if xs else np.zeros([0], np.int64)
        self._em_pbase = torch.from_numpy(cat(pb).astype(np.int64))
        self._em_pfbase = torch.from_numpy(cat(fb).astype(np.int64))
        self._em_nch = torch.from_numpy(cat(nch).astype(np.int32))
        self._em_bs = torch.from_numpy(cat(bsz).astype(np.int32))
        # tied sum vectors whose flows live in several slots (parflow_fusing.py:11-78)
        self._tied_sum_fusing = []
        for src, item in self._node2tiednodes.items():
            if len(item[0]) > 1:
                n = src._param_flow_range[1] - src._param_flow_range[0]
                srcs = torch.tensor([r[0] for r in item[1]], dtype=torch.long)
                self._tied_sum_fusing.append((src._param_flow_range[0], n, srcs))

    def _normalize_host(self, params: torch.Tensor, pseudocount: float = 0.0):
        """FP64 sum-to-one normalisation on the host (used at construction)."""
        p = params.double().numpy()
        for pbase, k, bs in zip(self._em_pbase.tolist(), self._em_nch.tolist(), self._em_bs.tolist()):
            slab = p[pbase:pbase + k * bs].reshape(k, bs)
            tot = slab.sum(axis=0)
            p[pbase:pbase + k * bs] = ((slab + pseudocount / k) / (tot + pseudocount)).reshape(-1)
        params.copy_(torch.from_numpy(p).float())

    def _init_parameters(self, perturbation: float = 4.0, pseudocount: float = 0.0):
        """Random / node-provided parameters, normalised (tensorcircuit.py:1094-1120)."""
        for ns in self.root_ns:
            if not ns.is_tied() and (ns.is_sum() or ns.is_input()) and not ns.has_params():
                ns.init_parameters(perturbation=perturbation, recursive=False)
        params = torch.exp(torch.rand([self.num_sum_params]) * -perturbation)
        params[:self.num_dummy_params] = 0.0
        for ns in self.root_ns:
            if ns.is_sum() and not ns.is_tied() and ns.has_params():
                ns.gather_parameters(params)
        self._normalize_host(params, pseudocount)
        self.params = nn.Parameter(params, requires_grad=False)
        for layer in self.input_layer_group:
            layer._init_parameters(perturbation)

    # ------------------------------------------------------------------ device
    def to(self, device):
        device = torch.device(device) if not isinstance(device, int) else torch.device(f"cuda:{device}")
        super().to(device)
        for g in self.inner_layer_groups:
            g.to(device)
        self.input_layer_group.to(device)
        self.device = device
        return self

    def cuda(self, device=None):
        return self.to(torch.device("cuda", device if device is not None else torch.cuda.current_device()))

    def _tables(self):
        key = (self.device.type, self.device.index)
        t = self._dev_tables.get(key)
        if t is None:
            t = dict(pbase=self._em_pbase.to(self.device), pfbase=self._em_pfbase.to(self.device),
                     nch=self._em_nch.to(self.device), bs=self._em_bs.to(self.device),
                     fusing=[(d, n, s.to(self.device)) for d, n, s in self._tied_sum_fusing])
            self._dev_tables[key] = t
        return t

    def _buffer(self, name: str, rows: int, B: int, fresh_value: float):
        t = self.__dict__.get(name)
        if not isinstance(t, torch.Tensor) or t.shape != (rows, B) or t.device != self.device:
            t = torch.full((rows, B), fresh_value, device=self.device, dtype=torch.float32)
            self.__dict__[name] = t
        return t

    # ------------------------------------------------------------------ passes
    def set_propagation_alg(self, propagation_alg: str, **kwargs):
        """Default propagation algorithm of ``forward`` (tensorcircuit.py:192-205): "LL",
        "MPE" or "GeneralLL" (with ``alpha``)."""
        if propagation_alg in ("LL", "MPE"):
            self.default_propagation_alg = propagation_alg
            self.propagation_alg_kwargs.clear()
        elif propagation_alg == "GeneralLL":
            if "alpha" not in kwargs:
                raise ValueError("Argument `alpha` should be provided for the `GeneralLL` propagation algorithm.")
            self.default_propagation_alg = "GeneralLL"
            self.propagation_alg_kwargs.clear()
            self.propagation_alg_kwargs["alpha"] = kwargs["alpha"]
        else:
            raise NotImplementedError(f"Unknown propagation algorithm {propagation_alg}.")

    def forward_ll(self, *args, **kwargs):
        return self.forward(*args, propagation_alg="LL", **kwargs)

    def forward_mpe(self, *args, **kwargs):
        return self.forward(*args, propagation_alg="MPE", **kwargs)

    def forward_general_ll(self, *args, alpha: float = 1.0, **kwargs):
        return self.forward(*args, propagation_alg="GeneralLL", alpha=alpha, **kwargs)

    def _em_view(self, group_id: int) -> torch.Tensor:
        """Element values of product layer group ``group_id`` (rows indexed like ``element_mars``)."""
        if self.recompute_element_values:
            return self.element_mars
        off, rows = self._em_region[group_id]
        return self._em_resident[off:off + rows]

    def _side_stream(self, main: torch.cuda.Stream, i: int = 0) -> torch.cuda.Stream:
        """Side stream ``i`` of the device of ``main`` (created on first use)."""
        pool = self._side_streams.setdefault(main.device, [])
        while len(pool) <= i:
            pool.append(torch.cuda.Stream(device=main.device))
        return pool[i]

    # Sum layers whose packed weights would be byte-identical (tied layers: the time steps of
    # a homogeneous HMM) share one packed buffer, packed once per pass.
    share_tied_packs = True

    def _share_tied_packs(self):
        """Point the packed-weight buffers of sum layers with identical packing inputs at one
        buffer (once per device).

        A packed tile is a function of the parameter values and of (rows, terms, the terms'
        weight offsets kw[k_off ..], w_add, g_stride) and the layout (rows per block, weight
        stride, format): two buffers whose tables agree in all of these hold the same bytes
        whenever both are packed from the same parameters. Tables are compared per role
        (forward tiles, forward 128-term chunks, element-flow tiles and chunks), so the layers
        sharing a buffer also make the same kernel choices; the pack jobs then name the
        buffer once (``_multi_pack`` drops repeated buffers)."""
        key = (self.device.type, self.device.index)
        done = self.__dict__.setdefault("_shared_packs_done", set())
        if key in done or not TensorCircuit.share_tied_packs:
            return
        done.add(key)
        canon = dict()

        def content(tiles, kw):
            t = tiles.cpu().numpy().astype(np.int64)
            kwn = kw.cpu().numpy()
            if t.shape[0] == 0:
                return None
            cnt = t[:, 3]
            idx = np.arange(int(cnt.sum())) + np.repeat(t[:, 2] - (np.cumsum(cnt) - cnt), cnt)
            h = hashlib.sha1(np.ascontiguousarray(t[:, [1, 3, 4, 6]]).tobytes())
            h.update(kwn[idx].astype(np.int64).tobytes())
            return (t.shape[0], h.hexdigest())

        def share(role, holder, tab_key, pack_key, rpb, w_stride, kw, lazy):
            tab = holder.get(tab_key)
            if tab is None:
                return
            c = content(tab, kw)
            if c is None:
                return
            k = (role, rpb, w_stride) + c
            first = canon.get(k)
            if first is None:
                canon[k] = (holder, pack_key, lazy)
                return
            fh, fk, flazy = first
            holder[pack_key] = _ch_pack(fh, fk) if flazy else fh[fk]

        for group in self.inner_layer_groups:
            if not group.is_sum():
                continue
            for layer in group:
                d = layer._desc(self.device)
                share("fw", d, "fw_tiles", "fw_pack", layer.block_size, 1, d["kw"], False)
                share("fwch", d, "fw_ch", "fw_ch_pack", layer.block_size, 1, d["kw"], True)
                for eg in d["el_groups"]:
                    share("el", eg, "tiles", "pack", eg["cbs"], layer.block_size, eg["kw"], False)
                    share("elch", eg, "ch", "ch_pack", eg["cbs"], layer.block_size, eg["kw"], True)

    # Parameter flows of a tied set of sum layers (the time steps of a homogeneous HMM) in one
    # launch (pcb_sum_pflows_tc05_tied) once the last of them has its node flows, instead of
    # one launch per layer that re-reads and re-writes the shared flow slots.
    tied_pflows = True

    def _tied_pflow_sets(self, modify_of: dict):
        """Tied sets of sum layers for pcb_sum_pflows_tc05_tied (cached per flow-rewrite
        pattern): layers whose parameter-flow tables (64-child tiles) agree except for a
        constant shift of their node rows and of their children's element rows, with the same
        parameters and flow slots, block size and rewrite mode. Each set: its members, the
        group of the member that the backward pass reaches last (smallest group index; its
        tables are the reference), and per member (node row, element row) shifts relative to
        it, the element shift including the distance between the members' element-value
        regions."""
        key = (self.device.type, self.device.index, tuple(sorted(modify_of.items())))
        cache = self.__dict__.setdefault("_tied_pflow_cache", dict())
        if key in cache:
            return cache[key]
        by_key = dict()
        for gi, group in enumerate(self.inner_layer_groups):
            if not group.is_sum():
                continue
            for layer in group:
                if not layer._has_tied:
                    continue
                d = layer._desc(self.device)
                pt = d["pf_tiles"].cpu().numpy().astype(np.int64)
                if pt.shape[0] == 0:
                    continue
                krow = d["krow"].cpu().numpy().astype(np.int64)
                h = hashlib.sha1(np.ascontiguousarray(pt[:, 1:]).tobytes())
                h.update((pt[:, 0] - pt[0, 0]).tobytes())
                h.update((krow - krow[0]).tobytes())
                h.update(d["kw"].cpu().numpy().astype(np.int64).tobytes())
                h.update(d["kpf"].cpu().numpy().astype(np.int64).tobytes())
                k = (layer.block_size, bool(modify_of.get(gi)), pt.shape[0], h.hexdigest())
                by_key.setdefault(k, []).append((gi, layer, int(pt[0, 0]), int(krow[0])))
        sets = []
        for members in by_key.values():
            if len(members) < 2:
                continue
            members.sort(key=lambda m: m[0])
            rgi, _, rn, rk = members[0]
            roff = self._em_region[rgi - 1][0]
            deltas = [(n - rn, (self._em_region[gi - 1][0] - roff) + (k - rk)) for gi, _, n, k in members]
            sets.append(dict(last_gi=rgi, ref=members[0][1], layers=[m[1] for m in members],
                             deltas=torch.tensor(deltas, dtype=torch.int32).reshape(-1).to(self.device)))
        cache[key] = sets
        return sets

    def _multi_pack(self, jobs) -> bool:
        """All given weight packs (``SumLayer.forward_pack_job`` tuples) in one launch on the
        current stream; returns whether anything was launched. A buffer named by several jobs
        (shared by tied layers) is packed once."""
        if not jobs:
            return False
        seen, uniq = set(), []
        for j in jobs:
            if (int(j[2].data_ptr()), int(j[5])) not in seen:
                seen.add((int(j[2].data_ptr()), int(j[5])))
                uniq.append(j)
        jobs = uniq
        key = tuple((int(j[2].data_ptr()), int(j[5])) for j in jobs)  # packed buffer and format
        tab = self._pack_tables.get(key)
        if tab is None:
            rec = np.zeros(len(jobs), dtype=_PACK_JOB)
            tj, ti = [], []
            for n, (t, kw, packed, rpb, w_stride, fmt) in enumerate(jobs):
                if rpb <= 0 or rpb & (rpb - 1):
                    raise ValueError("rows per block must be a power of two")
                rec[n] = (t.data_ptr(), kw.data_ptr(), packed.data_ptr(), t.size(0), rpb.bit_length() - 1, w_stride,
                          fmt)
                tj.append(np.full(t.size(0), n, np.int32))
                ti.append(np.arange(t.size(0), dtype=np.int32))
            dev = jobs[0][0].device
            tab = (torch.from_numpy(rec.view(np.uint8).copy()).to(dev), torch.from_numpy(np.concatenate(tj)).to(dev),
                   torch.from_numpy(np.concatenate(ti)).to(dev))
            self._pack_tables[key] = tab
        nat.call("pcb_pack_weights_multi", nat.ptr(self.params), nat.ptr(tab[0]), nat.ptr(tab[1]), nat.ptr(tab[2]),
                 tab[1].size(0), nat.stream())
        return True

    def _pack_state_key(self, B: int, force_use_fp32: bool):
        """What the element-flow packs depend on: the parameter values (storage, torch version
        counter, in-library writes) and the settings that select the packed layers."""
        return (self.params.data_ptr(), self.params._version, self._param_epoch, B, bool(force_use_fp32),
                SumLayer.bf16_form, SumLayer.pack_short_weights, SumLayer.tc05_min_tiles)

    # The forward of the run of small levels next to the root (product layer fused into the
    # single-stage sum kernel above it) in one persistent launch (pcb_lse_levels_short)
    # instead of one launch per level. Off by default: on HCLT-784 (batch 512, BF16) the
    # EM step took 2.65 ms with it against 2.42 ms with the per-level launches, whose
    # programmatic dependent launches already hide most of the launch gaps.
    fuse_levels_forward = False
    # CTAs of that launch (0: four per SM). The run's levels hold a few dozen work items each,
    # so fewer CTAs leave SMs to the side-stream weight packs that overlap it.
    levels_forward_ctas = 0

    def _level_run(self, B, force_use_bf16, force_use_fp32):
        """Sum group indices of the longest run of consecutive small levels that the
        persistent launch can take (each: one product layer with a forward fusion table below
        one single-stage sum layer), or []."""
        groups = self.inner_layer_groups
        ok = []
        for g in range(1, len(groups), 2):
            if not (groups[g].is_sum() and groups[g - 1].is_prod() and len(groups[g]) == 1 and len(groups[g - 1]) == 1):
                ok.append(False)
                continue
            h = self._fusion_host.get(g - 1)
            layer = groups[g][0]
            ok.append(h is not None and h["fw"] is not None and TensorCircuit.fuse_products and
                      SumLayer.short_kernels and
                      layer.runs_single_stage(self.device, B, force_use_bf16, force_use_fp32))
        best, cur = [], []
        for i, o in enumerate(ok):
            cur = cur + [2 * i + 1] if o else []
            if len(cur) > len(best):
                best = cur
        return best if len(best) >= 2 else []

    def _level_tables(self, run, B, force_use_bf16, force_use_fp32):
        """Concatenated tables and level records of a pcb_lse_levels_short launch (cached)."""
        first = self.inner_layer_groups[run[0]][0]
        prec = _mma(first._fw_tc05(first._desc(self.device), B, force_use_bf16, force_use_fp32)[0])
        key = (tuple(run), B, prec, SumLayer.pack_short_weights, id(self.__dict__.get("_em_resident")),
               id(self.element_mars), self.recompute_element_values)
        t = self._level_runs.get(key)
        if t is not None:
            return t
        tb = 32
        nsl = -(-B // tb)
        tiles, krow, kw, tch, recs = [], [], [], [], []
        koff = tile0 = need = item0 = 0
        for g in run:
            layer = self.inner_layer_groups[g][0]
            d = layer._host_desc()
            dd = layer._desc(self.device)
            tt = d["fw_tiles"].numpy().astype(np.int64).copy()
            tt[:, 2] += koff
            tiles.append(tt)
            krow.append(d["krow"].numpy())
            kw.append(d["kw"].numpy())
            tch.append(self._fusion_host[g - 1]["fw"].reshape(-1))
            splits = -(-int(d["fw_tm"]) // 64)
            # the items convert the weights themselves, before their dependency wait
            packed = 0
            per_slice = tt.shape[0] * splits
            recs.append((packed, self._em_view(g - 1).data_ptr(), tile0, tt.shape[0], layer.block_size.bit_length() - 1,
                         1, splits, need, 1 if d["fw_wlayout"] == 1 else 0, item0))
            koff += d["krow"].numel()
            tile0 += tt.shape[0]
            need += per_slice
            item0 += per_slice * nsl
        dev = self.device
        rec = np.zeros(len(recs), dtype=_SHORT_LEVEL)
        for i, r in enumerate(recs):
            rec[i] = r
        t = dict(tiles=torch.from_numpy(np.concatenate(tiles).astype(np.int32)).to(dev),
                 krow=torch.from_numpy(np.concatenate(krow).astype(np.int32)).to(dev),
                 kw=torch.from_numpy(np.concatenate(kw).astype(np.int32)).to(dev),
                 tch=torch.from_numpy(np.concatenate(tch).astype(np.int32)).to(dev),
                 levels=torch.from_numpy(rec.view(np.uint8).copy()).to(dev), num_levels=len(run),
                 items=item0, slices=nsl, tb=tb, prec=prec,
                 counters=torch.zeros([1 + nsl], dtype=torch.int32, device=dev))
        self._level_runs[key] = t
        return t

    def _run_inner_forward(self, force_use_bf16, force_use_fp32, propagation_alg, **kwargs):
        # The weights that the sum kernels read packed are packed on a side stream in two
        # launches: the forward's (waited for before the first layer that reads them) and the
        # element-flow weights of the backward pass that follows (joined at the end).
        main = torch.cuda.current_stream()
        side = self._side_stream(main)
        side.wait_stream(main)
        self._share_tied_packs()
        B = self.node_mars.size(1)
        plain = propagation_alg == "LL" if isinstance(propagation_alg, str) else all(a == "LL" for a in propagation_alg)
        run = (self._level_run(B, force_use_bf16, force_use_fp32)
               if (TensorCircuit.fuse_levels_forward and plain and not self._fw_partial_eval_enabled) else [])
        fw_jobs, el_jobs, fw_groups = [], [], set()
        for gi, group in enumerate(self.inner_layer_groups):
            if group.is_sum():
                for layer in group:
                    job = None if gi in run else layer.forward_pack_job(self.device, B, force_use_bf16, force_use_fp32)
                    if job is not None:
                        fw_jobs.append(job)
                        fw_groups.add(gi)
                    el_jobs += layer.flow_pack_jobs(self.device, B, force_use_fp32)
        fw_ready = None
        with torch.cuda.stream(side):
            if self._multi_pack(fw_jobs):
                fw_ready = torch.cuda.Event()
                fw_ready.record(side)
            self._multi_pack(el_jobs)
        self._el_pack_state = self._pack_state_key(B, force_use_fp32)
        groups = self.inner_layer_groups
        in_run = set(run) | set(g - 1 for g in run)
        for gi, group in enumerate(groups):
            alg = propagation_alg if isinstance(propagation_alg, str) else propagation_alg[gi]
            if gi in in_run:
                if gi == run[0] - 1:  # the whole run in one launch
                    if fw_ready is not None:
                        main.wait_event(fw_ready)
                        fw_ready = None
                    lt = self._level_tables(run, B, force_use_bf16, force_use_fp32)
                    nat.call("pcb_lse_levels_short", nat.ptr(self.node_mars), self.node_mars.stride(0), B,
                             nat.ptr(self.params), nat.ptr(lt["tiles"]), nat.ptr(lt["krow"]), nat.ptr(lt["kw"]),
                             nat.ptr(lt["tch"]), nat.ptr(lt["levels"]), lt["num_levels"], lt["items"], lt["slices"],
                             nat.ptr(lt["counters"]), lt["prec"], lt["tb"], 0,
                             TensorCircuit.levels_forward_ctas or 4 * _num_sms(), nat.stream())
                continue
            if group.is_prod():
                fused = (not self._fw_partial_eval_enabled and gi + 1 < len(groups) and
                         self._fusion_tables(gi, "fw") is not None and
                         groups[gi + 1][0].runs_single_stage(self.device, B, force_use_bf16, force_use_fp32))
                if not fused:  # else the next sum layer computes (and writes) these element values
                    group(self.node_mars, self._em_view(gi))
            else:
                if gi in fw_groups and fw_ready is not None:
                    main.wait_event(fw_ready)
                    fw_ready = None
                fz = None if self._fw_partial_eval_enabled else self._fusion_tables(gi - 1, "fw")
                if fz is not None and not group[0].runs_single_stage(self.device, B, force_use_bf16, force_use_fp32):
                    fz = None
                if alg != "LL" and fz is not None:  # the fused kernels run LL only
                    raise RuntimeError("forward product fusion runs the LL algorithm only")
                group(self.node_mars, self._em_view(gi - 1), self.params, force_use_bf16=force_use_bf16,
                      force_use_fp32=force_use_fp32, propagation_alg=alg, _weights_packed=True,
                      _fuse_fw=None if fz is None else (fz, self._em_view(gi - 1)), **kwargs)
        main.wait_stream(side)

    def forward(self, inputs: torch.Tensor, input_layer_fn: Optional[Union[str, Callable]] = None,
                cache: Optional[dict] = None, return_cache: bool = False, record_cudagraph: bool = False,
                apply_cudagraph: bool = True, force_use_bf16: bool = False, force_use_fp32: bool = False,
                propagation_alg: Optional[str] = None, _inner_layers_only: bool = False,
                _no_buffer_reset: bool = False, **kwargs):
        """Log-likelihoods ``[B, num_root_nodes]`` of ``inputs`` (``[B, num_vars]`` int64)."""
        if self.device.type != "cuda":
            raise RuntimeError("TensorCircuit runs on CUDA only: call pc.to('cuda') first")
        if propagation_alg is None:
            propagation_alg = self.default_propagation_alg
            kwargs.update(self.propagation_alg_kwargs)
        if not isinstance(propagation_alg, str):
            propagation_alg = tuple(propagation_alg)
            if len(propagation_alg) != len(self.inner_layer_groups):
                raise ValueError("a per-layer propagation_alg needs one entry per inner layer group")
        with torch.no_grad():
            B = inputs.size(0)
            origin_inputs = inputs
            if input_layer_fn is None:
                if inputs.dim() != 2:
                    raise ValueError("inputs must be [B, num_vars]")
                data = inputs.permute(1, 0).to(self.device).contiguous()
            nm = self._buffer("node_mars", self.num_nodes, B, 0.0)
            em = self._buffer("element_mars", self.num_elements, B, -float("inf"))
            # dummy rows of every region keep their initial -inf (nothing writes them)
            if not self.recompute_element_values:
                self._buffer("_em_resident", self._em_rows, B, -float("inf"))
            if not _no_buffer_reset:
                nat.call("pcb_fill_rows", nat.ptr(nm), B, 0, self.num_dummy_nodes, 0.0, nat.stream())
                nat.call("pcb_fill_rows", nat.ptr(em), B, 0, self.num_dummy_eles, -float("inf"), nat.stream())
            if cache is not None and "node_mars" in cache and cache["node_mars"].shape == nm.shape:
                nm.copy_(cache["node_mars"])
            if not _inner_layers_only:
                for layer in self.input_layer_group:
                    if input_layer_fn is None:
                        layer(data, nm, **kwargs)
                    elif isinstance(input_layer_fn, str):
                        getattr(layer, input_layer_fn)(inputs, nm, **kwargs)
                    else:
                        ret = input_layer_fn(layer, inputs, nm, **kwargs)
                        if not ret and ret is not None:
                            layer(data, nm, **kwargs)
            sig = (0, id(nm), id(em), id(self.__dict__.get("_em_resident")), id(self.params), B, force_use_bf16,
                   force_use_fp32,
                   propagation_alg, kwargs.get("alpha"), self._partial_epoch)
            run = partial(self._run_inner_forward, force_use_bf16, force_use_fp32, propagation_alg, **kwargs)
            if record_cudagraph and sig not in self._recorded_cuda_graphs:
                self._recorded_cuda_graphs[sig] = self._capture(run)
            if apply_cudagraph and sig in self._recorded_cuda_graphs:
                self._recorded_cuda_graphs[sig].replay()
            else:
                run()
            lls = nm[self._root_node_range[0]:self._root_node_range[1], :].permute(1, 0)
        if return_cache:
            cache = dict() if cache is None else cache
            cache["node_mars"] = nm.clone()
        out = lls.clone()
        if torch.is_grad_enabled():
            out.requires_grad = True
            # the backward contraction runs in the precision form the forward used
            out.register_hook(partial(_pc_model_backward_hook, pc=self, inputs=origin_inputs,
                                      record_cudagraph=record_cudagraph, apply_cudagraph=apply_cudagraph,
                                      propagation_alg=propagation_alg, force_use_fp32=force_use_fp32, **kwargs))
        if return_cache:
            return out, cache
        return out

    def _capture(self, fn, reset=None):
        """CUDA graph of ``fn`` after two warm-up runs; ``reset`` (if given) restores the state
        that ``fn`` reads before each warm-up run."""
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(2):
                if reset is not None:
                    reset()
                fn()
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        return g

    def _run_inner_backward(self, compute_param_flows, allow_modify_flows, logspace_flows, force_use_fp32,
                            propagation_alg="LL", negate_pflows=False, **kwargs):
        # Parameter flows go to side streams: nothing later in the pass reads them, so they run
        # alongside the element-flow / product chain and join before the pass ends. The
        # parameter-flow launches of the small levels are latency-bound, so consecutive levels
        # take turns over several streams and overlap one another.
        main = torch.cuda.current_stream()
        sides = [self._side_stream(main, i) for i in range(max(1, TensorCircuit.pflow_streams))]
        for side in sides:
            side.wait_stream(main)
        B = self.node_mars.size(1)
        self._share_tied_packs()
        # Element-flow weights: packed by the forward pass when the parameters have not changed
        # since (the state is set by the forward only, so that every run of a captured backward
        # makes the same choice); otherwise packed here in one launch.
        el_ready = None
        if self._el_pack_state != self._pack_state_key(B, force_use_fp32):
            el_jobs = [job for group in self.inner_layer_groups if group.is_sum() for layer in group
                       for job in layer.flow_pack_jobs(self.device, B, force_use_fp32)]
            with torch.cuda.stream(sides[0]):
                if self._multi_pack(el_jobs):
                    el_ready = torch.cuda.Event()
                    el_ready.record(sides[0])
        kwargs = dict(kwargs, _weights_packed=True)
        plain = (propagation_alg == "LL" if isinstance(propagation_alg, str) else
                 all(a == "LL" for a in propagation_alg)) and not negate_pflows and not logspace_flows and \
            not kwargs.get("allow_neg_flows") and not self._bk_partial_eval_enabled
        turn = 0
        def rewrites(g):  # large layers rewrite their node flows as log f - log m
            return allow_modify_flows and any(
                layer._desc(self.device)["fw_tiles"].size(0) >= SumLayer.tc05_min_tiles
                for layer in self.inner_layer_groups[g])

        # product layers fused into the element-flow kernel above them in this pass
        fuse_bw = dict()
        for g, group in enumerate(self.inner_layer_groups):
            if not group.is_sum() or rewrites(g) or not plain:
                continue
            fz = self._fusion_tables(g - 1, "bw")
            if fz is not None and group[0].runs_single_stage(self.device, B, force_use_fp32=force_use_fp32,
                                                             backward=True):
                fuse_bw[g] = fz
        fused_prod = set(g - 1 for g in fuse_bw)
        # parameter flows of tied sets in one launch each (tcgen05 form, resident element values)
        pprec = 0 if force_use_fp32 or B < 16 else _mma(SumLayer.bf16_form)
        tied_sets = []
        if (TensorCircuit.tied_pflows and compute_param_flows and plain and pprec > 0 and
                not self.recompute_element_values and SumLayer.pflow_tc05 is not False and
                SumLayer.pflow_tile_children in (None, 0, 64)):
            tied_sets = self._tied_pflow_sets({g: rewrites(g) for g, grp in enumerate(self.inner_layer_groups)
                                               if grp.is_sum()})
        pflow_skip = {id(l) for ts in tied_sets for l in ts["layers"]}
        rw_flags, rewritten = (self._rewrite_plan(fused_prod) if (TensorCircuit.fuse_flow_rewrite and
                                                                  allow_modify_flows and not logspace_flows)
                               else (dict(), set()))

        for layer_id in range(len(self.inner_layer_groups) - 1, -1, -1):
            group = self.inner_layer_groups[layer_id]
            if group.is_prod():
                if layer_id in fused_prod:  # the sum layer above wrote these flows
                    continue
                # element rows that the sum group above left unwritten (parentless elements)
                for a, b in self._ef_init_ranges.get(layer_id, ()):
                    nat.call("pcb_fill_rows", nat.ptr(self.element_flows), B, a, b,
                             -float("inf") if logspace_flows else 0.0, nat.stream())
                rf = rw_flags.get(layer_id)
                group.backward(self.node_flows, self.element_flows, logspace_flows=logspace_flows,
                               _modify=None if rf is None else (self.node_mars, rf))
            else:
                # The element values of the forward pass are still resident (no recomputation). Small
                # layers form log f - log m inside the flow kernels instead of rewriting the node flows
                # in place (one launch fewer); large ones rewrite them once (allow_modify_flows) so that
                # the two flow kernels read one row per node instead of two.
                modify = rewrites(layer_id)
                if el_ready is not None:
                    main.wait_event(el_ready)
                    el_ready = None
                fz = fuse_bw.get(layer_id)
                alg = propagation_alg if isinstance(propagation_alg, str) else propagation_alg[layer_id]
                pstream = sides[turn % len(sides)]
                if self.recompute_element_values:
                    # the element values of the product group below, recomputed into the shared
                    # buffer; the parameter flows then stay on this stream (the next recompute
                    # overwrites the buffer)
                    self.inner_layer_groups[layer_id - 1](self.node_mars, self.element_mars)
                    pstream = None
                group.backward(self.node_flows, self.element_flows, self.node_mars, self._em_view(layer_id - 1),
                               self.params,
                               param_flows=self.param_flows if compute_param_flows else None,
                               allow_modify_flows=modify, logspace_flows=logspace_flows,
                               force_use_fp32=force_use_fp32, _pflow_stream=pstream, _fuse_bw=fz,
                               _flows_modified=layer_id in rewritten, propagation_alg=alg,
                               negate_pflows=negate_pflows, _pflow_skip=pflow_skip, **kwargs)
                turn += 1
                for ts in tied_sets:
                    if ts["last_gi"] != layer_id:
                        continue
                    # every member has its (rewritten) node flows now
                    ev = torch.cuda.Event()
                    ev.record(main)
                    side = sides[turn % len(sides)]
                    side.wait_event(ev)
                    ref = ts["ref"]
                    rd = ref._desc(self.device)
                    pt = rd["pf_tiles"]
                    with torch.cuda.stream(side):
                        nat.call("pcb_sum_pflows_tc05_tied", nat.ptr(self.node_flows), nat.ptr(self.node_mars),
                                 nat.ptr(self._em_view(layer_id - 1)), self.node_mars.stride(0), B,
                                 nat.ptr(self.params), nat.ptr(self.param_flows), nat.ptr(pt), pt.size(0),
                                 ref.block_size, nat.ptr(rd["krow"]), nat.ptr(rd["kw"]), nat.ptr(rd["kpf"]),
                                 1 if modify else 0, 1, 64, pprec, nat.ptr(ts["deltas"]), len(ts["layers"]),
                                 nat.stream())
                    turn += 1
        for side in sides:
            main.wait_stream(side)

    def backward(self, inputs: Optional[torch.Tensor] = None, ll_weights: Optional[torch.Tensor] = None,
                 compute_param_flows: bool = True, flows_memory: float = 1.0,
                 input_layer_fn: Optional[Union[str, Callable]] = None, cache: Optional[dict] = None,
                 sum_layer_pre_backward_callback: Optional[Callable] = None,
                 sum_layer_post_backward_callback: Optional[Callable] = None, return_cache: bool = False,
                 record_cudagraph: bool = False, apply_cudagraph: bool = True, allow_modify_flows: bool = True,
                 propagation_alg: str = "LL", logspace_flows: bool = False, negate_pflows: bool = False,
                 _inner_layers_only: bool = False, _disable_buffer_init: bool = False, force_use_fp32: bool = False,
                 **kwargs):
        """Node flows, element flows and (accumulated) parameter flows of the last forward batch."""
        if self.node_mars is None or self.element_mars is None:
            raise RuntimeError("Should run forward path first.")
        if allow_modify_flows and logspace_flows:
            raise ValueError("`allow_modify_flows` should be set to `False` when using `logspace_flows`.")
        if not isinstance(propagation_alg, str):
            propagation_alg = tuple(propagation_alg)
        if propagation_alg != "LL" or negate_pflows or kwargs.get("allow_neg_flows") or self._bk_partial_eval_enabled:
            # the kernels of these modes read unmodified node flows (the results are the same)
            allow_modify_flows = False
        if sum_layer_pre_backward_callback is not None or sum_layer_post_backward_callback is not None:
            raise NotImplementedError("sum-layer callbacks are not supported")
        self._run_params.update(allow_modify_flows=allow_modify_flows, propagation_alg=propagation_alg,
                                logspace_flows=logspace_flows, negate_pflows=negate_pflows,
                                force_use_fp32=force_use_fp32)
        with torch.no_grad():
            B = self.node_mars.size(1)
            if input_layer_fn is None:
                if inputs is None or inputs.dim() != 2 or inputs.size(1) != self.num_vars:
                    raise ValueError("inputs must be [B, num_vars]")
                data = inputs.permute(1, 0).to(self.device).contiguous()
            init = -float("inf") if logspace_flows else 0.0
            nf = self._buffer("node_flows", self.num_nodes, B, init)
            ef = self._buffer("element_flows", self.num_elements, B, init)
            if not _disable_buffer_init:
                # only the rows that no product layer overwrites (see _plan_node_flow_init)
                if len(self._nf_init_ranges) > 16:
                    nf.fill_(init)
                else:
                    for a, b in self._nf_init_ranges:
                        nat.call("pcb_fill_rows", nat.ptr(nf), B, a, b, init, nat.stream())
                nat.call("pcb_fill_rows", nat.ptr(ef), B, 0, self.num_dummy_eles, init, nat.stream())
            r0, r1 = self._root_node_range
            if ll_weights is None:
                nf[r0:r1, :] = 0.0 if logspace_flows else 1.0
            else:
                w = ll_weights.unsqueeze(0) if ll_weights.dim() == 1 else ll_weights
                if w.size(0) != self.num_root_nodes:
                    raise ValueError("ll_weights must be [num_root_nodes, B]")
                nf[r0:r1, :] = w.log() if logspace_flows else w
            if compute_param_flows:
                if self._cum_flow_dev is None or self._cum_flow_dev.device != self.device:
                    self._cum_flow_dev = torch.zeros([], dtype=torch.float64, device=self.device)
                if ll_weights is None:
                    self._cum_flow_dev += float((r1 - r0) * B)
                else:
                    self._cum_flow_dev += ll_weights.double().sum()
            if cache is not None and "node_flows" in cache and cache["node_flows"].shape == nf.shape:
                nf.copy_(cache["node_flows"])
            if compute_param_flows:
                self.init_param_flows(flows_memory=flows_memory)
            sig = (1, id(nf), id(ef), id(self.node_mars), id(self.__dict__.get("_em_resident")), id(self.params),
                   id(self.param_flows), B, allow_modify_flows, logspace_flows, force_use_fp32, compute_param_flows,
                   propagation_alg, negate_pflows, kwargs.get("alpha"), self._partial_epoch)
            run = partial(self._run_inner_backward, compute_param_flows, allow_modify_flows, logspace_flows,
                          force_use_fp32, propagation_alg=propagation_alg, negate_pflows=negate_pflows, **kwargs)
            if record_cudagraph and sig not in self._recorded_cuda_graphs:
                # The pass rewrites node flows in place and accumulates parameter flows, so each
                # warm-up run starts from the state of this call and the state is put back after
                # the capture (a second run on rewritten flows can overflow).
                saved_nf = nf.clone()
                saved_pf = self.param_flows.clone() if compute_param_flows else None

                def reset():
                    nf.copy_(saved_nf)
                    if saved_pf is not None:
                        self.param_flows.copy_(saved_pf)

                self._recorded_cuda_graphs[sig] = self._capture(run, reset)
                reset()
                del saved_nf, saved_pf
            if apply_cudagraph and sig in self._recorded_cuda_graphs:
                self._recorded_cuda_graphs[sig].replay()
            else:
                run()
            if not _inner_layers_only:
                for layer in self.input_layer_group:
                    if input_layer_fn is None:
                        layer.backward(data, nf, self.node_mars, logspace_flows=logspace_flows, **kwargs)
                    elif isinstance(input_layer_fn, str):
                        getattr(layer, input_layer_fn)(inputs, nf, self.node_mars, logspace_flows=logspace_flows, **kwargs)
                    else:
                        ret = input_layer_fn(layer, inputs, nf, self.node_mars, logspace_flows=logspace_flows, **kwargs)
                        if not ret and ret is not None:
                            layer.backward(data, nf, self.node_mars, logspace_flows=logspace_flows, **kwargs)
        if return_cache:
            cache = dict() if cache is None else cache
            cache["node_flows"] = nf.clone()
            return cache
        return None

    @property
    def _cum_flow(self) -> float:
        return 0.0 if self._cum_flow_dev is None else float(self._cum_flow_dev.item())

    def mini_batch_em(self, step_size: float, pseudocount: float = 0.0, keep_zero_params: bool = False,
                      step_size_rescaling: bool = False, use_cudagraph: bool = True, use_f64_flows: bool = False):
        """EM update from the accumulated parameter flows (tensorcircuit.py:549-590).

        ``use_f64_flows``: update from the FP64 epoch flows (``param_flows_f64``, see
        :meth:`accumulate_param_flows_f64`) instead of the FP32 ``param_flows``.
        """
        if not (0.0 < step_size <= 1.0):
            raise ValueError("`step_size` should be between 0 and 1.")
        if step_size_rescaling:
            # mini-batch EM objective (tensorcircuit.py:566-577): the accumulated flows are scaled
            # by step / (total root flow) and the walk's own flows are added with weight 1 - step;
            # the update then uses step 1
            if use_f64_flows:
                raise ValueError("step_size_rescaling works on the FP32 parameter flows")
            cum = self._cum_flow
            if not cum > 0.0:
                raise RuntimeError("Please perform a backward pass before calling `mini_batch_em`.")
            with torch.no_grad():
                self.init_param_flows(flows_memory=step_size / cum)
                from .top_down import eval_top_down_probs
                eval_top_down_probs(self, update_pflow=True, scale=1.0 - step_size, use_cudagraph=use_cudagraph)
            self._cum_flow_dev.zero_()
            step_size = 1.0
        if self.param_flows is None and not use_f64_flows:
            raise RuntimeError("run a backward pass before mini_batch_em")
        if use_f64_flows and self.param_flows_f64 is None:
            raise RuntimeError("no FP64 flows: call init_param_flows_f64 / accumulate_param_flows_f64 first")
        with torch.no_grad():
            for layer in self.input_layer_group:
                layer.mini_batch_em(step_size=step_size, pseudocount=pseudocount, keep_zero_params=keep_zero_params,
                                    use_f64_flows=use_f64_flows)
            t = self._tables()
            pf = self.param_flows_f64 if use_f64_flows else self.param_flows
            for dst, n, srcs in t["fusing"]:
                nat.call("pcb_pflow_accum_f64" if use_f64_flows else "pcb_pflow_accum", nat.ptr(pf), dst, n,
                         nat.ptr(srcs), srcs.size(0), nat.stream())
            nat.call("pcb_sum_em_f64flows" if use_f64_flows else "pcb_sum_em", nat.ptr(self.params), nat.ptr(pf),
                     nat.ptr(t["pbase"]), nat.ptr(t["pfbase"]), nat.ptr(t["nch"]), nat.ptr(t["bs"]), t["nch"].size(0),
                     float(step_size), float(pseudocount), 1 if keep_zero_params else 0, nat.stream())
            self._param_epoch += 1

    def init_param_flows_f64(self):
        """Zero the FP64 epoch-level parameter flows (sum and input layers)."""
        n = max(self.num_param_flows, 1)
        if self.param_flows_f64 is None or self.param_flows_f64.device != self.device or self.param_flows_f64.numel() != n:
            self.param_flows_f64 = torch.zeros([n], dtype=torch.float64, device=self.device)
        else:
            self.param_flows_f64.zero_()
        for layer in self.input_layer_group:
            layer.init_param_flows_f64()

    def accumulate_param_flows_f64(self):
        """Add the FP32 parameter flows of the last backward pass(es) to the FP64 epoch flows.

        An epoch of full-batch EM then reads: per batch ``init_param_flows(0)``, forward,
        backward, ``accumulate_param_flows_f64()``; at the end
        ``mini_batch_em(1.0, pseudocount, use_f64_flows=True)``. The reference sums the
        batches' flows in FP32 (``cumulate_flows``, tensorcircuit.py:592-595); here each
        batch's FP32 flows are added into FP64 on the device (``pcb_flows_accumulate_f64``).
        """
        if self.param_flows is None:
            raise RuntimeError("run a backward pass first")
        if self.param_flows_f64 is None or self.param_flows_f64.device != self.device:
            self.init_param_flows_f64()
        with torch.no_grad():
            nat.call("pcb_flows_accumulate_f64", nat.ptr(self.param_flows_f64), nat.ptr(self.param_flows),
                     self.num_param_flows, nat.stream())
            for layer in self.input_layer_group:
                layer.accumulate_param_flows_f64()

    def set_params_from_logits(self, logits: torch.Tensor):
        """Sum weights = softmax of ``logits`` over each node's children (``logits`` in the
        layout of ``params``; entries outside the nodes' weights are ignored)."""
        if logits.shape != self.params.shape or logits.dtype != torch.float32 or logits.device != self.device:
            raise ValueError("logits must be a float32 tensor shaped like `params` on the circuit's device")
        t = self._tables()
        with torch.no_grad():
            nat.call("pcb_sum_softmax", nat.ptr(logits.contiguous()), nat.ptr(self.params), nat.ptr(t["pbase"]),
                     nat.ptr(t["nch"]), nat.ptr(t["bs"]), t["nch"].size(0), nat.stream())
        self._param_epoch += 1

    def sum_logit_grad(self, scale: float = 1.0, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Gradient with respect to softmax logits of the sum weights from the current parameter
        flows: ``scale * (pf - theta * sum_children pf)`` in the layout of ``params`` (tied flow
        slots are summed into their source slots first)."""
        if self.param_flows is None:
            raise RuntimeError("run a backward pass first")
        t = self._tables()
        out = torch.zeros_like(self.params) if out is None else out
        with torch.no_grad():
            for dst, n, srcs in t["fusing"]:
                nat.call("pcb_pflow_accum", nat.ptr(self.param_flows), dst, n, nat.ptr(srcs), srcs.size(0),
                         nat.stream())
            nat.call("pcb_sum_logit_grad", nat.ptr(self.params), nat.ptr(self.param_flows), nat.ptr(t["pbase"]),
                     nat.ptr(t["pfbase"]), nat.ptr(t["nch"]), nat.ptr(t["bs"]), t["nch"].size(0), float(scale),
                     nat.ptr(out), nat.stream())
        return out

    def normalize_parameters(self, pseudocount: float = 0.0):
        """Renormalise the sum parameters in place on the device (FP64)."""
        t = self._tables()
        nat.call("pcb_sum_normalize", nat.ptr(self.params), nat.ptr(t["pbase"]), nat.ptr(t["nch"]), nat.ptr(t["bs"]),
                 t["nch"].size(0), float(pseudocount), nat.stream())
        self._param_epoch += 1

    def cumulate_flows(self, inputs: torch.Tensor, params: Optional[torch.Tensor] = None, fp64: bool = False):
        """Forward + backward adding this batch's parameter flows to the kept ones
        (tensorcircuit.py:592-595). ``fp64``: the batch's flows go to the FP64 epoch flows
        instead (``param_flows`` then holds this batch's flows only)."""
        if params is not None:
            raise NotImplementedError("external parameters have no CUDA path")
        with torch.no_grad():
            self.forward(inputs)
            self.backward(inputs=inputs, compute_param_flows=True, flows_memory=0.0 if fp64 else 1.0)
            if fp64:
                self.accumulate_param_flows_f64()

    def init_param_flows(self, flows_memory: float = 1.0, batch_size: Optional[int] = None):
        if not (0.0 <= flows_memory <= 1.0):
            raise ValueError("`flows_memory` should be in [0.0, 1.0]")
        if batch_size is not None:
            raise NotImplementedError("per-sample parameter flows are not supported")
        pf = self.param_flows
        if not isinstance(pf, torch.Tensor) or pf.shape != (self.num_param_flows,) or pf.device != self.device:
            self.param_flows = torch.zeros([self.num_param_flows], device=self.device)
        elif flows_memory == 0.0:
            self.param_flows.zero_()  # write-only; same as multiplying finite flows by zero
        elif flows_memory != 1.0:
            self.param_flows.mul_(flows_memory)
        for layer in self.input_layer_group:
            layer.init_param_flows(flows_memory=flows_memory)

    def zero_param_flows(self):
        self.init_param_flows(flows_memory=0.0)

    def update_parameters(self, clone: bool = True):
        params = self.params.detach().cpu()
        for ns in self.root_ns:
            if ns.is_sum() and not ns.is_tied():
                ns.update_parameters(params, clone=clone)
        for layer in self.input_layer_group:
            layer.update_parameters()

    def update_param_flows(self, clone: bool = True, origin_ns_only: bool = True):
        pf = self.param_flows.detach().cpu()
        for ns in self.root_ns:
            if ns.is_sum() and not ns.is_tied():
                ns.update_param_flows(pf, clone=clone, origin_ns_only=origin_ns_only)

    def print_statistics(self):
        print(f"> Number of nodes: {self.num_nodes}")
        print(f"> Number of edges: {self.num_edges}")
        print(f"> Number of sum parameters: {self.num_sum_params}")
        print(f"> Number of input parameters: {sum(l.params.numel() for l in self.input_layer_group)}")

    def get_node_mars(self, ns: CircuitNodes):
        nsid, neid = ns._output_ind_range
        if ns.is_sum() or ns.is_input():
            return self.node_mars[nsid:neid, :].detach()
        for group in self.inner_layer_groups:
            for layer in group:
                if layer.is_prod() and any(n is ns for n in layer.nodes):
                    layer(self.node_mars, self.element_mars)
                    return self.element_mars[nsid:neid, :].detach()
        raise ValueError("node not found in the circuit")

    def get_node_flows(self, ns: CircuitNodes, **kwargs):
        nsid, neid = ns._output_ind_range
        if ns.is_sum() or ns.is_input():
            return self.node_flows[nsid:neid, :].detach()
        for idx, group in enumerate(self.inner_layer_groups):
            for layer in group:
                if layer.is_prod() and any(n is ns for n in layer.nodes):
                    self.inner_layer_groups[idx].forward(self.node_mars, self.element_mars, _for_backward=True)
                    self.inner_layer_groups[idx + 1].backward(
                        self.node_flows, self.element_flows, self.node_mars, self.element_mars, self.params,
                        param_flows=None, allow_modify_flows=False, force_use_fp32=True)
                    return self.element_flows[nsid:neid, :].detach()
        raise ValueError("node not found in the circuit")

    def enable_partial_evaluation(self, scopes, forward: bool = False, backward: bool = False, overwrite: bool = False):
        """Evaluate only the node vectors whose scope is one of ``scopes`` (BitSets, or variable
        ids for single-variable scopes) in later forward and/or backward passes; every other
        row keeps its value (tensorcircuit.py:815-841). Typical use: after a full pass with
        ``return_cache=True``, change some variables and re-run with the scopes that contain
        them (``nodes.get_subsumed_scopes``) and ``cache=``."""
        from ..nodes.scope import BitSet
        if not overwrite and ((forward and self._fw_partial_eval_enabled) or
                              (backward and self._bk_partial_eval_enabled)):
            raise RuntimeError("Partial evaluation already enabled, consider calling `disable_partial_evaluation` first.")
        scopes = [BitSet.from_array([v]) if isinstance(v, int) else v for v in scopes]
        fw = scopes if forward else None
        bk = scopes if backward else None
        for layer in self.input_layer_group:
            layer.enable_partial_evaluation(fw_scopes=fw, bk_scopes=bk)
        for group in self.inner_layer_groups:
            group.enable_partial_evaluation(fw_scopes=fw, bk_scopes=bk)
        self._fw_partial_eval_enabled |= forward
        self._bk_partial_eval_enabled |= backward
        self._partial_epoch += 1

    def disable_partial_evaluation(self, forward: bool = True, backward: bool = True):
        for layer in self.input_layer_group:
            layer.disable_partial_evaluation(forward=forward, backward=backward)
        for group in self.inner_layer_groups:
            group.disable_partial_evaluation(forward=forward, backward=backward)
        if forward:
            self._fw_partial_eval_enabled = False
        if backward:
            self._bk_partial_eval_enabled = False
        self._partial_epoch += 1

    def layers(self, reverse: bool = False, ret_layer_groups: bool = False, ignore_input_layers: bool = False):
        groups = ([] if ignore_input_layers else [self.input_layer_group]) + list(self.inner_layer_groups)
        if reverse:
            groups = groups[::-1]
        for g in groups:
            if ret_layer_groups:
                yield g
            else:
                for l in g:
                    yield l

    def dataset_ll_accumulate(self, lls: torch.Tensor, acc: torch.Tensor):
        """Adds sum_b lls[b, 0] to the FP64 device scalar ``acc`` (dataset-level LL, FP64)."""
        if acc.dtype != torch.float64 or not acc.is_cuda:
            raise ValueError("acc must be a float64 CUDA tensor")
        x = lls[:, 0].contiguous()
        nat.call("pcb_ll_sum_f64", nat.ptr(x), x.numel(), x.numel(), 0, nat.ptr(acc), nat.stream())


def compile(ns: CircuitNodes, layer_sparsity_tol: float = 0.5, max_num_partitions: Optional[int] = None,
            disable_gpu_compilation: bool = False, force_gpu_compilation: bool = False,
            max_tied_ns_per_parflow_block: int = 8, device: Optional[Union[int, torch.device]] = None,
            verbose: bool = False) -> TensorCircuit:
    """Compile a circuit DAG into a ``TensorCircuit`` (reference: tensorcircuit.py:1224-1261)."""
    return TensorCircuit(ns, layer_sparsity_tol=layer_sparsity_tol, max_num_partitions=max_num_partitions,
                         max_tied_ns_per_parflow_block=max_tied_ns_per_parflow_block, device=device, verbose=verbose)
