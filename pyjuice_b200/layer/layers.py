"""Compiled layers: input (Categorical), product and sum layers, and layer groups.

Each layer keeps the reference's compiled tables (``partitioned_*``, ``_layer_nid_range``
and friends, see ``compilation.py``) and, per CUDA device, a set of compact int32 kernel
descriptors derived from them (tile lists and block lists without the power-of-2
padding). ``forward`` / ``backward`` launch the sm_100a kernels of ``libpcb200.so``
through ``_native``; there is no CPU path.

Interfaces follow the reference's ``SumLayer`` (src/pyjuice/layer/sum_layer.py:30-384),
``ProdLayer`` (src/pyjuice/layer/prod_layer.py:28-237), ``InputLayer``
(src/pyjuice/layer/input_layer.py:32-724) and ``LayerGroup``
(src/pyjuice/layer/layer_group.py:14-108).
"""

from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np
import torch

from ctypes import c_void_p

from .. import _native as nat
from ..autotune import TUNER
from .compilation import compile_prod_layer, compile_sum_layer
from .input_layer_compile import compile_input_layer


def _i32(x) -> torch.Tensor:
    a = np.asarray(x, dtype=np.int64)
    if a.size and (a.max() >= 2 ** 31 or a.min() < -2 ** 31):
        raise ValueError("index exceeds the int32 range of the kernel tables")
    return torch.from_numpy(a.astype(np.int32))


_MAX_ROWS = 128  # tallest contraction tile (rows that share one staged set of terms)


def _tile_rows(max_rows: int) -> int:
    t = 1
    while t < max_rows and t < _MAX_ROWS:
        t *= 2
    return t


_SHORT_K = 128  # terms per tile handled by the single-stage kernels (pcb_lse_contract_short)
_NUM_SMS = None
_PACK_BYTES = 65536  # packed bf16 hi + lo weights of one tile (pcb_pack_weights)


def _num_sms() -> int:
    global _NUM_SMS
    if _NUM_SMS is None:
        _NUM_SMS = max(1, int(nat.load().pcb_num_sms()))
    return _NUM_SMS


def _short_batch_tile(num_tiles: int, tile_rows: int, B: int, fused: bool = False) -> int:
    """Samples per CTA for pcb_lse_contract_short: the widest slice that still launches two
    CTAs per SM (small layers get narrow slices and therefore more CTAs); at most 32 when a
    product layer is fused in."""
    splits = 1 if tile_rows <= 32 else -(-tile_rows // 64)
    for tb in ((32,) if fused else (64, 32)):
        if num_tiles * splits * -(-B // tb) >= 2 * _num_sms():
            return tb
    return 16


def _tc05_batch_tile(num_tiles: int, B: int) -> int:
    """Samples per CTA for pcb_lse_contract_tc05 (two CTAs per SM fit in shared memory)."""
    return 64 if num_tiles * -(-B // 64) >= 2 * _num_sms() else 32


def _tc05_slices_per_cta(num_tiles: int, B: int, batch_tile: int) -> int:
    """Sample slices per CTA for pcb_lse_contract_tc05. One, unless SumLayer.tc05_slices_per_cta
    says otherwise: on HCLT-784 (B = 512) runs of 4 slices per CTA (weights copied once, the
    next slice prefetched into L2) measured no faster than one CTA per slice."""
    return SumLayer.tc05_slices_per_cta or 1


def _run_rows(tiles_np: np.ndarray, krow_np: np.ndarray) -> int:
    """32 or 8 when every tile's terms come in runs of that many consecutive source rows
    (the box height of pcb_lse_contract_tc05_ws), else 0."""
    for rr in (32, 8):
        ok = True
        for off, cnt in {(int(t[2]), int(t[3])) for t in tiles_np}:
            k = krow_np[off:off + cnt]
            idx = np.arange(cnt)
            if not np.array_equal(k, k[(idx // rr) * rr] + idx % rr):
                ok = False
                break
        if ok:
            return rr
    return 0


_MAX_CHUNK_TILES = 4096  # sub-tiles (64 KB of packed weights each, 256 MB) a layer may split its long tiles into


def _chunk_table(tiles_np: np.ndarray):
    """Tiles of more than 128 terms as consecutive chunks of at most 128 terms: chunk j holds
    terms 128 j .. of every tile that has them (same output rows; ``k_off`` advanced, which
    also advances the weights). Returns ``(table, [(start, count) per chunk])`` or None when
    every tile is short (or the split would exceed ``_MAX_CHUNK_TILES``)."""
    if not tiles_np.shape[0] or int(tiles_np[:, 3].max()) <= _SHORT_K:
        return None
    nch = -(-int(tiles_np[:, 3].max()) // _SHORT_K)
    parts, ranges, start = [], [], 0
    for j in range(nch):
        t = tiles_np[tiles_np[:, 3] > _SHORT_K * j].copy()
        t[:, 2] += _SHORT_K * j
        t[:, 3] = np.minimum(t[:, 3] - _SHORT_K * j, _SHORT_K)
        parts.append(t)
        ranges.append((start, t.shape[0]))
        start += t.shape[0]
    if start > _MAX_CHUNK_TILES:
        return None
    return np.concatenate(parts), ranges


def _ch_pack(holder: dict, key: str) -> torch.Tensor:
    """The packed-weight buffer of a long-tile chunk table, allocated on the device at first
    use (``holder[key + '_bytes']`` bytes)."""
    if holder[key] is None:
        holder[key] = torch.empty([holder[key + "_bytes"]], dtype=torch.uint8, device=holder["fw_ch" if key ==
                                  "fw_ch_pack" else "ch"].device)
    return holder[key]


def _chunk_plan(table: torch.Tensor, ranges):
    """The chunk table with each tile's output rows moved into a partials buffer (chunk j's
    rows at j * S + the row's index among the S output rows), the output row and the number
    of chunks of each of those S rows (for pcb_chunk_combine)."""
    t = table.cpu().numpy().astype(np.int64).copy()
    n = t[:, 1]
    rows_all = np.arange(int(n.sum())) + np.repeat(t[:, 0] - (np.cumsum(n) - n), n)
    rows = np.unique(rows_all)
    S = rows.shape[0]
    nch = np.zeros(S, np.int64)
    for j, (a, c) in enumerate(ranges):
        first = np.searchsorted(rows, t[a:a + c, 0])
        cover = np.arange(int(n[a:a + c].sum())) + np.repeat(first - (np.cumsum(n[a:a + c]) - n[a:a + c]), n[a:a + c])
        nch[cover] = j + 1
        t[a:a + c, 0] = j * S + first
    dev = table.device
    return dict(table=_i32(t).to(dev), dst=_i32(rows).to(dev), nch=_i32(nch).to(dev), S=S, nchunks=len(ranges))


_CHUNK_SCRATCH = dict()  # device -> FP32 partials buffer shared by the long-tile contractions
_CHUNK_SCRATCH_MAX_BYTES = 1 << 30


_CHUNK_SCRATCH_RETIRED = []  # smaller buffers replaced by a larger one: CUDA graphs captured earlier still write them


def _chunk_scratch(device, rows: int, ld: int) -> torch.Tensor:
    """A [rows, ld] view of the device's partials buffer (grown when too small; a replaced
    buffer is kept alive, since a CUDA graph captured with it still uses its address). The
    contractions that use it run one after another on the pass's stream; passes of
    different circuits on concurrent streams would share it."""
    key = (device.type, device.index)
    buf = _CHUNK_SCRATCH.get(key)
    if buf is None or buf.numel() < rows * ld:
        if buf is not None:
            _CHUNK_SCRATCH_RETIRED.append(buf)
        buf = torch.empty([rows * ld], dtype=torch.float32, device=device)
        _CHUNK_SCRATCH[key] = buf
    return buf[:rows * ld].view(rows, ld)


def _tc05_chunks(src, src2, aux, out, ld, B, pack, table, ranges, krow, mode, prec, stream, holder=None,
                 plan_key=None):
    """A contraction over tiles of any length on the tcgen05 kernels, in 128-term chunks.

    With ``SumLayer.chunk_partials`` (and a ``holder`` dict to cache the plan in), when the
    later chunks hold too few tiles to fill the GPU: every chunk of every tile in one launch,
    each writing its partial result to its own rows of a shared buffer, then
    pcb_chunk_combine (log-sum-exp for the forward, sum for element flows) into the output.
    Otherwise: one launch per chunk index, the first overwriting the output and every later
    one combining into it (pcb_lse_contract_tc05_accum)."""
    # Only where the per-chunk launches would leave SMs idle: a layer whose later chunks
    # hold enough tiles to fill the GPU pays more for the partial rows (written, then read
    # back by the combine) than it gains (PD-784: 4.44 s against 3.87 s per epoch).
    later = max((n for _, n in ranges[1:]), default=0)
    plan = None
    if SumLayer.chunk_partials and holder is not None and later * -(-B // 64) < 2 * _num_sms():
        plan = holder.get(plan_key)
        if plan is None:
            plan = _chunk_plan(table, ranges)
            holder[plan_key] = plan
        if plan["S"] * plan["nchunks"] * ld * 4 > _CHUNK_SCRATCH_MAX_BYTES:
            plan = None
    if plan is not None:
        part = _chunk_scratch(out.device, plan["S"] * plan["nchunks"], ld)
        _tc05_call(src, src2, aux, part, ld, B, pack, plan["table"], krow, mode, prec, stream)
        nat.call("pcb_chunk_combine", nat.ptr(part), ld, B, plan["S"], nat.ptr(plan["dst"]), nat.ptr(plan["nch"]),
                 nat.ptr(out), mode, stream)
        return
    for j, (a, n) in enumerate(ranges):
        t = table[a:a + n]
        pk = pack[a * _PACK_BYTES:(a + n) * _PACK_BYTES]
        _tc05_call(src, src2, aux, out, ld, B, pk, t, krow, mode, prec, stream, accum=j > 0)


def _mma(prec: int) -> int:
    """Precision form for the kernels without an E4M3 form (mma.sync, FP32, parameter flows):
    form 3 (E4M3 tcgen05 contractions) runs them in split bf16."""
    return 2 if prec == 3 else prec


def _ws_ok(ld, B, *bufs) -> bool:
    """Whether pcb_lse_contract_tc05_ws takes these buffers: whole 16-byte chunks per row."""
    return B % 4 == 0 and ld % 4 == 0 and all(b is None or b.data_ptr() % 16 == 0 for b in bufs)


def _tc05_call(src, src2, aux, out, ld, B, pack, tiles, krow, mode, prec, stream, run_rows=0, accum=False):
    """One tcgen05 contraction: the persistent warp-specialised kernel
    (pcb_lse_contract_tc05_ws, 32- or 64-sample units) or the CTA-per-slice kernel
    (pcb_lse_contract_tc05, 32 or 64 samples and 1 or 2 slices per CTA), chosen by the
    autotuner per mode, precision form, tile count and batch. ``SumLayer.tc05_ws`` forces
    (True) or excludes (False) the persistent kernel; ``SumLayer.tc05_slices_per_cta`` fixes
    the CTA-per-slice kernel's slices and its static batch tile. ``run_rows``: the tile
    table's runs of consecutive source rows (``_run_rows``; 0 excludes the persistent kernel).
    ``accum``: combine into the output (a later chunk of long tiles; static launch shape, since
    timing candidates would accumulate repeatedly)."""
    nt = tiles.size(0)
    if accum:
        nat.call("pcb_lse_contract_tc05_accum", nat.ptr(src), nat.ptr(src2), nat.ptr(aux), nat.ptr(out), ld, B,
                 nat.ptr(pack), nat.ptr(tiles), nt, nat.ptr(krow), mode, prec, _tc05_batch_tile(nt, B), 1, stream)
        return

    def run(c):
        if c[0] == "ws":
            nat.call("pcb_lse_contract_tc05_ws", nat.ptr(src), nat.ptr(src2), nat.ptr(aux), nat.ptr(out), ld, B,
                     src.size(0), out.size(0), nat.ptr(pack), nat.ptr(tiles), nt, nat.ptr(krow), mode, prec, c[1],
                     run_rows, 0,
                     stream)
        else:
            nat.call("pcb_lse_contract_tc05", nat.ptr(src), nat.ptr(src2), nat.ptr(aux), nat.ptr(out), ld, B,
                     nat.ptr(pack), nat.ptr(tiles), nt, nat.ptr(krow), mode, prec, c[0], c[1], stream)

    ws_ok = (SumLayer.tc05_ws is not False and prec != 3 and run_rows in (8, 32)
             and _ws_ok(ld, B, src, src2, aux, out))
    ws_bt = 32 if mode == 2 or nt * -(-B // 64) < _num_sms() else 64
    if SumLayer.tc05_ws and ws_ok:
        return run(("ws", ws_bt))
    bt = _tc05_batch_tile(nt, B)
    if SumLayer.tc05_slices_per_cta is not None:
        return run((bt, _tc05_slices_per_cta(nt, B, bt)))
    cands = [(bt, 1)] + [c for c in ((64, 1), (32, 1), (64, 2), (32, 2)) if c != (bt, 1)]
    if ws_ok:
        ws_c = [("ws", ws_bt), ("ws", 96 - ws_bt)]
        # static default: the persistent kernel once the layer has a unit per SM
        cands = ws_c + cands if nt * -(-B // ws_bt) >= _num_sms() else cands + ws_c
    run(TUNER.pick(("tc05", mode, prec, nt, B), cands, run))


def _short_tile(key, num_tiles: int, tile_rows: int, B: int, fused: bool, run) -> None:
    """Launch ``run(batch_tile)`` of a single-stage contraction with the autotuned samples per
    CTA (16, 32 or 64; at most 32 with a fused product layer); ``SumLayer.short_batch_tile``
    fixes it, 0 keeps the static rule (_short_batch_tile)."""
    static = _short_batch_tile(num_tiles, tile_rows, B, fused)
    fixed = SumLayer.short_batch_tile
    if fixed is not None:
        return run(static if fixed == 0 else (min(fixed, 32) if fused else fixed))
    cands = [static] + [t for t in ((16, 32) if fused else (16, 32, 64)) if t != static]
    run(TUNER.pick(("short",) + tuple(key) + (num_tiles, tile_rows, B, fused), cands, run))


_SCRATCH = {}


def _pflow_scratch(like: torch.Tensor) -> torch.Tensor:
    """A buffer shaped like the parameter flows for timing accumulating candidates."""
    key = (like.device, like.numel())
    t = _SCRATCH.get(key)
    if t is None:
        t = torch.zeros_like(like)
        _SCRATCH[key] = t
    return t


def _rows_vec4(tiles: np.ndarray, kw: np.ndarray, rpb: int, w_stride: int) -> bool:
    """Weights of 4 consecutive rows are consecutive and 16-byte aligned (forward tables)."""
    return (w_stride == 1 and rpb % 4 == 0 and bool(np.all(kw % 4 == 0)) and bool(np.all(tiles[:, 4] % 4 == 0))
            and bool(np.all(tiles[:, 6] % 4 == 0)))


def _terms_vec4(tiles: np.ndarray, kw: np.ndarray, w_stride: int) -> bool:
    """Weights of 4 consecutive terms (aligned groups of each tile) are consecutive and
    16-byte aligned (element-flow tables)."""
    if w_stride % 4 or not np.all(tiles[:, 4] % 4 == 0) or not np.all(tiles[:, 6] % 4 == 0):
        return False
    for k_off, k_cnt in zip(tiles[:, 2].tolist(), tiles[:, 3].tolist()):
        seg = kw[k_off:k_off + k_cnt]
        full = (k_cnt // 4) * 4
        g = seg[:full].reshape(-1, 4)
        if g.size and (np.any(g[:, 0] % 4) or np.any(g - g[:, :1] != np.arange(4)[None, :])):
            return False
    return True


def _merge_chains(starts, klists, wlists, flists, rpb: int):
    """Group consecutive blocks into tiles that share one set of contraction terms.

    Blocks ``i .. i + c - 1`` merge when their term lists (``klists``) are identical, their
    first rows are ``rpb`` apart, and their weight (and flow) offsets differ by one constant
    stride; at most ``_MAX_ROWS`` rows per chain. Returns ``(first, count, w_stride, f_stride)``.
    In a structured circuit every region (the node blocks of one sum vector over one
    product vector) becomes one chain.
    """
    chains = []
    n = len(starts)
    max_blocks = max(1, _MAX_ROWS // rpb)
    i = 0
    while i < n:
        j = i + 1
        gs_w = gs_f = 0
        while j < n and j - i < max_blocks:
            if starts[j] != starts[j - 1] + rpb or klists[j].shape != klists[i].shape or \
                    not np.array_equal(klists[j], klists[i]) or klists[i].size == 0:
                break
            dw = wlists[j] - wlists[j - 1]
            if not np.all(dw == dw[0]) or (j - i > 1 and int(dw[0]) != gs_w):
                break
            if flists is not None:
                df = flists[j] - flists[j - 1]
                if not np.all(df == df[0]) or (j - i > 1 and int(df[0]) != gs_f):
                    break
                if j - i == 1:
                    gs_f = int(df[0])
            if j - i == 1:
                gs_w = int(dw[0])
            j += 1
        chains.append((i, j - i, gs_w, gs_f))
        i = j
    return chains


class Layer:
    propagation_alg_mapping = {"LL": 0, "MPE": 1, "GeneralLL": 2}

    def __init__(self, nodes):
        self.nodes = list(nodes)
        self.scopes = []
        for ns in self.nodes:
            if ns.scope not in self.scopes:
                self.scopes.append(ns.scope)
        self.device = torch.device("cpu")
        self._dev = {}

    def is_sum(self):
        return False

    def is_prod(self):
        return False

    def is_input(self):
        return False

    def provided(self, name):
        return hasattr(self, name) and getattr(self, name) is not None

    def _desc(self, device: torch.device):
        key = (device.type, device.index)
        d = self._dev.get(key)
        if d is None:
            def mv(v):
                if isinstance(v, torch.Tensor):
                    return v.to(device)
                if isinstance(v, (list, tuple)):
                    return type(v)(mv(x) for x in v)
                if isinstance(v, dict):
                    return {kk: mv(vv) for kk, vv in v.items()}
                return v
            d = {k: mv(v) for k, v in self._host_desc().items()}
            self._dev[key] = d
        return d

    def _host_desc(self):
        raise NotImplementedError()

    # ---- partial evaluation (layer.py:38-75): only the node vectors whose scope is one of the
    # given scopes are evaluated; the other rows keep their values
    _fw_partial = None
    _bk_partial = None

    @staticmethod
    def _ranges(node_vectors, scopes) -> list:
        """Output-row ranges of the node vectors whose scope is in ``scopes``."""
        return [ns._output_ind_range for ns in node_vectors if ns.scope in scopes]

    @staticmethod
    def _keep_rows(first_rows, ranges) -> np.ndarray:
        first_rows = np.asarray(first_rows, np.int64).reshape(-1)
        keep = np.zeros(first_rows.shape[0], dtype=bool)
        for lo, hi in ranges:
            keep |= (first_rows >= lo) & (first_rows < hi)
        return keep

    def _partial(self, which: str, device: torch.device):
        """The device copy of a partial-evaluation table set (``_fw_partial`` / ``_bk_partial``)."""
        host = self._fw_partial if which == "fw" else self._bk_partial
        if host is None:
            return None
        key = (which, device.type, device.index, id(host))
        cache = self.__dict__.setdefault("_partial_dev", {})
        t = cache.get(key)
        if t is None:
            def mv(v):
                if isinstance(v, torch.Tensor):
                    return v.to(device)
                if isinstance(v, list):
                    return [mv(x) for x in v]
                if isinstance(v, dict):
                    return {kk: mv(vv) for kk, vv in v.items()}
                return v
            t = mv(host)
            cache.clear()
            cache[key] = t
        return t

    def disable_partial_evaluation(self, forward: bool = True, backward: bool = True):
        if forward:
            self._fw_partial = None
        if backward:
            self._bk_partial = None

    def to(self, device):
        device = torch.device(device)
        for name in self._tensor_lists:
            setattr(self, name, [t.to(device) for t in getattr(self, name)])
        self.device = device
        return self


class SumLayer(Layer):
    """A layer of sum node vectors with the same block size.

    Precision forms of the sum contractions: plain FP32 (``force_use_fp32``) or the
    tensor-core form. ``SumLayer.bf16_form`` selects the latter's variant: 2 (default)
    splits both operands into bf16 hi + lo parts (three MMAs, FP32-like accuracy), 1 uses
    single bf16 operands, 3 runs the tcgen05 contractions (layers of at least
    ``tc05_min_tiles`` tiles, forward and element flows) in E4M3 with per-row weight scales
    and the rest in split bf16.
    """

    bf16_form = 2
    short_kernels = True  # single-stage kernels for tiles of <= 128 terms
    tc05_min_tiles = 6    # layers with at least this many tiles use the tcgen05 kernels (BF16 forms)
    tc05_slices_per_cta = None  # sample slices per tcgen05 CTA (None: one)
    tc05_ws = None        # persistent warp-specialised tcgen05 kernel: None autotuned, True forced, False off
    tc05_long = True      # tiles of more than 128 terms as accumulating tcgen05 chunks (BF16 / E4M3 forms)
    chunk_partials = True  # all chunks of a layer in one launch into partial rows, then pcb_chunk_combine
    # The single-stage kernels of small layers read pre-packed weights too (the circuit packs
    # all layers' weights in one launch per pass, so the kernels skip their own conversion).
    pack_short_weights = True
    # Children per parameter-flow tile (32, 64 or 128): with all children of a region in one
    # tile, its node rows are exponentiated once per sample slice instead of once per chunk.
    # (None: chosen per layer shape by the autotuner; the static default is 64.)
    pflow_tile_children = None
    # BF16 parameter flows on the tcgen05 tensor cores (accumulators in tensor memory) or on
    # the warp-level mma.sync kernel (False); None: chosen by the autotuner.
    pflow_tc05 = None
    # Samples per CTA of the single-stage kernels: None autotuned, 0 the static rule, else fixed.
    short_batch_tile = None

    _tensor_lists = ("partitioned_nids", "partitioned_cids", "partitioned_pids", "partitioned_pfids",
                     "partitioned_chids", "partitioned_parids", "partitioned_parpids")

    def __init__(self, nodes: Sequence, global_nid_start: int, global_pid_start: int, global_pfid_start: int,
                 node2tiednodes: dict, layer_sparsity_tol: Optional[float] = None,
                 max_num_partitions: Optional[int] = None, max_tied_ns_per_parflow_block: int = 8, **kwargs):
        super().__init__(nodes)
        if len(self.nodes) == 0 or len(set(self.nodes)) != len(self.nodes):
            raise ValueError("a sum layer needs distinct node vectors")
        self.block_size = self.nodes[0].block_size
        for ns in self.nodes:
            if ns.block_size != self.block_size:
                raise ValueError("`block_size` of nodes in the same layer must be identical.")
        c = compile_sum_layer(self.nodes, global_nid_start, global_pid_start, global_pfid_start, node2tiednodes,
                              layer_sparsity_tol, max_num_partitions, max_tied_ns_per_parflow_block)
        self.num_nodes = c["num_nodes"]
        self.num_edges = c["num_edges"]
        self._layer_nid_range = c["nid_range"]
        self._layer_pid_range = c["pid_range"]
        self._layer_pfid_range = c["pfid_range"]
        self.partitioned_nids, self.partitioned_cids = c["nids"], c["cids"]
        self.partitioned_pids, self.partitioned_pfids = c["pids"], c["pfids"]
        self.partitioned_chids, self.partitioned_parids = c["chids"], c["parids"]
        self.partitioned_parpids = c["parpids"]
        self.cs_block_sizes = c["cs_block_sizes"]
        self.num_fw_partitions = len(self.partitioned_nids)
        self.num_bk_partitions = len(self.partitioned_chids)
        self._has_tied = any(ns.is_tied() for ns in self.nodes)

    @property
    def num_parameters(self):
        return self._layer_pid_range[1] - self._layer_pid_range[0]

    @property
    def num_param_flows(self):
        return self._layer_pfid_range[1] - self._layer_pfid_range[0]

    @property
    def nid_range(self):
        return self._layer_nid_range

    def is_sum(self):
        return True

    # ---- kernel descriptors ----
    def _host_desc(self):
        bs = self.block_size
        # forward blocks (shared with sampling and parameter flows)
        blk_nid, blk_koff, blk_kcnt, krow, kw, kpf = [], [], [], [], [], []
        off = 0
        for nids, cids, pids, pfids in zip(self.partitioned_nids, self.partitioned_cids, self.partitioned_pids,
                                           self.partitioned_pfids):
            n_np, c_np, p_np, f_np = nids.cpu().numpy(), cids.cpu().numpy(), pids.cpu().numpy(), pfids.cpu().numpy()
            for l in range(n_np.shape[0]):
                real = c_np[l] != 0
                cnt = int(real.sum())
                if not np.all(real[:cnt]):
                    raise RuntimeError("sum layer children are not a prefix of the padded row")
                blk_nid.append(int(n_np[l]))
                blk_koff.append(off)
                blk_kcnt.append(cnt)
                krow.append(c_np[l, :cnt])
                kw.append(p_np[l, :cnt])
                kpf.append(f_np[l, :cnt])
                off += cnt
        chains = _merge_chains(blk_nid, krow, kw, kpf, bs)
        krow_c = np.concatenate(krow) if krow else np.zeros([0], np.int64)
        kw_c = np.concatenate(kw) if kw else np.zeros([0], np.int64)
        kpf_c = np.concatenate(kpf) if kpf else np.zeros([0], np.int64)
        blk_nid = np.asarray(blk_nid, np.int64)
        blk_koff = np.asarray(blk_koff, np.int64)
        blk_kcnt = np.asarray(blk_kcnt, np.int64)

        fw_tiles, pf_tiles, pf_tiles32, pf_tiles128 = [], [], [], []
        for g, cnt, gs_w, gs_f in chains:
            rows = cnt * bs
            for i0 in range(0, rows, _MAX_ROWS):
                nr = min(_MAX_ROWS, rows - i0)
                fw_tiles.append((blk_nid[g] + i0, nr, blk_koff[g], blk_kcnt[g], i0, 0, gs_w, 0))
                for kc, lst in ((64, pf_tiles), (32, pf_tiles32), (128, pf_tiles128)):
                    for k0 in range(0, int(blk_kcnt[g]), kc):
                        lst.append((blk_nid[g] + i0, nr, blk_koff[g] + k0, min(kc, int(blk_kcnt[g]) - k0), i0,
                                    gs_w, gs_f, 0))
        fw_tm = _tile_rows(max(t[1] for t in fw_tiles)) if fw_tiles else 1
        node2blk = np.zeros([self.num_nodes // bs], np.int64)
        node2blk[(blk_nid - self._layer_nid_range[0]) // bs] = np.arange(blk_nid.shape[0])

        # element-flow tiles, one launch per child block size
        el_groups = []
        for cbs in sorted(set(self.cs_block_sizes)):
            starts, klist, wlist = [], [], []
            for chids, parids, parpids, pcbs in zip(self.partitioned_chids, self.partitioned_parids,
                                                    self.partitioned_parpids, self.cs_block_sizes):
                if pcbs != cbs:
                    continue
                ch_np, pa_np, pp_np = chids.cpu().numpy(), parids.cpu().numpy(), parpids.cpu().numpy()
                for l in range(ch_np.shape[0]):
                    npar = int((pa_np[l] != 0).sum())
                    starts.append(int(ch_np[l]))
                    klist.append((pa_np[l, :npar][:, None] + np.arange(bs)[None, :]).reshape(-1))
                    wlist.append((pp_np[l, :npar][:, None] + np.arange(bs)[None, :]).reshape(-1))
            if not starts:
                continue
            ech = _merge_chains(starts, klist, wlist, None, cbs)
            offs = np.zeros(len(klist) + 1, np.int64)
            offs[1:] = np.cumsum([k.shape[0] for k in klist])
            tiles = []
            for g, cnt, gs_w, _ in ech:
                rows = cnt * cbs
                for j0 in range(0, rows, _MAX_ROWS):
                    nr = min(_MAX_ROWS, rows - j0)
                    tiles.append((starts[g] + j0, nr, offs[g], klist[g].shape[0], j0 * bs, starts[g] + j0, gs_w, 0))
            tiles_np = np.asarray(tiles, np.int64).reshape(-1, 8)
            kw_np = np.concatenate(wlist)
            ech_t = _chunk_table(tiles_np)
            el_groups.append(dict(
                ch=None if ech_t is None else _i32(ech_t[0]), ch_ranges=None if ech_t is None else ech_t[1],
                ch_pack=None, ch_pack_bytes=0 if ech_t is None else ech_t[0].shape[0] * _PACK_BYTES,
                cbs=cbs, tm=_tile_rows(max(t[1] for t in tiles)), tiles=_i32(tiles_np),
                krow=_i32(np.concatenate(klist)), kw=_i32(kw_np),
                short=int(tiles_np[:, 3].max()) <= _SHORT_K,
                wlayout=2 if _terms_vec4(tiles_np, kw_np, bs) else 0,
                run=_run_rows(tiles_np, np.concatenate(klist)),
                pack=torch.empty([tiles_np.shape[0] * _PACK_BYTES], dtype=torch.uint8)))

        fw_np = np.asarray(fw_tiles, np.int64).reshape(-1, 8)
        fch = _chunk_table(fw_np)
        return dict(
            fw_ch=None if fch is None else _i32(fch[0]), fw_ch_ranges=None if fch is None else fch[1],
            fw_ch_pack=None, fw_ch_pack_bytes=0 if fch is None else fch[0].shape[0] * _PACK_BYTES,
            fw_tiles=_i32(fw_np), fw_tm=fw_tm, fw_run=_run_rows(fw_np, krow_c),
            fw_short=bool(fw_np.shape[0]) and int(fw_np[:, 3].max()) <= _SHORT_K,
            fw_wlayout=1 if (fw_np.shape[0] and _rows_vec4(fw_np, kw_c, bs, 1)) else 0,
            fw_pack=torch.empty([fw_np.shape[0] * _PACK_BYTES], dtype=torch.uint8),
            krow=_i32(krow_c), kw=_i32(kw_c), kpf=_i32(kpf_c),
            blk_nid=_i32(blk_nid), blk_koff=_i32(blk_koff), blk_kcnt=_i32(blk_kcnt), node2blk=_i32(node2blk),
            min_kcnt=int(blk_kcnt.min()) if blk_kcnt.size else 0,
            pf_tiles=_i32(np.asarray(pf_tiles, np.int64).reshape(-1, 8)),
            pf_tiles32=_i32(np.asarray(pf_tiles32, np.int64).reshape(-1, 8)),
            pf_tiles128=_i32(np.asarray(pf_tiles128, np.int64).reshape(-1, 8)),
            el_groups=el_groups,
        )

    def enable_partial_evaluation(self, fw_scopes=None, bk_scopes=None):
        """Tile subsets for the node vectors with the given scopes: forward tiles of those
        sum vectors; backward element-flow tiles of their product children (rows = elements)
        and parameter-flow tiles of the sum vectors."""
        d = self._host_desc()
        if fw_scopes is not None:
            rng = self._ranges(self.nodes, set(fw_scopes))
            t = d["fw_tiles"]
            self._fw_partial = dict(tiles=t[torch.from_numpy(self._keep_rows(t[:, 0].numpy(), rng))].contiguous())
        if bk_scopes is not None:
            scopes = set(bk_scopes)
            rng = self._ranges(self.nodes, scopes)
            prods = []
            for ns in self.nodes:
                for cs in ns.chs:
                    if cs not in prods:
                        prods.append(cs)
            erng = self._ranges(prods, scopes)
            el = [eg["tiles"][torch.from_numpy(self._keep_rows(eg["tiles"][:, 0].numpy(), erng))].contiguous()
                  for eg in d["el_groups"]]
            pt = d["pf_tiles"]
            self._bk_partial = dict(el=el, pf=pt[torch.from_numpy(self._keep_rows(pt[:, 0].numpy(), rng))].contiguous())

    # ---- forward / backward ----
    def _use_bf16(self, d, B, force_use_bf16, force_use_fp32):
        if force_use_bf16 and force_use_fp32:
            raise ValueError("`force_use_bf16` and `force_use_fp32` are exclusive")
        eligible = d["fw_tm"] >= 16
        if force_use_bf16:
            return eligible
        if force_use_fp32:
            return False
        # Reference default: tensor-core contraction when the tiles are at least 16 wide
        # (sum_layer.py:871-880).
        return eligible and d["min_kcnt"] >= 16 and B >= 16

    def _fw_tc05(self, d, B, force_use_bf16, force_use_fp32):
        """Precision form of the forward and whether it runs on the tcgen05 kernel."""
        prec = SumLayer.bf16_form if self._use_bf16(d, B, force_use_bf16, force_use_fp32) else 0
        return prec, prec > 0 and d["fw_short"] and d["fw_tiles"].size(0) >= SumLayer.tc05_min_tiles

    def _el_prec(self, eg, B, force_use_fp32):
        return SumLayer.bf16_form if (not force_use_fp32 and eg["tm"] >= 16 and B >= 16) else 0

    def _fw_long(self, d, prec):
        """Whether the forward runs its tiles of more than 128 terms as tcgen05 chunks."""
        return (prec > 0 and SumLayer.tc05_long and not d["fw_short"] and d["fw_ch"] is not None
                and d["fw_ch"].size(0) >= SumLayer.tc05_min_tiles)

    def _el_long(self, eg, prec):
        return (prec > 0 and SumLayer.tc05_long and not eg["short"] and eg["ch"] is not None
                and eg["ch"].size(0) >= SumLayer.tc05_min_tiles)

    def _el_tc05(self, eg, prec):
        return prec > 0 and eg["short"] and eg["tiles"].size(0) >= SumLayer.tc05_min_tiles

    def runs_single_stage(self, device: torch.device, B: int, force_use_bf16: bool = False,
                          force_use_fp32: bool = False, backward: bool = False) -> bool:
        """Whether the forward (or every element-flow launch) runs pcb_lse_contract_short with
        these settings, so that a product layer can be fused into it."""
        d = self._desc(device)
        if not SumLayer.short_kernels:
            return False
        if not backward:
            return d["fw_short"] and not self._fw_tc05(d, B, force_use_bf16, force_use_fp32)[1]
        return all(eg["short"] and not self._el_tc05(eg, self._el_prec(eg, B, force_use_fp32))
                   for eg in d["el_groups"])

    def forward_pack_job(self, device: torch.device, B: int, force_use_bf16: bool = False,
                         force_use_fp32: bool = False):
        """``(tiles, kw, packed, rows_per_block, w_stride, format)`` of the forward weights this
        layer reads packed (tcgen05 layers; also the single-stage ones with
        ``pack_short_weights``), or None; format 1: E4M3 (precision form 3 on tcgen05)."""
        d = self._desc(device)
        prec, tc05 = self._fw_tc05(d, B, force_use_bf16, force_use_fp32)
        if tc05 or (SumLayer.pack_short_weights and prec > 0 and d["fw_short"]):
            return (d["fw_tiles"], d["kw"], d["fw_pack"], self.block_size, 1, 1 if (tc05 and prec == 3) else 0)
        if self._fw_long(d, prec):
            return (d["fw_ch"], d["kw"], _ch_pack(d, "fw_ch_pack"), self.block_size, 1, 1 if prec == 3 else 0)
        return None

    def flow_pack_jobs(self, device: torch.device, B: int, force_use_fp32: bool = False):
        """Pack jobs (see forward_pack_job) of the element-flow weights this layer reads packed."""
        d = self._desc(device)
        jobs = []
        for eg in d["el_groups"]:
            prec = self._el_prec(eg, B, force_use_fp32)
            tc05 = self._el_tc05(eg, prec)
            if tc05 or (SumLayer.pack_short_weights and prec > 0 and eg["short"]):
                jobs.append((eg["tiles"], eg["kw"], eg["pack"], eg["cbs"], self.block_size,
                             1 if (tc05 and prec == 3) else 0))
            elif self._el_long(eg, prec):
                jobs.append((eg["ch"], eg["kw"], _ch_pack(eg, "ch_pack"), eg["cbs"], self.block_size, 1 if prec == 3 else 0))
        return jobs

    @staticmethod
    def _run_pack_job(params: torch.Tensor, job) -> None:
        t, kw, packed, rpb, w_stride, fmt = job
        nat.call("pcb_pack_weights_fp8" if fmt == 1 else "pcb_pack_weights", nat.ptr(params), nat.ptr(t), t.size(0),
                 rpb, nat.ptr(kw), w_stride, nat.ptr(packed), nat.stream())

    def pack_forward_weights(self, params: torch.Tensor, B: int, force_use_bf16: bool = False,
                             force_use_fp32: bool = False) -> bool:
        """Pack the weights the forward reads packed (on the current stream); returns whether
        this layer uses them. ``forward(..., _weights_packed=True)`` then skips the pack."""
        job = self.forward_pack_job(params.device, B, force_use_bf16, force_use_fp32)
        if job is not None:
            self._run_pack_job(params, job)
        return job is not None

    def pack_flow_weights(self, params: torch.Tensor, B: int, force_use_fp32: bool = False) -> bool:
        """Pack the element-flow weights this layer reads packed (see pack_forward_weights)."""
        jobs = self.flow_pack_jobs(params.device, B, force_use_fp32)
        for job in jobs:
            self._run_pack_job(params, job)
        return bool(jobs)

    @staticmethod
    def _alg(propagation_alg: str, kwargs) -> tuple:
        """(algorithm id, alpha) of a propagation algorithm (layer.py:11-15, 89-97)."""
        if propagation_alg not in Layer.propagation_alg_mapping:
            raise ValueError(f"Unknown propagation algorithm {propagation_alg}.")
        alpha = 0.0
        if propagation_alg == "GeneralLL":
            if "alpha" not in kwargs:
                raise ValueError("Argument `alpha` should be provided for the `GeneralLL` propagation algorithm.")
            alpha = float(kwargs["alpha"])
            if not alpha > 0.0:
                raise ValueError("`alpha` must be positive")
        return Layer.propagation_alg_mapping[propagation_alg], alpha

    def forward(self, node_mars: torch.Tensor, element_mars: torch.Tensor, params: torch.Tensor,
                force_use_bf16: bool = False, force_use_fp32: bool = False, propagation_alg: str = "LL",
                _weights_packed: bool = False, **kwargs) -> None:
        if params.dim() != 1:
            raise ValueError("Expecting a 1D `params`.")
        d = self._desc(node_mars.device)
        B = node_mars.size(1)
        ld = node_mars.stride(0)
        if element_mars.stride(0) != ld or node_mars.stride(1) != 1 or element_mars.stride(1) != 1:
            raise ValueError("node_mars and element_mars must share a row-major layout")
        if propagation_alg != "LL":
            # MPE / GeneralLL: the FP32 kernel of these modes (pcb_sum_fwd_generic)
            alg, alpha = self._alg(propagation_alg, kwargs)
            t = d["fw_tiles"]
            nat.call("pcb_sum_fwd_generic", nat.ptr(element_mars), nat.ptr(node_mars), ld, B, nat.ptr(params),
                     nat.ptr(t), t.size(0), self.block_size, nat.ptr(d["krow"]), nat.ptr(d["kw"]), 1, alg, alpha,
                     nat.stream())
            return
        prec, tc05 = self._fw_tc05(d, B, force_use_bf16, force_use_fp32)
        t = d["fw_tiles"]
        st = nat.stream()
        part = self._partial("fw", node_mars.device)
        if part is not None:
            # a subset of the tiles: the kernels that read the weights directly (the packed
            # weights are indexed by the full table's tile numbers)
            t = part["tiles"]
            if t.size(0) == 0:
                return
            if d["fw_short"] and SumLayer.short_kernels:
                nat.call("pcb_lse_contract_short", nat.ptr(element_mars), nat.ptr(None), nat.ptr(None),
                         nat.ptr(node_mars), ld, B, nat.ptr(params), nat.ptr(t), t.size(0), d["fw_tm"],
                         self.block_size, nat.ptr(d["krow"]), nat.ptr(d["kw"]), 1, 0, _mma(prec), nat.ptr(None),
                         d["fw_wlayout"], _short_batch_tile(t.size(0), d["fw_tm"], B), nat.ptr(None), st)
            else:
                nat.call("pcb_lse_contract", nat.ptr(element_mars), nat.ptr(None), nat.ptr(None), nat.ptr(node_mars),
                         ld, B, nat.ptr(params), nat.ptr(t), t.size(0), d["fw_tm"], self.block_size,
                         nat.ptr(d["krow"]), nat.ptr(d["kw"]), 1, 0, _mma(prec), st)
            return
        if tc05:
            if not _weights_packed:
                self.pack_forward_weights(params, B, force_use_bf16, force_use_fp32)
                _weights_packed = True
            _tc05_call(element_mars, None, None, node_mars, ld, B, d["fw_pack"], t, d["krow"], 0, prec, st,
                       d["fw_run"])
            return
        if self._fw_long(d, prec):
            if not _weights_packed:
                self.pack_forward_weights(params, B, force_use_bf16, force_use_fp32)
            _tc05_chunks(element_mars, None, None, node_mars, ld, B, _ch_pack(d, "fw_ch_pack"), d["fw_ch"], d["fw_ch_ranges"],
                         d["krow"], 0, prec, st, holder=d, plan_key="fw_ch_plan")
            return
        prec = _mma(prec)
        # _fuse_fw = (term_children, element values out): the product layer below is fused in
        # (the terms are sums of node rows; the element values are written as a side output)
        fuse = kwargs.get("_fuse_fw")
        if d["fw_short"] and SumLayer.short_kernels:
            packed = d["fw_pack"] if (_weights_packed and prec > 0 and SumLayer.pack_short_weights) else None
            fusion = nat.short_fusion(fuse[0], fuse[1]) if fuse is not None else nat.ptr(None)
            st = nat.stream()

            def run(bt):
                nat.call("pcb_lse_contract_short", nat.ptr(element_mars if fuse is None else node_mars),
                         nat.ptr(None), nat.ptr(None), nat.ptr(node_mars), ld, B, nat.ptr(params), nat.ptr(t),
                         t.size(0), d["fw_tm"], self.block_size, nat.ptr(d["krow"]), nat.ptr(d["kw"]), 1, 0, prec,
                         nat.ptr(packed), d["fw_wlayout"], bt, fusion, st)

            _short_tile((0, prec, packed is not None), t.size(0), d["fw_tm"], B, fuse is not None, run)
            return
        if fuse is not None:
            raise RuntimeError("a fused product layer needs the single-stage sum kernel")
        nat.call("pcb_lse_contract", nat.ptr(element_mars), nat.ptr(None), nat.ptr(None), nat.ptr(node_mars), ld, B,
                 nat.ptr(params), nat.ptr(t), t.size(0), d["fw_tm"], self.block_size, nat.ptr(d["krow"]),
                 nat.ptr(d["kw"]), 1, 0, prec, nat.stream())

    __call__ = forward

    def backward(self, node_flows: torch.Tensor, element_flows: torch.Tensor, node_mars: torch.Tensor,
                 element_mars: torch.Tensor, params: torch.Tensor, param_flows: Optional[torch.Tensor] = None,
                 allow_modify_flows: bool = False, propagation_alg: str = "LL", logspace_flows: bool = False,
                 negate_pflows: bool = False, accumulate_ch_flows: bool = False, allow_neg_flows: bool = False,
                 force_use_fp32: bool = False, _weights_packed: bool = False, **kwargs) -> None:
        if allow_modify_flows and logspace_flows:
            raise ValueError("`allow_modify_flows` should be set to `False` when using `logspace_flows`.")
        if accumulate_ch_flows and logspace_flows:
            raise ValueError("`accumulate_ch_flows` should be set to `False` when using `logspace_flows`.")
        if allow_neg_flows and (logspace_flows or propagation_alg != "LL"):
            raise ValueError("`allow_neg_flows` needs linear LL flows")
        d = self._desc(node_mars.device)
        B = node_mars.size(1)
        ld = node_mars.stride(0)
        for t in (node_flows, element_flows, element_mars):
            if t.stride(0) != ld or t.stride(1) != 1:
                raise ValueError("node/element mars/flows must share a row-major layout")
        if propagation_alg != "LL" or logspace_flows or negate_pflows or accumulate_ch_flows or allow_neg_flows:
            if allow_modify_flows:
                raise ValueError("these flow modes read unmodified node flows: pass allow_modify_flows=False")
            self._backward_generic(node_flows, element_flows, node_mars, element_mars, params, param_flows,
                                   propagation_alg, logspace_flows, negate_pflows, accumulate_ch_flows, kwargs)
            return
        part = self._partial("bk", node_mars.device)
        if part is not None:
            self._backward_partial(part, node_flows, element_flows, node_mars, element_mars, params, param_flows,
                                   force_use_fp32)
            return
        if allow_modify_flows and not kwargs.get("_flows_modified"):
            nat.call("pcb_modify_flows", nat.ptr(node_flows), nat.ptr(node_mars), ld, B, self._layer_nid_range[0],
                     self._layer_nid_range[1], nat.stream())
        skip = kwargs.get("_pflow_skip")
        if skip and id(self) in skip:  # the circuit launches them once for this layer's tied set
            param_flows = None
        # The parameter flows only read this layer's node flows / mars and its children's element
        # values, so with a side stream they run concurrently with the element flows (and with
        # everything the caller issues next on the current stream).
        pflow_stream = kwargs.get("_pflow_stream")
        ready = None
        if param_flows is not None and pflow_stream is not None:
            ready = torch.cuda.Event()
            ready.record()
        # element flows
        if not _weights_packed and any(self._el_tc05(eg, p) or self._el_long(eg, p)
                                       for eg in d["el_groups"] for p in (self._el_prec(eg, B, force_use_fp32),)):
            self.pack_flow_weights(params, B, force_use_fp32)
            _weights_packed = True
        for eg in d["el_groups"]:
            et = eg["tiles"]
            prec = self._el_prec(eg, B, force_use_fp32)
            if self._el_tc05(eg, prec):
                st = nat.stream()
                _tc05_call(node_flows, None if allow_modify_flows else node_mars, element_mars, element_flows, ld, B,
                           eg["pack"], et, eg["krow"], 1 if allow_modify_flows else 2, prec, st, eg["run"])
                continue
            if self._el_long(eg, prec):
                _tc05_chunks(node_flows, None if allow_modify_flows else node_mars, element_mars, element_flows, ld,
                             B, _ch_pack(eg, "ch_pack"), eg["ch"], eg["ch_ranges"], eg["krow"], 1 if allow_modify_flows else 2,
                             prec, nat.stream(), holder=eg, plan_key="ch_plan")
                continue
            prec = _mma(prec)
            if eg["short"] and SumLayer.short_kernels:
                packed = eg["pack"] if (_weights_packed and prec > 0 and SumLayer.pack_short_weights) else None
                # _fuse_bw = out_children: the product layer below is fused in (each element's
                # flow goes straight to the node-flow rows of its children)
                fuse = kwargs.get("_fuse_bw")
                if fuse is not None and allow_modify_flows:
                    raise RuntimeError("a fused product layer needs unmodified node flows")
                mode = 1 if allow_modify_flows else 2
                fz = nat.short_fusion(out_children=fuse) if fuse is not None else nat.ptr(None)
                st = nat.stream()

                def run(bt, eg=eg, et=et, packed=packed, prec=prec, mode=mode, fuse=fuse, fz=fz, st=st):
                    nat.call("pcb_lse_contract_short", nat.ptr(node_flows),
                             nat.ptr(None if allow_modify_flows else node_mars), nat.ptr(element_mars),
                             nat.ptr(element_flows if fuse is None else node_flows), ld, B, nat.ptr(params),
                             nat.ptr(et), et.size(0), eg["tm"], eg["cbs"], nat.ptr(eg["krow"]), nat.ptr(eg["kw"]),
                             self.block_size, mode, prec, nat.ptr(packed), eg["wlayout"], bt, fz, st)

                _short_tile((mode, prec, packed is not None), et.size(0), eg["tm"], B, fuse is not None, run)
                continue
            if kwargs.get("_fuse_bw") is not None:
                raise RuntimeError("a fused product layer needs the single-stage element-flow kernel")
            nat.call("pcb_lse_contract", nat.ptr(node_flows), nat.ptr(None if allow_modify_flows else node_mars),
                     nat.ptr(element_mars), nat.ptr(element_flows), ld, B, nat.ptr(params), nat.ptr(et), et.size(0),
                     eg["tm"], eg["cbs"], nat.ptr(eg["krow"]), nat.ptr(eg["kw"]), self.block_size,
                     1 if allow_modify_flows else 2, prec, nat.stream())
        # parameter flows
        if param_flows is not None:
            if ready is not None:
                pflow_stream.wait_event(ready)
            with torch.cuda.stream(pflow_stream if ready is not None else torch.cuda.current_stream()):
                self.param_flows_only(node_flows, node_mars, element_mars, params, param_flows,
                                      allow_modify_flows=allow_modify_flows, force_use_fp32=force_use_fp32)

    def _backward_partial(self, part, node_flows, element_flows, node_mars, element_mars, params, param_flows,
                          force_use_fp32):
        """Element flows of the selected elements and parameter flows of the selected nodes,
        on the kernels that read the weights directly (unmodified node flows)."""
        d = self._desc(node_mars.device)
        B = node_mars.size(1)
        ld = node_mars.stride(0)
        st = nat.stream()
        for eg, et in zip(d["el_groups"], part["el"]):
            if et.size(0) == 0:
                continue
            prec = _mma(self._el_prec(eg, B, force_use_fp32))
            if eg["short"] and SumLayer.short_kernels:
                nat.call("pcb_lse_contract_short", nat.ptr(node_flows), nat.ptr(node_mars), nat.ptr(element_mars),
                         nat.ptr(element_flows), ld, B, nat.ptr(params), nat.ptr(et), et.size(0), eg["tm"], eg["cbs"],
                         nat.ptr(eg["krow"]), nat.ptr(eg["kw"]), self.block_size, 2, prec, nat.ptr(None),
                         eg["wlayout"], _short_batch_tile(et.size(0), eg["tm"], B), nat.ptr(None), st)
            else:
                nat.call("pcb_lse_contract", nat.ptr(node_flows), nat.ptr(node_mars), nat.ptr(element_mars),
                         nat.ptr(element_flows), ld, B, nat.ptr(params), nat.ptr(et), et.size(0), eg["tm"], eg["cbs"],
                         nat.ptr(eg["krow"]), nat.ptr(eg["kw"]), self.block_size, 2, prec, st)
        pt = part["pf"]
        if param_flows is not None and pt.size(0) > 0:
            prec = 0 if force_use_fp32 or B < 16 else _mma(SumLayer.bf16_form)
            nat.call("pcb_sum_pflows", nat.ptr(node_flows), nat.ptr(node_mars), nat.ptr(element_mars), ld, B,
                     nat.ptr(params), nat.ptr(param_flows), nat.ptr(pt), pt.size(0), self.block_size,
                     nat.ptr(d["krow"]), nat.ptr(d["kw"]), nat.ptr(d["kpf"]), 0, 1 if self._has_tied else 0, 64, prec, st)

    def _backward_generic(self, node_flows, element_flows, node_mars, element_mars, params, param_flows,
                          propagation_alg, logspace_flows, negate_pflows, accumulate_ch_flows, kwargs):
        """Element and parameter flows of the MPE / GeneralLL algorithms, of log-space flows, of
        negated parameter flows and of accumulated child flows (pcb_sum_ele_generic,
        pcb_sum_par_generic; FP32)."""
        alg, alpha = self._alg(propagation_alg, kwargs)
        d = self._desc(node_mars.device)
        B = node_mars.size(1)
        ld = node_mars.stride(0)
        st = nat.stream()
        for eg in d["el_groups"]:
            et = eg["tiles"]
            nat.call("pcb_sum_ele_generic", nat.ptr(node_flows), nat.ptr(node_mars), nat.ptr(element_mars),
                     nat.ptr(element_flows), ld, B, nat.ptr(params), nat.ptr(et), et.size(0), eg["cbs"],
                     nat.ptr(eg["krow"]), nat.ptr(eg["kw"]), self.block_size, alg, alpha, 1 if logspace_flows else 0,
                     1 if accumulate_ch_flows else 0, st)
        if param_flows is not None:
            pt = d["pf_tiles"]
            nat.call("pcb_sum_par_generic", nat.ptr(node_flows), nat.ptr(node_mars), nat.ptr(element_mars), ld, B,
                     nat.ptr(params), nat.ptr(param_flows), nat.ptr(pt), pt.size(0), self.block_size,
                     nat.ptr(d["krow"]), nat.ptr(d["kw"]), nat.ptr(d["kpf"]), alg, 1 if logspace_flows else 0,
                     1 if negate_pflows else 0, st)

    def param_flows_only(self, node_flows: torch.Tensor, node_mars: torch.Tensor, element_mars: torch.Tensor,
                         params: torch.Tensor, param_flows: torch.Tensor, allow_modify_flows: bool = False,
                         force_use_fp32: bool = False) -> None:
        """Accumulate this layer's parameter flows on the current stream (``allow_modify_flows``:
        node_flows already hold log f - log m for this layer's nodes)."""
        d = self._desc(node_mars.device)
        B = node_mars.size(1)
        ld = node_mars.stride(0)
        for t in (node_flows, element_mars):
            if t.size(1) != B or t.stride(0) != ld or t.stride(1) != 1:
                raise ValueError("node flows, node values and element values must share one [rows, B] layout")
        prec = 0 if force_use_fp32 or B < 16 else _mma(SumLayer.bf16_form)
        st = nat.stream()

        def run(c, target):
            tc05, kc = c
            pt = d[{128: "pf_tiles128", 64: "pf_tiles", 32: "pf_tiles32"}[kc]]
            nat.call("pcb_sum_pflows_tc05" if tc05 else "pcb_sum_pflows", nat.ptr(node_flows), nat.ptr(node_mars),
                     nat.ptr(element_mars), ld, B, nat.ptr(params), nat.ptr(target), nat.ptr(pt), pt.size(0),
                     self.block_size, nat.ptr(d["krow"]), nat.ptr(d["kw"]), nat.ptr(d["kpf"]),
                     1 if allow_modify_flows else 0, 1 if self._has_tied else 0, kc, prec, st)

        kc_fixed, tc_fixed = SumLayer.pflow_tile_children, SumLayer.pflow_tc05
        if prec == 0:
            cands = [(False, k) for k in ((kc_fixed,) if kc_fixed else (64, 32, 128))]
        else:
            kcs = (kc_fixed,) if kc_fixed else (64, 128, 32)
            tcs = (tc_fixed,) if tc_fixed is not None else (True, False)
            cands = [(t, k) for t in tcs for k in kcs if not (t and k == 32)]
        if len(cands) == 1:
            return run(cands[0], param_flows)
        # candidates accumulate into a scratch copy while they are timed
        scratch = _pflow_scratch(param_flows)
        choice = TUNER.pick(("pflows", prec, bool(allow_modify_flows), self._has_tied, d["pf_tiles"].size(0),
                             int(d["fw_tm"]), B), cands, lambda c: run(c, scratch))
        run(choice, param_flows)

    def __repr__(self):
        return f"SumLayer(nid_range={self._layer_nid_range}, num_nodes={self.num_nodes}, num_edges={self.num_edges})"


class ProdLayer(Layer):
    """A layer of product node vectors."""

    _tensor_lists = ("partitioned_nids", "partitioned_cids", "partitioned_u_cids", "partitioned_parids")
    # Backward: add the flows to the child rows (True) or overwrite them (False, set by the
    # circuit for layers that are the first to write all of their child rows).
    bk_accumulate = True

    def __init__(self, nodes: Sequence, global_nid_start: Optional[int] = None,
                 layer_sparsity_tol: Optional[float] = None, max_num_partitions: Optional[int] = None, **kwargs):
        super().__init__(nodes)
        if len(self.nodes) == 0 or len(set(self.nodes)) != len(self.nodes):
            raise ValueError("a product layer needs distinct node vectors")
        bs0 = self.nodes[0].block_size
        if global_nid_start is None:
            global_nid_start = bs0
        c = compile_prod_layer(self.nodes, global_nid_start, layer_sparsity_tol, max_num_partitions)
        self.use_block_sparse_edges = c["use_block_sparse"]
        self.block_size = c["block_size"]
        self.num_nodes = c["num_nodes"]
        self.num_edges = c["num_edges"]
        self._layer_nid_range = c["nid_range"]
        self.partitioned_nids, self.partitioned_cids = c["nids"], c["cids"]
        self.partitioned_u_cids, self.partitioned_parids = c["u_cids"], c["parids"]
        self.num_fw_partitions = len(self.partitioned_nids)
        self.num_bk_partitions = len(self.partitioned_u_cids)

    def is_prod(self):
        return True

    def _host_desc(self):
        def blocks(rows_list, chs_list):
            row, off, cnt, chs = [], [], [], []
            o = 0
            for r, c in zip(rows_list, chs_list):
                r_np, c_np = r.cpu().numpy(), c.cpu().numpy()
                for l in range(r_np.shape[0]):
                    real = c_np[l][c_np[l] != 0]
                    row.append(int(r_np[l]))
                    off.append(o)
                    cnt.append(real.shape[0])
                    chs.append(real)
                    o += real.shape[0]
            chs = np.concatenate(chs) if chs else np.zeros([0], np.int64)
            return _i32(row), _i32(off), _i32(cnt), _i32(chs)

        fr, fo, fc, fch = blocks(self.partitioned_nids, self.partitioned_cids)
        br, bo, bc, bch = blocks(self.partitioned_u_cids, self.partitioned_parids)
        lo, hi = self._layer_nid_range
        elem2blk = np.full([hi - lo], -1, np.int64)
        rows = fr.numpy().astype(np.int64)
        for i in range(self.block_size):
            elem2blk[rows + i - lo] = np.arange(rows.shape[0])
        return dict(fw_row=fr, fw_off=fo, fw_cnt=fc, fw_chs=fch, bk_row=br, bk_off=bo, bk_cnt=bc, bk_chs=bch,
                    elem2blk=_i32(elem2blk))

    def enable_partial_evaluation(self, fw_scopes=None, bk_scopes=None):
        """Block subsets: forward blocks of the product vectors with the given scopes, backward
        blocks writing the child vectors with the given scopes."""
        d = self._host_desc()

        def subset(prefix, keep):
            k = torch.from_numpy(keep)
            rows, offs, cnts = d[prefix + "_row"], d[prefix + "_off"], d[prefix + "_cnt"]
            return dict(row=rows[k].contiguous(), off=offs[k].contiguous(), cnt=cnts[k].contiguous(),
                        chs=d[prefix + "_chs"])
        if fw_scopes is not None:
            rng = self._ranges(self.nodes, set(fw_scopes))
            self._fw_partial = subset("fw", self._keep_rows(d["fw_row"].numpy(), rng))
        if bk_scopes is not None:
            kids = []
            for ns in self.nodes:
                for cs in ns.chs:
                    if cs not in kids:
                        kids.append(cs)
            rng = self._ranges(kids, set(bk_scopes))
            self._bk_partial = subset("bk", self._keep_rows(d["bk_row"].numpy(), rng))

    def forward(self, node_mars: torch.Tensor, element_mars: torch.Tensor, _for_backward: bool = False, **kwargs):
        d = self._desc(node_mars.device)
        part = self._partial("fw", node_mars.device)
        if part is not None:
            if part["row"].size(0) == 0:
                return
            d = dict(fw_row=part["row"], fw_off=part["off"], fw_cnt=part["cnt"], fw_chs=part["chs"])
        B = node_mars.size(1)
        ld = node_mars.stride(0)
        if element_mars.stride(0) != ld:
            raise ValueError("node_mars and element_mars must share a row-major layout")
        nat.call("pcb_prod_gather_sum", nat.ptr(node_mars), nat.ptr(element_mars), ld, B, nat.ptr(d["fw_row"]),
                 nat.ptr(d["fw_off"]), nat.ptr(d["fw_cnt"]), nat.ptr(d["fw_chs"]), d["fw_row"].size(0),
                 self.block_size, 0, 0, nat.stream())

    __call__ = forward

    def backward(self, node_flows: torch.Tensor, element_flows: torch.Tensor, logspace_flows: bool = False, **kwargs):
        d = self._desc(node_flows.device)
        B = node_flows.size(1)
        ld = node_flows.stride(0)
        if element_flows.stride(0) != ld:
            raise ValueError("node_flows and element_flows must share a row-major layout")
        part = self._partial("bk", node_flows.device)
        if part is not None:
            if part["row"].size(0) == 0:
                return
            # the selected child rows only; accumulate (they may also be written by other layers)
            nat.call("pcb_prod_gather_sum", nat.ptr(element_flows), nat.ptr(node_flows), ld, B, nat.ptr(part["row"]),
                     nat.ptr(part["off"]), nat.ptr(part["cnt"]), nat.ptr(part["chs"]), part["row"].size(0),
                     self.block_size, 1 if self.bk_accumulate else 0, 1 if logspace_flows else 0, nat.stream())
            return
        # _modify = (node_mars, block flags): the flows of the flagged child blocks are written
        # as log f - log m (what the sum layer below would rewrite them to); overwrite mode only
        mod = kwargs.get("_modify")
        if mod is not None:
            if self.bk_accumulate or logspace_flows:
                raise RuntimeError("fused flow rewriting needs an overwriting product layer and linear flows")
            nat.call("pcb_prod_gather_sum_modify", nat.ptr(element_flows), nat.ptr(node_flows), ld, B,
                     nat.ptr(d["bk_row"]), nat.ptr(d["bk_off"]), nat.ptr(d["bk_cnt"]), nat.ptr(d["bk_chs"]),
                     d["bk_row"].size(0), self.block_size, nat.ptr(mod[0]), nat.ptr(mod[1]), nat.stream())
            return
        nat.call("pcb_prod_gather_sum", nat.ptr(element_flows), nat.ptr(node_flows), ld, B, nat.ptr(d["bk_row"]),
                 nat.ptr(d["bk_off"]), nat.ptr(d["bk_cnt"]), nat.ptr(d["bk_chs"]), d["bk_row"].size(0),
                 self.block_size, 1 if self.bk_accumulate else 0, 1 if logspace_flows else 0, nat.stream())

    def __repr__(self):
        return f"ProdLayer(nid_range={self._layer_nid_range}, num_nodes={self.num_nodes}, num_edges={self.num_edges})"


_DIST_KIND = {"Categorical": 0, "Bernoulli": 1, "Gaussian": 2, "DiscreteLogistic": 3,
              "ExternSoftEvidenceCategorical": 4}
_CATEGORICAL_KINDS = (0, 4)  # parameter layout, flow histogram and EM of the Categorical


class InputLayer(Layer, torch.nn.Module):
    """A layer of input node vectors of one distribution: Categorical (lookups, counting-sort
    flows, soft evidence), Bernoulli, Gaussian or DiscreteLogistic (``input_dists.cu``), or
    SoftEvidenceCategorical (``input_poe.cu``: categorical nodes times per-sample evidence)."""

    _tensor_lists = ()

    def __init__(self, nodes: Sequence, cum_nodes: int = 0, pc_num_vars: int = 0,
                 max_tied_ns_per_parflow_block: int = 4):
        torch.nn.Module.__init__(self)
        c = compile_input_layer(nodes, cum_nodes, max_tied_ns_per_parflow_block)
        Layer.__init__(self, c["nodes"])
        self.pc_num_vars = pc_num_vars
        if c["signature"] not in _DIST_KIND:
            raise NotImplementedError(f"input distribution {c['signature']} has no CUDA path")
        self.kind = _DIST_KIND[c["signature"]]
        if c["num_vars_per_node"] != 1:
            raise NotImplementedError("multivariate input nodes have no CUDA path")
        self._output_ind_range = c["nid_range"]
        self.num_nodes = c["num_nodes"]
        self.num_parameters = c["num_parameters"]
        self.num_param_flows = c["num_param_flows"]
        self.dist_signature = c["signature"]
        self.num_vars_per_node = 1
        for name in ("vids", "s_pids", "s_pfids", "metadata", "s_mids", "nids", "source_nids", "node_id2source_id"):
            self.register_buffer(name, c[name])
        self.tied2source_nids = c["tied2source_nids"]
        self.params = torch.nn.Parameter(torch.empty([max(self.num_parameters, 1)], dtype=torch.float32),
                                         requires_grad=False)
        self.param_flows = None
        self.param_flows_f64 = None

    def is_input(self):
        return True

    def get_dist(self):
        return self.nodes[0].dist

    def get_data_dtype(self):
        return self.nodes[0].get_data_dtype()

    def to(self, device):
        torch.nn.Module.to(self, device)
        self.device = torch.device(device)
        if self.param_flows is not None:
            self.param_flows = self.param_flows.to(device)
        return self

    def _host_desc(self):
        vids = self.vids[:, 0].cpu().numpy()
        meta = self.metadata.cpu()
        if self.kind in _CATEGORICAL_KINDS:
            ncats = meta[self.s_mids.cpu()].long().numpy()
        else:
            ncats = np.ones(vids.shape[0], np.int64)
        # per-node metadata of input_dists.cu: Gaussian min_sigma; DiscreteLogistic
        # (lo, hi, num_cats, min_std)
        width = {2: 1, 3: 4}.get(self.kind, 1)
        if self.kind in (2, 3):
            sm = self.s_mids.cpu().long()
            node_meta = torch.stack([meta[sm + j].float() for j in range(width)], dim=1).reshape(-1)
        else:
            node_meta = torch.zeros([vids.shape[0]])
        # runs of consecutive nodes over the same variable
        change = np.ones(vids.shape[0], dtype=bool)
        change[1:] = vids[1:] != vids[:-1]
        starts = np.nonzero(change)[0]
        counts = np.diff(np.append(starts, vids.shape[0]))
        tied = []
        for dst, n, ch in self.tied2source_nids:
            tied.append((int(dst), int(n), ch.clone().long()))
        # nodes of every variable (CSR over the variable ids 0 .. max vid), for the evidence
        # backward contractions
        # the index of each group's variable among the layer's variables (the evidence row of
        # a SoftEvidenceCategorical layer), and the group of each node
        layer_vars = np.unique(vids)
        grp_lvid = np.searchsorted(layer_vars, vids[starts])
        node_grp = np.repeat(np.arange(starts.shape[0]), counts)
        order = np.argsort(vids, kind="stable")
        var_ptr = np.zeros(int(vids.max()) + 2, np.int64)
        np.add.at(var_ptr, vids + 1, 1)
        var_ptr = np.cumsum(var_ptr)
        return dict(vids=_i32(vids), s_pids=_i32(self.s_pids.cpu()), s_pfids=_i32(self.s_pfids.cpu()),
                    ncats=_i32(ncats), source_nids=_i32(self.source_nids.cpu()),
                    grp_var=_i32(vids[starts]), grp_node0=_i32(starts), grp_count=_i32(counts),
                    grp_ncats=_i32(ncats[starts]), max_ncats=int(ncats.max()), min_ncats=int(ncats.min()), max_grp=int(counts.max()),
                    shared_slots=bool(np.unique(self.s_pfids.cpu().numpy()).size < self.s_pfids.numel()),
                    node_meta=node_meta.contiguous(), grp_lvid=_i32(grp_lvid), node_grp=_i32(node_grp),
                    node_lvid=_i32(grp_lvid[node_grp]),
                    num_layer_vars=int(layer_vars.shape[0]),
                    tied=tied, var_ptr=var_ptr, var_nodes=order.astype(np.int64))

    def _init_parameters(self, perturbation: float = 2.0):
        p0 = 0
        with torch.no_grad():
            for ns in self.nodes:
                if ns.is_tied():
                    continue
                p1 = p0 + ns.num_nodes * ns.dist.num_parameters()
                src = ns._params if ns.has_params() else ns.init_parameters(perturbation=perturbation, ret_params=True)
                self.params[p0:p1] = src.to(self.params.device, torch.float32)
                p0 = p1

    def init_param_flows(self, flows_memory: float = 1.0):
        if self.param_flows is None or self.param_flows.device != self.params.device:
            self.param_flows = torch.zeros([max(self.num_param_flows, 1)], device=self.params.device)
        elif flows_memory == 0.0:
            self.param_flows.zero_()  # write-only; same as multiplying finite flows by zero
        elif flows_memory < 1.0:
            self.param_flows.mul_(flows_memory)

    def _mask_args(self, missing_mask, B: int, device, batch_first: bool = True):
        """(uint8 tensor or None, sample stride, variable stride) of a missing mask: ``[num_vars]``,
        ``[B, num_vars]`` or, with ``batch_first=False`` and ambiguous sizes, ``[num_vars, B]``
        (input_layer.py:378-385, 439-451)."""
        if missing_mask is None:
            return None, 0, 0
        m = missing_mask.to(device=device, dtype=torch.bool)
        if m.dim() == 1:
            return m.view(torch.uint8), 0, m.stride(0)
        if m.dim() != 2:
            raise ValueError("`missing_mask` must be [num_vars], [B, num_vars] or [num_vars, B]")
        if batch_first or m.size(1) == self.pc_num_vars:
            return m.view(torch.uint8), m.stride(0), m.stride(1)
        return m.view(torch.uint8), m.stride(1), m.stride(0)

    def forward(self, data: torch.Tensor, node_mars: torch.Tensor, params=None, missing_mask=None,
                _batch_first: bool = True, **kwargs):
        """``data`` is ``[num_vars, B]`` (int64), as passed by ``TensorCircuit.forward``;
        variables set in ``missing_mask`` are summed out (their nodes' values are log 1)."""
        if params is not None:
            raise NotImplementedError("external input parameters have no CUDA path")
        d = self._desc(node_mars.device)
        B = node_mars.size(1)
        m, sb, sv = self._mask_args(missing_mask, B, node_mars.device, _batch_first)
        if self.kind == 4:
            self._forward_poe(data, node_mars, d, B, (m, sb, sv), kwargs)
            return
        if self.kind != 0:
            xf = data.to(torch.float32)
            if xf.stride(1) != 1:
                xf = xf.contiguous()
            nat.call("pcb_input_dist_fwd", self.kind, nat.ptr(xf), xf.stride(0), nat.ptr(self.params),
                     nat.ptr(d["vids"]), nat.ptr(d["s_pids"]), nat.ptr(d["node_meta"]), self.num_nodes,
                     self._output_ind_range[0],
                     nat.ptr(node_mars), node_mars.stride(0), B, nat.ptr(m), sb, sv, nat.stream())
            return
        data = data.to(torch.long)
        if data.stride(1) != 1:
            data = data.contiguous()
        part = self._partial("fw", node_mars.device)
        runs = [(0, self.num_nodes)] if part is None else part["runs"]
        for n0, cnt in runs:  # the node tables are passed from the run's first node on
            nat.call("pcb_input_cat_fwd", nat.ptr(data), data.stride(0), nat.ptr(self.params),
                     c_void_p(d["vids"].data_ptr() + 4 * n0), c_void_p(d["s_pids"].data_ptr() + 4 * n0),
                     c_void_p(d["ncats"].data_ptr() + 4 * n0), cnt, self._output_ind_range[0] + n0,
                     nat.ptr(node_mars), node_mars.stride(0), B, nat.ptr(m), sb, sv, nat.stream())

    def _poe_evidence(self, d, B: int, device, kwargs):
        """(log-weights, category ids or None) of a SoftEvidenceCategorical layer's evidence,
        ``categorical_evidence_logp`` [B, num_layer_vars, K] (FP32) and optionally
        ``soft_evidence_cat_ids`` (int64, same shape) (softevi_categorical.py:25-84)."""
        ev = kwargs.get("categorical_evidence_logp")
        if ev is None:
            raise ValueError("a SoftEvidenceCategorical input layer needs `categorical_evidence_logp`")
        if ev.dim() != 3 or ev.dtype != torch.float32 or ev.device != device:
            raise ValueError("`categorical_evidence_logp` must be a float32 [B, num_vars, num_cats] tensor "
                             "on the circuit's device")
        if ev.size(0) != B or ev.size(1) < d["num_layer_vars"]:
            raise ValueError(f"`categorical_evidence_logp` must be [{B}, >= {d['num_layer_vars']}, K]")
        ids = kwargs.get("soft_evidence_cat_ids")
        if ids is None and ev.size(2) > d["min_ncats"]:
            raise ValueError("`categorical_evidence_logp` has more categories than the nodes")
        if ev.stride(2) != 1:
            ev = ev.contiguous()
        if ids is not None:
            if ids.shape != ev.shape or ids.device != device:
                raise ValueError("`soft_evidence_cat_ids` must have the shape of `categorical_evidence_logp`")
            ids = ids.to(torch.long)
            if ids.stride() != ev.stride():
                ids = ids.contiguous()
                ev = ev.contiguous()
        return ev, ids

    def _forward_poe(self, data, node_mars, d, B, mask, kwargs):
        ev, ids = self._poe_evidence(d, B, node_mars.device, kwargs)
        data = data.to(torch.long)
        if data.stride(1) != 1:
            data = data.contiguous()
        m, sb, sv = mask
        nat.call("pcb_input_poe_fwd", nat.ptr(data), data.stride(0), nat.ptr(ev), nat.ptr(ids), ev.stride(0),
                 ev.stride(1), ev.size(2), nat.ptr(self.params), nat.ptr(d["grp_var"]), nat.ptr(d["grp_lvid"]),
                 nat.ptr(d["grp_node0"]), nat.ptr(d["grp_count"]), d["grp_var"].size(0), d["max_grp"],
                 nat.ptr(d["node_grp"]), self.num_nodes, nat.ptr(d["s_pids"]), nat.ptr(d["ncats"]),
                 self._output_ind_range[0], nat.ptr(node_mars), node_mars.stride(0), B, nat.ptr(m), sb, sv,
                 nat.stream())

    def _backward_poe_evidence(self, data, node_flows, node_mars, d, B, logspace_flows, kwargs):
        """``categorical_evidence_logp_grad`` += the gradient of the flow-weighted node values
        with respect to the evidence log-weights (softevi_categorical.py:502-661)."""
        ev, ids = self._poe_evidence(d, B, node_flows.device, kwargs)
        grad = kwargs["categorical_evidence_logp_grad"]
        if grad.shape != ev.shape or grad.dtype != torch.float32 or grad.device != node_flows.device or \
                grad.stride(2) != 1:
            raise ValueError("`categorical_evidence_logp_grad` must be a float32 tensor shaped like the evidence, "
                             "contiguous over categories")
        nat.call("pcb_input_poe_evidence_bwd", nat.ptr(data), data.stride(0), nat.ptr(node_flows),
                 nat.ptr(node_mars), node_flows.stride(0), B, 1 if logspace_flows else 0, nat.ptr(ev), nat.ptr(ids),
                 ev.stride(0), ev.stride(1), ev.size(2), nat.ptr(grad), grad.stride(0), grad.stride(1),
                 nat.ptr(self.params), nat.ptr(d["grp_var"]), nat.ptr(d["grp_lvid"]), nat.ptr(d["grp_node0"]),
                 nat.ptr(d["grp_count"]), d["grp_var"].size(0), d["max_grp"], nat.ptr(d["s_pids"]),
                 nat.ptr(d["ncats"]), self._output_ind_range[0], nat.stream())

    def forward_soft(self, evidence: torch.Tensor, node_mars: torch.Tensor, missing_mask=None,
                     _batch_first: bool = True, **kwargs):
        """Soft evidence ``[B, num_vars, num_cats]`` (FP32, entries in [0, 1]):
        ``node_mars = min(log sum_k E[b, v, k] theta[n, k], 0)`` (conditional.py:25-68, 108-111)."""
        if self.kind != 0:
            raise NotImplementedError("soft evidence is defined for Categorical input layers")
        if evidence.dim() != 3 or evidence.dtype != torch.float32:
            raise ValueError("soft evidence must be a float32 [B, num_vars, num_cats] tensor")
        d = self._desc(node_mars.device)
        ev = evidence.to(node_mars.device)
        B = node_mars.size(1)
        if ev.size(0) != B or ev.size(2) < d["max_ncats"]:
            raise ValueError("soft evidence must be [B, num_vars, >= num_cats]")
        m, sb, sv = self._mask_args(missing_mask, B, node_mars.device, _batch_first)
        nat.call("pcb_input_cat_soft_fwd", nat.ptr(ev), ev.stride(0), ev.stride(1), ev.stride(2), nat.ptr(self.params),
                 nat.ptr(d["grp_var"]), nat.ptr(d["grp_node0"]), nat.ptr(d["grp_count"]), nat.ptr(d["grp_ncats"]),
                 d["grp_var"].size(0), d["max_grp"], nat.ptr(d["s_pids"]), self._output_ind_range[0],
                 nat.ptr(node_mars), node_mars.stride(0), B, nat.ptr(m), sb, sv, nat.stream())

    def enable_partial_evaluation(self, fw_scopes=None, bk_scopes=None):
        """Node subsets of the input vectors with the given scopes: runs of consecutive nodes
        (forward) and the variable groups (backward) that hold them."""
        d = self._host_desc()
        start = self._output_ind_range[0]

        def node_runs(scopes):
            runs = []
            for lo, hi in self._ranges(self.nodes, set(scopes)):
                runs.append((lo - start, hi - lo))
            return runs
        if fw_scopes is not None:
            self._fw_partial = dict(runs=node_runs(fw_scopes))
        if bk_scopes is not None:
            keep = np.zeros(d["grp_var"].numel(), dtype=bool)
            g0, gc = d["grp_node0"].numpy(), d["grp_count"].numpy()
            for n0, cnt in node_runs(bk_scopes):
                keep |= (g0 >= n0) & (g0 < n0 + cnt)
            k = torch.from_numpy(keep)
            self._bk_partial = {name: d[name][k].contiguous() for name in ("grp_var", "grp_node0", "grp_count",
                                                                          "grp_ncats")}

    def evidence_backward(self, node_flows: torch.Tensor, node_mars: Optional[torch.Tensor] = None,
                          target_vars=None, mode: int = 0) -> torch.Tensor:
        """``[B, T, max_ncats]``: per target variable and category, ``sum_n W[n, b] theta[n, k]``
        over the variable's nodes, W = node flows (mode 0) or node flows / exp(node_mars)
        (mode 1, the derivative of the weighted log-likelihood with respect to soft evidence)."""
        if self.kind != 0:
            raise NotImplementedError("per-category evidence quantities are defined for Categorical input layers")
        d = self._desc(node_flows.device)
        B = node_flows.size(1)
        nv = d["var_ptr"].shape[0] - 1
        tv = list(range(nv)) if target_vars is None else [int(v) for v in target_vars]
        key = ("tgt", tuple(tv) if target_vars is not None else None)
        tab = d.get(key)
        if tab is None:
            ptr, nodes = [0], []
            for v in tv:
                a, b = (int(d["var_ptr"][v]), int(d["var_ptr"][v + 1])) if 0 <= v < nv else (0, 0)
                nodes.append(d["var_nodes"][a:b])
                ptr.append(ptr[-1] + b - a)
            tab = (_i32(ptr).to(node_flows.device),
                   _i32(np.concatenate(nodes) if nodes else np.zeros([0], np.int64)).to(node_flows.device))
            d[key] = tab
        out = torch.empty([B, len(tv), d["max_ncats"]], dtype=torch.float32, device=node_flows.device)
        nat.call("pcb_input_cat_evidence_bwd", nat.ptr(node_flows), nat.ptr(node_mars), node_flows.stride(0), B,
                 nat.ptr(self.params), nat.ptr(tab[0]), nat.ptr(tab[1]), len(tv), nat.ptr(d["s_pids"]),
                 nat.ptr(d["ncats"]), self._output_ind_range[0], d["max_ncats"], mode, nat.ptr(out), nat.stream())
        return out

    __call__ = forward

    def backward(self, data: torch.Tensor, node_flows: torch.Tensor, node_mars: torch.Tensor, params=None,
                 logspace_flows: bool = False, missing_mask=None, _batch_first: bool = True, **kwargs):
        if params is not None:
            raise NotImplementedError("external input parameters have no CUDA path")
        d = self._desc(node_flows.device)
        if self.param_flows is None:
            self.init_param_flows(0.0)
        B = node_flows.size(1)
        m, sb, sv = self._mask_args(missing_mask, B, node_flows.device, _batch_first)
        if self.kind == 4:
            # parameter flows: the categorical histogram of the observed categories, missing or
            # not; then the evidence gradient when asked for (softevi_categorical.py:87-123, 464-500)
            if "categorical_evidence_logp" not in kwargs:
                return
            m, sb, sv = None, 0, 0
        if self.kind not in _CATEGORICAL_KINDS:
            xf = data.to(torch.float32)
            if xf.stride(1) != 1:
                xf = xf.contiguous()
            nat.call("pcb_input_dist_bwd", self.kind, nat.ptr(xf), xf.stride(0), nat.ptr(node_flows),
                     node_flows.stride(0), B, nat.ptr(self.params), nat.ptr(d["vids"]), nat.ptr(d["s_pids"]),
                     nat.ptr(d["s_pfids"]), nat.ptr(d["node_meta"]), self.num_nodes, self._output_ind_range[0],
                     nat.ptr(self.param_flows),
                     1 if logspace_flows else 0, nat.ptr(m), sb, sv, 1 if d["shared_slots"] else 0, nat.stream())
            return
        data = data.to(torch.long)
        if data.stride(1) != 1:
            data = data.contiguous()
        g = self._partial("bk", node_flows.device) or d
        if g["grp_var"].numel() == 0:
            return
        nat.call("pcb_input_cat_bwd", nat.ptr(data), data.stride(0), nat.ptr(node_flows), node_flows.stride(0), B,
                 nat.ptr(g["grp_var"]), nat.ptr(g["grp_node0"]), nat.ptr(g["grp_count"]), nat.ptr(g["grp_ncats"]),
                 g["grp_var"].size(0), d["max_ncats"], nat.ptr(d["s_pfids"]), self._output_ind_range[0],
                 nat.ptr(self.param_flows), 1 if logspace_flows else 0, nat.ptr(m), sb, sv, nat.ptr(d["s_pids"]),
                 nat.ptr(self.params), 1 if d["shared_slots"] else 0, nat.stream())
        if self.kind == 4 and "categorical_evidence_logp_grad" in kwargs:
            self._backward_poe_evidence(data, node_flows, node_mars, d, B, logspace_flows, kwargs)

    def mini_batch_em(self, step_size: float, pseudocount: float = 0.0, keep_zero_params: bool = False,
                      use_f64_flows: bool = False):
        d = self._desc(self.params.device)
        pf = self.param_flows_f64 if use_f64_flows else self.param_flows
        if pf is None:
            raise RuntimeError("no parameter flows for the input layer")
        for dst, n, ch in d["tied"]:
            nat.call("pcb_pflow_accum_f64" if use_f64_flows else "pcb_pflow_accum", nat.ptr(pf), dst, n, nat.ptr(ch),
                     ch.size(0), nat.stream())
        if self.kind not in _CATEGORICAL_KINDS:
            if use_f64_flows:
                raise NotImplementedError("FP64 epoch flows are kept for Categorical input layers")
            nat.call("pcb_input_dist_em", self.kind, nat.ptr(self.params), nat.ptr(pf), nat.ptr(d["s_pids"]),
                     nat.ptr(d["s_pfids"]), nat.ptr(d["node_meta"]), nat.ptr(d["source_nids"]),
                     d["source_nids"].size(0), float(step_size), float(pseudocount), nat.stream())
            return
        nat.call("pcb_input_cat_em_f64flows" if use_f64_flows else "pcb_input_cat_em", nat.ptr(self.params),
                 nat.ptr(pf), nat.ptr(d["s_pids"]), nat.ptr(d["s_pfids"]), nat.ptr(d["ncats"]),
                 nat.ptr(d["source_nids"]), d["source_nids"].size(0), float(step_size), float(pseudocount),
                 1 if keep_zero_params else 0, nat.stream())

    def init_param_flows_f64(self):
        n = max(self.num_param_flows, 1)
        if self.param_flows_f64 is None or self.param_flows_f64.device != self.params.device:
            self.param_flows_f64 = torch.zeros([n], dtype=torch.float64, device=self.params.device)
        else:
            self.param_flows_f64.zero_()

    def accumulate_param_flows_f64(self):
        if self.param_flows_f64 is None or self.param_flows_f64.device != self.params.device:
            self.init_param_flows_f64()
        nat.call("pcb_flows_accumulate_f64", nat.ptr(self.param_flows_f64), nat.ptr(self.param_flows),
                 self.param_flows.numel(), nat.stream())

    def update_parameters(self):
        for ns in self.nodes:
            if ns.is_tied():
                continue
            p0, p1 = ns._param_range
            ns._params = self.params.data[p0:p1].detach().cpu().clone()
            ns._param_initialized = True

    def __repr__(self):
        return f"InputLayer(nid_range={self._output_ind_range}, num_nodes={self.num_nodes})"


class LayerGroup:
    """Layers of one type at one depth, run one after another."""

    def __init__(self, layers: Sequence[Layer]):
        if len(layers) == 0:
            raise ValueError("A `LayerGroup` must contain at least 1 layer.")
        for l in layers:
            if type(l) is not type(layers[0]):
                raise ValueError("layers of a group must have the same type")
        self.layers = list(layers)
        self.num_layers = len(self.layers)
        if layers[0].is_input():
            self.layer_type = "input"
        elif layers[0].is_prod():
            self.layer_type = "prod"
        else:
            self.layer_type = "sum"

    def to(self, device):
        for l in self.layers:
            l.to(device)
        return self

    def forward(self, *args, **kwargs):
        for l in self.layers:
            l.forward(*args, **kwargs)

    __call__ = forward

    def backward(self, *args, **kwargs):
        for l in self.layers:
            l.backward(*args, **kwargs)

    def enable_partial_evaluation(self, fw_scopes=None, bk_scopes=None):
        for l in self.layers:
            l.enable_partial_evaluation(fw_scopes=fw_scopes, bk_scopes=bk_scopes)

    def disable_partial_evaluation(self, forward: bool = True, backward: bool = True):
        for l in self.layers:
            l.disable_partial_evaluation(forward=forward, backward=backward)

    def callback(self, fn, *args, **kwargs):
        if fn is not None:
            for l in self.layers:
                fn(l, *args, **kwargs)

    def is_input(self):
        return self.layer_type == "input"

    def is_prod(self):
        return self.layer_type == "prod"

    def is_sum(self):
        return self.layer_type == "sum"

    def __len__(self):
        return self.num_layers

    def __getitem__(self, idx):
        return self.layers[idx]

    def __iter__(self):
        return iter(self.layers)
