"""EM-step throughput of a compiled HCLT on B200 (one JSON line on rank 0).

Workload: HCLT over 28x28 variables with 256 categories, 128 latents, block size 32,
batch 512; data = seeded Gaussian random fields (length scale 3 px) quantised to 256
levels (stand-in for MNIST, same shapes). One step = ``init_param_flows(0)`` ->
forward -> backward -> ``mini_batch_em(step_size=0.1, pseudocount=0.1)``.

* ``value``: samples/s of the BF16 tensor-core form, whole step captured in one CUDA
  graph, inputs resident in HBM, device time (CUDA events), max over ranks;
* ``fp32_plain``: the same for the plain FP32 form;
* ``e2e``: the BF16 form through the public API (``lls = pc(x, record_cudagraph=True)``,
  ``lls.mean().backward()``, ``pc.mini_batch_em``) with every step's batch copied from
  pinned host memory (on a copy stream, while the previous step computes, as an input
  pipeline does; the first copy starts after the timer) and the log-likelihoods read back
  every step;
* ``roofline``: the parameter-flow launch of the largest sum layer (the kernel with the
  largest share of the step), timed per launch with CUDA events;
* ``cpu_baseline``: the FP32 PyTorch CPU restatement of the same step (``oracle/torch_port.py``)
  at the same batch on all host cores, a few whole steps.

``--impl reference`` times that CPU implementation of the same step instead (the reference
itself is Python + Triton with no CPU path; its arithmetic is restated by ``oracle/``, whose
FP64 version is pinned to the reference's own outputs), on all host cores, at the same
batch, rank 0 only.

Multi-GPU (``torchrun``): data-parallel replicas; each rank runs its own batch and the
parameter flows are summed with an NCCL all-reduce before every EM update
(weak scaling).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIDE = 28
NUM_CATS = 256
LATENTS = 128
BLOCK = 32
BATCH = 512
STEP_SIZE = 0.1
PSEUDOCOUNT = 0.1
# DRAM bytes (read + written) of the roofline launch, the largest layer's parameter flows,
# from one ncu capture of `bench.py --profile-step` (-k regex:sum_pflows -s 63 -c 1).
PFLOW_TRAFFIC_BYTES = 81_879_552
METRIC = "EM samples/s (fwd+bwd+update) 1xB200, BF16-TC vs FP32 plain; dLL vs FP64 oracle"
WORKLOAD = "HCLT 28x28 vars x 256 cats, 128 latents, block 32, EM step (fwd+bwd+mini_batch_em)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--batch", type=int, default=BATCH)
    p.add_argument("--workload", default="em", choices=["em", "adjoint", "pd", "hmm"],
                   help="em: the EM step on HCLT-784 (default); adjoint: the soft-evidence log-likelihood and its "
                        "gradients on HCLT-3072 (32x32x3 fields, 256 latents, batch 128); pd: full-batch EM epochs "
                        "on a Poon-Domingos circuit over 28x28 (256 latents, block 64, batch 256); hmm: 16 uneven "
                        "HMMs (hidden 256-4096, vocab 8192) in one circuit, EM steps on 64 sequences each")
    p.add_argument("--fd", action="store_true", help="adjoint workload: also check coordinates of both gradients "
                                                     "against FP64 central differences of the oracle (minutes)")
    p.add_argument("--profile-step", action="store_true",
                   help="run one warm-up step and one EM step (BF16 form) inside the NVTX range 'em_step', "
                        "for kernel profilers; prints the kernels launched per step")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def make_data(num_samples: int):
    from pyjuice_b200.synthetic import gaussian_field_data
    return gaussian_field_data(num_samples, side=SIDE, num_cats=NUM_CATS, length_scale=3.0, seed=0)


def build_circuit(data: torch.Tensor, device):
    """HCLT over the data's Chow-Liu tree (mutual information from the first 8192 samples)."""
    import pyjuice_b200 as juice
    from pyjuice_b200.nodes.distributions import Categorical
    from pyjuice_b200.structures import hclt_from_tree, chow_liu_tree
    from pyjuice_b200.structures.hclt import mutual_information_chunked
    x = data[:8192].float()
    if device.type == "cuda":
        x = x.to(device)
    mi = mutual_information_chunked(x, x, 32, 0.5 / 32, chunk_size=64).cpu().numpy()
    tree = chow_liu_tree(mi)
    root = tree.center()
    torch.manual_seed(0)
    ns = hclt_from_tree(tree.dfs_postorder(root), tree.bfs_children(root), root, LATENTS,
                        input_dist=Categorical(num_cats=NUM_CATS), block_size=BLOCK)
    return juice.compile(ns)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "20"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


def sum_forward_roofline(pc, x, precision_kw, reps=10):
    """Device time of every sum layer's forward (its weight-pack and contraction launches),
    each captured ``reps`` times in one CUDA graph and timed with CUDA events on the
    launching stream; element_mars holds the layer's children from the preceding product
    layers.

    Algorithmic bytes of a layer: each child row read once (4 B x batch), each node row
    written once (4 B x batch), each edge weight read once (4 B). Returns totals over the
    layers and the figures of the largest layer.
    """
    with torch.no_grad():
        pc(x, **precision_kw)
    B = x.size(0)
    per_layer = []

    def timed(fn):
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            fn()
        torch.cuda.current_stream().wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(reps):
                fn()
        graph.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        graph.replay()
        e1.record()
        e1.synchronize()
        del graph
        return e0.elapsed_time(e1) / 1e3 / reps

    with torch.no_grad():
        for gi, g in enumerate(pc.inner_layer_groups):
            if g.is_prod():
                g(pc.node_mars, pc.element_mars)
                continue
            for layer in g:
                d = layer._desc(x.device)
                child_rows = int(torch.unique(d["krow"]).numel())
                nbytes = 4 * B * (child_rows + layer.num_nodes) + 4 * layer.num_edges
                packs = layer.pack_forward_weights(pc.params, B, **precision_kw)
                # the contraction alone (the weights packed beforehand, as the forward pass
                # packs all layers' weights on a side stream), then the pack alone
                t_c = timed(lambda: layer(pc.node_mars, pc.element_mars, pc.params, _weights_packed=packs,
                                          **precision_kw))
                t_p = timed(lambda: layer.pack_forward_weights(pc.params, B, **precision_kw)) if packs else 0.0
                per_layer.append((nbytes, 2 * layer.num_edges * B, t_c, d["fw_tiles"].size(0), t_p))
    tot_b = sum(r[0] for r in per_layer)
    tot_f = sum(r[1] for r in per_layer)
    tot_s = sum(r[2] for r in per_layer)
    big = max(per_layer, key=lambda r: r[0])
    return {"layers": len(per_layer), "bytes": tot_b, "flops": tot_f, "seconds": tot_s,
            "pack_seconds": sum(r[4] for r in per_layer),
            "largest": {"bytes": big[0], "flops": big[1], "seconds": big[2], "tiles": big[3], "pack_seconds": big[4]}}


def pflows_roofline(pc, reps=10):
    """Device time of the parameter-flow launch of the largest sum layer (after a full
    forward + backward, so its node flows hold log f - log m), captured ``reps`` times in one
    CUDA graph and timed with CUDA events on the launching stream.

    Algorithmic bytes: the layer's node-flow rows and its children's element rows once
    (4 B x batch each), every edge's parameter once (4 B) and its flow slot read and
    written (8 B).
    """
    groups = pc.inner_layer_groups
    gi, layer = max(((gi, l) for gi, g in enumerate(groups) if g.is_sum() for l in g.layers),
                    key=lambda t: t[1].num_edges)
    d = layer._desc(pc.node_mars.device)
    B = pc.node_mars.size(1)
    em = pc._em_view(gi - 1)
    child_rows = int(torch.unique(d["krow"]).numel())
    nbytes = 4 * B * (layer.num_nodes + child_rows) + 12 * layer.num_edges

    def run():
        layer.param_flows_only(pc.node_flows, pc.node_mars, em, pc.params, pc.param_flows, allow_modify_flows=True)

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        run()
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(reps):
            run()
    graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    graph.replay()
    e1.record()
    e1.synchronize()
    secs = e0.elapsed_time(e1) / 1e3 / reps
    return {"bytes": nbytes, "seconds": secs, "flops": 2 * layer.num_edges * B, "group": gi,
            "tiles": d["pf_tiles"].size(0)}


def cpu_step_rate(layout, params, in_params, data, budget_s, batch=BATCH):
    """CPU implementation of the same EM step (``oracle/torch_port.py``: the FP32 PyTorch
    restatement of the reference's arithmetic, batched tensor operations on every host core),
    at the benchmark's batch: whole steps until about ``budget_s`` seconds have passed (one at
    least); returns (samples/s, description)."""
    from oracle import torch_port as tp
    tl = tp.TorchLayout(layout)
    p = torch.from_numpy(np.asarray(params, dtype=np.float32))
    q = torch.from_numpy(np.asarray(in_params, dtype=np.float32))
    x = data[:batch].long()
    times = []
    t_start = time.perf_counter()
    while not times or time.perf_counter() - t_start < budget_s:
        t0 = time.perf_counter()
        tp.em_step(tl, p, q, x, STEP_SIZE, PSEUDOCOUNT)
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return batch / med, (f"FP32 PyTorch CPU restatement of the EM step (oracle/torch_port.py), batch {batch}, "
                         f"median of {len(times)} whole steps ({med:.2f} s each)")


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    data = make_data(8192)
    # mutual information is structure building, not the timed path: use a GPU when present
    pc = build_circuit(data, torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu"))
    from oracle import pc_oracle as orc
    from oracle import torch_port as tp
    tl = tp.TorchLayout(orc.layout_from_circuit(pc))
    params = pc.params.detach().cpu().float()
    in_params = pc.input_layer_group[0].params.detach().cpu().float()
    B = args.batch
    x = data[:B].long()
    # A step of this CPU implementation takes seconds, so the run is bounded by time: the
    # requested warm-up steps (at most 3), then timed steps until about two minutes have
    # passed (at least 3, at most --steps).
    warm = max(1, min(args.warmup, 3))
    budget_s = 120.0
    times = []
    t_start = time.perf_counter()
    i = 0
    while True:
        t0 = time.perf_counter()
        params, in_params, _ = tp.em_step(tl, params, in_params, x, STEP_SIZE, PSEUDOCOUNT)
        if i >= warm:
            times.append(time.perf_counter() - t0)
        i += 1
        if len(times) >= max(1, args.steps):
            break
        if len(times) >= 3 and time.perf_counter() - t_start > budget_s:
            break
    v = B / statistics.median(times)
    sample = (f"FP32 PyTorch CPU restatement of the reference's EM step (oracle/torch_port.py) on {threads} "
              f"threads, batch {B}, median of {len(times)} steps")
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "samples/s", "n_gpus": args.gpus,
                      "steps": len(times), "warmup": warm, "ms_per_step": 1e3 * statistics.median(times),
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                      "data": "synthetic", "config": {"workload": WORKLOAD, "batch_per_gpu": B},
                      "cpu_baseline": {"value": v, "unit": "samples/s", "cores": threads, "kind": "port",
                                       "sample": sample},
                      "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def adjoint_workload(args):
    """Differentiable HCLT on 3072 vars (three 32x32 quantised random-field channels, 256
    categories), 256 latents, block 32, batch 128: per step, ``autograd.circuit_ll`` on
    soft evidence ``E [128, 3072, 256]`` (Dirichlet(1) rows) with sum weights
    ``softmax(z)``, then ``d mean-LL / d z`` and ``d mean-LL / d E`` (the hand-written
    adjoint). Timed with CUDA events over ``--steps`` steps after ``--warmup``; evidence and
    logits resident. ``--fd``: a few coordinates of both gradients at batch 2 against FP64
    central differences (h = 1e-6) of the oracle."""
    import pyjuice_b200 as juice
    from pyjuice_b200 import _native as nat
    from pyjuice_b200.nodes.distributions import Categorical
    from pyjuice_b200.structures import hclt_from_tree, chow_liu_tree
    from pyjuice_b200.structures.hclt import mutual_information_chunked
    from pyjuice_b200.synthetic import gaussian_field_data
    ws, rank, local = dist_env()
    if ws > 1 and rank != 0:
        return
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    nat.load()
    side, ch, lat, B, K = 32, 3, 256, 128, NUM_CATS
    data = gaussian_field_data(8192, side=side, num_cats=K, length_scale=3.0, channels=ch, seed=0)
    x = data.float().to(device)
    mi = mutual_information_chunked(x, x, 32, 0.5 / 32, chunk_size=64).cpu().numpy()
    del x
    tree = chow_liu_tree(mi)
    root = tree.center()
    torch.manual_seed(0)
    ns = hclt_from_tree(tree.dfs_postorder(root), tree.bfs_children(root), root, lat,
                        input_dist=Categorical(num_cats=K), block_size=BLOCK)
    pc = juice.compile(ns).to(device)
    V = side * side * ch
    gen = torch.Generator(device=device).manual_seed(5)
    z = torch.randn([pc.params.numel()], generator=gen, device=device).requires_grad_(True)
    ev = -torch.log(torch.rand([B, V, K], generator=gen, device=device).clamp_(min=1e-30))
    ev = (ev / ev.sum(dim=2, keepdim=True)).requires_grad_(True)   # Dirichlet(1) rows

    def step():
        z.grad = None
        ev.grad = None
        lls = juice.autograd.circuit_ll(pc, z, ev)
        lls.mean().backward()
        return lls

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        lls = step()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    ok = bool(torch.isfinite(lls).all()) and bool(torch.isfinite(z.grad).all()) and bool(torch.isfinite(ev.grad).all())
    peak_resident = torch.cuda.max_memory_allocated(device)
    # the same steps with the element values recomputed per layer group instead of resident
    pc.recompute_element_values = True
    pc.__dict__.pop("_em_resident", None)
    torch.cuda.empty_cache()
    torch.cuda.reset_peak_memory_stats(device)
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record()
    for _ in range(args.steps):
        step()
    e3.record()
    e3.synchronize()
    ms_rc = e2.elapsed_time(e3) / args.steps
    peak_recompute = torch.cuda.max_memory_allocated(device)
    pc.recompute_element_values = False
    out = {"metric": "adjoint samples/s (soft-evidence LL + d/d sum-logits + d/d evidence) 1xB200",
           "value": B / (ms / 1e3), "unit": "samples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "HCLT 32x32x3 vars x 256 cats, 256 latents, block 32, soft evidence, batch 128",
                      "num_nodes": pc.num_nodes, "num_edges": pc.num_edges, "evidence_bytes": ev.numel() * 4},
           "finite": ok, "mean_ll": float(lls.detach().mean()),
           "element_values": {"resident": {"ms_per_step": ms, "peak_bytes": peak_resident},
                              "recomputed_per_layer_group": {"ms_per_step": ms_rc, "peak_bytes": peak_recompute}}}
    if args.fd:
        out["fd_check"] = adjoint_fd_check(pc, z.detach(), ev.detach()[:2], device)
    print(json.dumps(out), flush=True)


def adjoint_fd_check(pc, z, ev, device, n_coords=2, h=1e-6):
    """Gradients of sum_b LL_b (b < 2) at the FP32 point against FP64 central differences of
    the oracle; returns the relative errors."""
    import pyjuice_b200 as juice
    from oracle import pc_oracle as orc
    lay = orc.layout_from_circuit(pc)
    q0 = pc.input_layer_group[0].params.double().cpu().numpy()
    pb, nch, bsz = pc._em_pbase.tolist(), pc._em_nch.tolist(), pc._em_bs.tolist()

    def softmax_params(zz):
        p = np.zeros_like(zz)
        for b0, k, bs in zip(pb, nch, bsz):
            blk = zz[b0:b0 + k * bs].reshape(k, bs)
            e = np.exp(blk - blk.max(axis=0))
            p[b0:b0 + k * bs] = (e / e.sum(axis=0)).reshape(-1)
        return p

    z64 = z.double().cpu().numpy()
    e64 = ev.double().cpu().numpy()

    def f(zz, ee):
        _, _, lls = orc.forward(lay, softmax_params(zz), q0, evidence=ee)
        return float(lls[:, 0].sum())

    zt = z.clone().requires_grad_(True)
    et = ev.clone().requires_grad_(True)
    juice.autograd.circuit_ll(pc, zt, et).sum().backward()
    gz, ge = zt.grad.double().cpu().numpy(), et.grad.double().cpu().numpy()
    rng = np.random.default_rng(3)
    used = np.concatenate([np.arange(b0, b0 + k * bs) for b0, k, bs in zip(pb, nch, bsz)])
    errs = {"logits": [], "evidence": []}
    for i in rng.choice(used, size=n_coords, replace=False):
        d = np.zeros_like(z64)
        d[i] = h
        fd = (f(z64 + d, e64) - f(z64 - d, e64)) / (2 * h)
        errs["logits"].append(abs(gz[i] - fd) / max(abs(fd), 1e-2))
    for _ in range(n_coords):
        b, v, k = rng.integers(ev.size(0)), rng.integers(ev.size(1)), rng.integers(ev.size(2))
        d = np.zeros_like(e64)
        d[b, v, k] = h
        fd = (f(z64, e64 + d) - f(z64, e64 - d)) / (2 * h)
        errs["evidence"].append(abs(ge[b, v, k] - fd) / max(abs(fd), 1e-2))
    return {"batch": int(ev.size(0)), "h": h, "coords_each": n_coords,
            "max_rel_err_logits": max(errs["logits"]), "max_rel_err_evidence": max(errs["evidence"])}


def pd_workload(args):
    """Poon-Domingos circuit over 28x28 vars (256 categories), 256 latents, block 64,
    split_intervals 4, ``torch.manual_seed(0)`` before construction; quantised random-field
    data. One full-batch EM epoch per precision form (plain FP32, split bf16, E4M3 on the
    tcgen05 levels): 234 batches of 256 (59,904 samples; the 96-sample remainder of 60,000
    is dropped), per batch forward + backward + FP64 flow accumulation, then one EM update
    from the FP64 flows. Epochs timed with CUDA events after one warm-up epoch of the form;
    the data is resident. LL error of each form against the FP64 oracle on 16 samples at the
    initial parameters."""
    import pyjuice_b200 as juice
    from pyjuice_b200 import _native as nat
    from pyjuice_b200.layer.layers import SumLayer
    from pyjuice_b200.nodes.distributions import Categorical
    from pyjuice_b200.structures import PD
    ws, rank, local = dist_env()
    if ws > 1 and rank != 0:
        return
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    nat.load()
    B, nb = 256, 234
    data = make_data(60000)
    torch.manual_seed(0)
    ns = PD((SIDE, SIDE), num_latents=256, split_intervals=4, block_size=64, input_dist=Categorical(num_cats=NUM_CATS))
    pc = juice.compile(ns).to(device)
    data_dev = data[:B * nb].to(device)
    forms = (("fp32", 2, {"force_use_fp32": True}), ("bf16_split", 2, {"force_use_bf16": True}),
             ("e4m3", 3, {"force_use_bf16": True}))
    # LL error at the initial parameters
    from oracle import pc_oracle as orc
    lay = orc.layout_from_circuit(pc)
    p64 = pc.params.detach().double().cpu().numpy()
    q64 = pc.input_layer_group[0].params.detach().double().cpu().numpy()
    xs = data[:16]
    _, _, lls_o = orc.forward(lay, p64, q64, xs.numpy())
    ll_err = {}
    with torch.no_grad():
        for name, form, kw in forms:
            SumLayer.bf16_form = form
            got = pc(xs.to(device), **kw).double().cpu().numpy()
            ll_err[name] = {"mean_abs_dll_nats": float(np.abs(got - lls_o).mean()),
                            "max_abs_dll_nats": float(np.abs(got - lls_o).max())}
    ll_err["mean_ll_nats"] = float(lls_o.mean())

    def epoch(kw):
        pc.init_param_flows_f64()
        for i in range(nb):
            x = data_dev[i * B:(i + 1) * B]
            pc.init_param_flows(flows_memory=0.0)
            with torch.no_grad():
                pc(x, **kw)
            pc.backward(inputs=x, allow_modify_flows=True, force_use_fp32="force_use_fp32" in kw)
            pc.accumulate_param_flows_f64()
        pc.mini_batch_em(step_size=1.0, pseudocount=PSEUDOCOUNT, use_f64_flows=True)

    res = {}
    init = pc.params.detach().clone(), pc.input_layer_group[0].params.detach().clone()
    for name, form, kw in forms:
        SumLayer.bf16_form = form
        pc.params.data.copy_(init[0])
        pc.input_layer_group[0].params.data.copy_(init[1])
        epoch(kw)  # warm-up (autotuning, buffers)
        pc.params.data.copy_(init[0])
        pc.input_layer_group[0].params.data.copy_(init[1])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        epoch(kw)
        e1.record()
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        res[name] = {"epoch_s": sec, "samples_per_s": B * nb / sec,
                     "params_finite": bool(torch.isfinite(pc.params).all())}
    SumLayer.bf16_form = 2
    out = {"metric": "full-batch EM epoch samples/s (fwd+bwd+FP64 flow accumulation, one EM update) 1xB200",
           "value": res["bf16_split"]["samples_per_s"], "unit": "samples/s", "n_gpus": 1, "steps": nb,
           "warmup": 1, "ms_per_step": res["bf16_split"]["epoch_s"] * 1e3 / nb, "higher_is_better": True,
           "dtype": "bf16", "data": "synthetic",
           "config": {"workload": "PD 28x28 vars x 256 cats, 256 latents, block 64, split_intervals 4, batch 256, "
                                  "epoch of 234 batches", "num_nodes": pc.num_nodes, "num_edges": pc.num_edges,
                      "num_sum_params": pc.num_sum_params},
           "forms": res, "ll_error_vs_fp64": ll_err}
    print(json.dumps(out), flush=True)


def hmm_workload(args):
    """16 HMMs of uneven size in one compiled circuit (``structures.batched_hmms``: a product
    of their roots over disjoint variables, so every layer group runs the same-depth layers
    of all HMMs in shared launches): hidden sizes cycling 256, 512, 1024, 2048, 4096, vocab
    8192, lengths ~ U[16, 64] (seed 0), transition / emission / initial rows ~
    Dirichlet(0.1); 64 sequences sampled from each HMM's own tables. One EM step (forward,
    backward, ``mini_batch_em``) in split bf16 is captured in a CUDA graph and replayed
    ``--steps`` times (CUDA events) after ``--warmup`` eager steps (the autotuner picks the
    launch shapes there); with and without the chunked tcgen05 path for the long tiles.
    LL error of the forest against the FP64 oracle on 2 sequences."""
    import pyjuice_b200 as juice
    from pyjuice_b200 import _native as nat
    from pyjuice_b200.layer.layers import SumLayer
    from pyjuice_b200.structures import batched_hmms
    ws, rank, local = dist_env()
    if ws > 1 and rank != 0:
        return
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    nat.load()
    V, S = 8192, 64
    rng = np.random.default_rng(0)
    hs = [256, 512, 1024, 2048, 4096]
    specs = [(int(rng.integers(16, 65)), hs[i % 5]) for i in range(16)]

    def dirichlet(*shape):
        g = rng.gamma(0.1, size=shape).astype(np.float64) + 1e-30
        return g / g.sum(-1, keepdims=True)

    params, tokens = [], []
    for T, L in specs:
        a, b, g = dirichlet(L, L), dirichlet(L, V), dirichlet(L)
        params.append((torch.from_numpy(a).float(), torch.from_numpy(b).float(), torch.from_numpy(g).float()))
        ca, cb = np.cumsum(a, axis=1), np.cumsum(b, axis=1)
        z = np.searchsorted(np.cumsum(g), rng.random(S) * np.cumsum(g)[-1]).clip(0, L - 1)
        seq = np.empty([S, T], np.int64)
        for t in range(T):
            u = rng.random(S)
            seq[:, t] = [min(int(np.searchsorted(cb[zi], ui * cb[zi, -1])), V - 1) for zi, ui in zip(z, u)]
            u = rng.random(S)
            z = np.array([min(int(np.searchsorted(ca[zi], ui * ca[zi, -1])), L - 1) for zi, ui in zip(z, u)])
        tokens.append(seq)
    x = torch.from_numpy(np.concatenate(tokens, axis=1)).to(device)
    t0 = time.time()
    pc = juice.compile(batched_hmms(specs, V, params=params)).to(device)
    compile_s = time.time() - t0

    def step():
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            pc(x, force_use_bf16=True)
        pc.backward(inputs=x, allow_modify_flows=True)
        pc.mini_batch_em(step_size=STEP_SIZE, pseudocount=PSEUDOCOUNT)

    if args.profile_step:  # one warm-up step, then one step in the NVTX range "em_step"
        step()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("em_step")
        step()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile_step": "hmm", "ok": bool(torch.isfinite(pc.params).all())}), flush=True)
        return
    init = pc.params.detach().clone(), pc.input_layer_group[0].params.detach().clone()
    res = {}
    for name, long_tc05 in (("tc05_chunks", True), ("mma_sync", False)):
        SumLayer.tc05_long = long_tc05
        pc.params.data.copy_(init[0])
        pc.input_layer_group[0].params.data.copy_(init[1])
        for _ in range(max(3, args.warmup)):
            step()
        torch.cuda.synchronize()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            step()
        torch.cuda.current_stream().wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            step()
        graph.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            graph.replay()
        e1.record()
        e1.synchronize()
        del graph
        ms = e0.elapsed_time(e1) / args.steps
        res[name] = {"ms_per_step": ms, "sequences_per_s": 16 * S / (ms / 1e3),
                     "tokens_per_s": S * int(x.size(1)) / (ms / 1e3),
                     "params_finite": bool(torch.isfinite(pc.params).all())}
    SumLayer.tc05_long = True
    best = min(res, key=lambda k: res[k]["ms_per_step"])
    # LL of the forest at the initial parameters against the FP64 oracle (2 sequences)
    from oracle import pc_oracle as orc
    pc.params.data.copy_(init[0])
    pc.input_layer_group[0].params.data.copy_(init[1])
    with torch.no_grad():
        got = pc(x[:2], force_use_fp32=True).double().cpu().numpy()
        got_bf = pc(x[:2].repeat(8, 1), force_use_bf16=True)[:2].double().cpu().numpy()
    lay = orc.layout_from_circuit(pc)
    _, _, lls_o = orc.forward(lay, init[0].double().cpu().numpy(), init[1].double().cpu().numpy(), x[:2].cpu().numpy())
    out = {"metric": "EM sequences/s (fwd+bwd+update) of 16 uneven HMMs in one circuit 1xB200",
           "value": res[best]["sequences_per_s"], "unit": "sequences/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": res[best]["ms_per_step"], "higher_is_better": True, "dtype": "bf16",
           "data": "synthetic",
           "config": {"workload": "16 HMMs (hidden 256..4096 cycling, vocab 8192, T ~ U[16,64]), 64 sequences each, "
                                  "one circuit, CUDA graph", "specs": specs, "num_nodes": pc.num_nodes,
                      "num_edges": pc.num_edges, "num_sum_params": pc.num_sum_params,
                      "layer_groups": len(pc.inner_layer_groups), "compile_s": compile_s},
           "paths": res, "best": best,
           "ll_error_vs_fp64": {"fp32_max_abs_dll_nats": float(np.abs(got - lls_o).max()),
                                "bf16_max_abs_dll_nats": float(np.abs(got_bf - lls_o).max()),
                                "mean_ll_nats": float(lls_o.mean())}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.workload == "hmm":
        return hmm_workload(args)
    if args.workload == "adjoint":
        return adjoint_workload(args)
    if args.workload == "pd":
        return pd_workload(args)
    if args.impl == "reference":
        return reference_arm(args)
    ws, rank, local = dist_env()
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    group = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)
        group = dist.group.WORLD
    from pyjuice_b200 import _native as nat
    nat.load()
    B = args.batch
    n_data = max(8192, B * 8)
    data = make_data(n_data)
    pc = build_circuit(data, device).to(device)
    data_dev = data[torch.arange(rank * B, rank * B + B * 8) % n_data].to(device)  # 8 resident batches per rank

    from pyjuice_b200.distributed import allreduce_param_flows, broadcast_parameters
    if group is not None:
        broadcast_parameters(pc, src=0, group=group)

    def allreduce_flows():
        if group is not None:
            allreduce_param_flows(pc, group=group)

    def step(x, kw):
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            pc(x, **kw)
        pc.backward(inputs=x, allow_modify_flows=True, force_use_fp32=kw.get("force_use_fp32", False))
        allreduce_flows()
        pc.mini_batch_em(step_size=STEP_SIZE, pseudocount=PSEUDOCOUNT)

    # kernels per step: every C-ABI call launches one kernel
    n0 = nat.CALLS
    step(data_dev[:B], {"force_use_bf16": True})
    kernels_per_step = nat.CALLS - n0
    if args.profile_step:
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("em_step")
        step(data_dev[B:2 * B], {"force_use_bf16": True})
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        if rank == 0:
            print(json.dumps({"profile_step": True, "kernels_per_step": kernels_per_step}), flush=True)
        return

    def timed(kw, use_graph, sample_clocks=False):
        x_static = data_dev[:B].clone()
        g = None
        if use_graph:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                for _ in range(2):
                    step(x_static, kw)
            torch.cuda.current_stream().wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                step(x_static, kw)
        # nvidia-smi needs a moment to start: the sampler runs from before the warm-up steps
        # to the end of the timed region
        clocks = Clocks(local) if sample_clocks else None
        for i in range(args.warmup):
            x_static.copy_(data_dev[(i % 8) * B:(i % 8 + 1) * B])
            g.replay() if g is not None else step(x_static, kw)
        torch.cuda.synchronize()
        if group is not None:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(args.steps):
            x_static.copy_(data_dev[(i % 8) * B:(i % 8 + 1) * B])
            g.replay() if g is not None else step(x_static, kw)
        e1.record()
        torch.cuda.synchronize()
        ck = clocks.stop() if clocks is not None else None
        ms = e0.elapsed_time(e1)
        if group is not None:
            import torch.distributed as dist
            t = torch.tensor([ms], device=device)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        del g
        return ms, ck

    from pyjuice_b200.layer.layers import SumLayer
    from pyjuice_b200.autotune import TUNER
    use_graph = ws == 1
    SumLayer.bf16_form = 1
    ms_bf16p, _ = timed({"force_use_bf16": True}, use_graph)
    SumLayer.bf16_form = 3
    ms_fp8, _ = timed({"force_use_bf16": True}, use_graph)
    SumLayer.bf16_form = 2
    ms_bf16, clocks = timed({"force_use_bf16": True}, use_graph, sample_clocks=True)
    ms_fp32, _ = timed({"force_use_fp32": True}, use_graph)
    value = ws * B * args.steps / (ms_bf16 / 1e3)
    value_fp32 = ws * B * args.steps / (ms_fp32 / 1e3)
    value_bf16p = ws * B * args.steps / (ms_bf16p / 1e3)
    value_fp8 = ws * B * args.steps / (ms_fp8 / 1e3)

    # end to end through the public API, host buffers, LLs read back every step
    host = data[:B * 8].pin_memory()
    ll_host = torch.empty([B, 1], dtype=torch.float32).pin_memory()
    e2e_steps = max(3, args.steps // 2)

    # Input pipeline: batch i + 1 is copied (pinned host -> one of two device buffers) on a
    # copy stream while step i computes; a buffer is refilled only after the step that read
    # it has finished.
    copy_stream = torch.cuda.Stream(device=device)
    xbuf = [torch.empty([B, SIDE * SIDE], dtype=host.dtype, device=device) for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]
    free = [torch.cuda.Event() for _ in range(2)]

    def prefetch(i, after=None):
        k = i % 2
        with torch.cuda.stream(copy_stream):
            if after is not None:
                copy_stream.wait_event(after)
            copy_stream.wait_event(free[k])
            xbuf[k].copy_(host[(i % 8) * B:(i % 8 + 1) * B], non_blocking=True)
            copied[k].record(copy_stream)

    def e2e_step(i, last):
        k = i % 2
        torch.cuda.current_stream().wait_event(copied[k])
        if i + 1 < last:
            prefetch(i + 1)
        x = xbuf[k]
        pc.init_param_flows(flows_memory=0.0)
        # the public API's own CUDA-graph option: the inner passes are recorded once, then replayed
        lls = pc(x, force_use_bf16=True, record_cudagraph=True)
        lls.mean().backward()
        allreduce_flows()
        pc.mini_batch_em(step_size=STEP_SIZE, pseudocount=PSEUDOCOUNT)
        ll_host.copy_(lls.detach(), non_blocking=True)
        free[k].record()

    prefetch(0)
    for i in range(2):
        e2e_step(i, 2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    prefetch(0, after=e0)
    for i in range(e2e_steps):
        e2e_step(i, e2e_steps)
    e1.record()
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    if group is not None:
        import torch.distributed as dist
        t = torch.tensor([ms_e2e], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e_value = ws * B * e2e_steps / (ms_e2e / 1e3)

    result = None
    if rank == 0:
        from oracle import pc_oracle as orc
        lay = orc.layout_from_circuit(pc)
        params = pc.params.detach().cpu().numpy().astype(np.float64)
        in_params = pc.input_layer_group[0].params.detach().cpu().numpy().astype(np.float64)
        xs = data[:64]
        _, _, lls_o = orc.forward(lay, params, in_params, xs.numpy())
        with torch.no_grad():
            SumLayer.bf16_form = 1
            l_bp = pc(xs.to(device), force_use_bf16=True).double().cpu().numpy()
            SumLayer.bf16_form = 3
            l_f8 = pc(xs.to(device), force_use_bf16=True).double().cpu().numpy()
            SumLayer.bf16_form = 2
            l_bf = pc(xs.to(device), force_use_bf16=True).double().cpu().numpy()
            l_32 = pc(xs.to(device), force_use_fp32=True).double().cpu().numpy()
        # parameter-flow error of each form against the FP64 oracle (16 samples, unit root flows)
        xp = xs[:16]
        nm_o, ems_o, _ = orc.forward(lay, params, in_params, xp.numpy())
        _, pf_o, ipf_o = orc.backward(lay, params, xp.numpy(), nm_o, ems_o)
        pf_err = {}
        for name, bform, kw in (("bf16_split", 2, {"force_use_bf16": True}), ("bf16_single", 1, {"force_use_bf16": True}),
                                ("e4m3", 3, {"force_use_bf16": True}), ("fp32", 2, {"force_use_fp32": True})):
            SumLayer.bf16_form = bform
            pc.init_param_flows(flows_memory=0.0)
            with torch.no_grad():
                pc(xp.to(device), **kw)
            pc.backward(inputs=xp.to(device), allow_modify_flows=True, force_use_fp32="force_use_fp32" in kw)
            got = pc.param_flows.double().cpu().numpy()
            gin = pc.input_layer_group[0].param_flows.double().cpu().numpy()[:ipf_o.shape[0]]
            pf_err[name] = {"sum_max_rel": float(np.abs(got - pf_o).max() / np.abs(pf_o).max()),
                            "input_max_rel": float(np.abs(gin - ipf_o).max() / np.abs(ipf_o).max())}
        SumLayer.bf16_form = 2
        ll_err = {"bf16_dmean_ll_nats": float(abs(l_bf.mean() - lls_o.mean())),
                  "bf16_mean_abs_dll_nats": float(np.abs(l_bf - lls_o).mean()),
                  "bf16_single_dmean_ll_nats": float(abs(l_bp.mean() - lls_o.mean())),
                  "bf16_single_mean_abs_dll_nats": float(np.abs(l_bp - lls_o).mean()),
                  "e4m3_dmean_ll_nats": float(abs(l_f8.mean() - lls_o.mean())),
                  "e4m3_mean_abs_dll_nats": float(np.abs(l_f8 - lls_o).mean()),
                  "fp32_max_rel_dll": float((np.abs(l_32 - lls_o) / np.abs(lls_o)).max()),
                  "fp32_dmean_ll_nats": float(abs(l_32.mean() - lls_o.mean())),
                  "mean_ll_nats": float(lls_o.mean()), "samples": int(xs.size(0))}
        hbm, tflops, src = peaks()
        # the roofline launches read the buffers of a full-batch step: run one (the error
        # measurements above left buffers of 16 and 64 samples)
        step(data_dev[:B], {"force_use_bf16": True})
        rf = sum_forward_roofline(pc, data_dev[:B], {"force_use_bf16": True})
        big = rf["largest"]
        achieved = big["bytes"] / big["seconds"] / 1e9
        step(data_dev[:B], {"force_use_bf16": True})  # node flows of the full batch (rewritten as log f - log m)
        pf = pflows_roofline(pc)
        achieved = pf["bytes"] / pf["seconds"] / 1e9
        roof = {"kernel": "pcb_sum_pflows (sum_pflows_kernel, split-bf16 form, 64-child tiles) of the largest "
                          "sum layer: the kernel with the largest share of the step",
                "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": PFLOW_TRAFFIC_BYTES,
                "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of this launch, one ncu capture "
                                  "of bench.py --profile-step (-k regex:sum_pflows -s 63 -c 1)",
                "peak_source": f"{src} hbm_gbs (of measured)" if src == "measured" else f"{src} hbm_gbs",
                "alg_bytes_per_launch": pf["bytes"], "us_per_launch": pf["seconds"] * 1e6,
                "tensor_tflops_achieved": pf["flops"] / pf["seconds"] / 1e12,
                "sum_forward_largest_layer": {"us": big["seconds"] * 1e6, "alg_bytes": big["bytes"],
                                              "achieved_gbs": big["bytes"] / big["seconds"] / 1e9,
                                              "frac": big["bytes"] / big["seconds"] / 1e9 / hbm,
                                              "tiles": big["tiles"],
                                              "kernel": "tcgen05 contraction (autotuned: persistent "
                                                        "warp-specialised or CTA-per-slice), weights packed "
                                                        "beforehand",
                                              "pack_us": big["pack_seconds"] * 1e6},
                "all_sum_layers_forward": {"layers": rf["layers"], "us_total": rf["seconds"] * 1e6,
                                           "achieved_gbs": rf["bytes"] / rf["seconds"] / 1e9,
                                           "frac": rf["bytes"] / rf["seconds"] / 1e9 / hbm,
                                           "pack_us_total": rf["pack_seconds"] * 1e6},
                "tc05_choices": {k: list(v) for k, v in TUNER.choices.items() if k.startswith("tc05|")}}
        threads = os.cpu_count() or 1
        torch.set_num_threads(threads)
        v, sample = cpu_step_rate(lay, params, in_params, data, budget_s=15.0, batch=B)
        cpu = {"value": v, "unit": "samples/s", "cores": threads, "kind": "port", "sample": sample}
        result = {
            "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_bf16 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
            "config": {"workload": WORKLOAD, "batch_per_gpu": B, "num_nodes": pc.num_nodes,
                       "num_edges": pc.num_edges, "parallelism": f"dp{ws}" if ws > 1 else "single",
                       "l2": "inputs larger than L2 (node_mars alone is 4*N*B bytes > 126 MB); no flush",
                       "cuda_graph": use_graph},
            "precision_form": "bf16 tensor cores, operands split into bf16 hi + lo (3 MMAs), FP32 accumulate",
            "fp32_plain": {"value": value_fp32, "unit": "samples/s", "ms_per_step": ms_fp32 / args.steps},
            "bf16_single": {"value": value_bf16p, "unit": "samples/s", "ms_per_step": ms_bf16p / args.steps},
            "e4m3": {"value": value_fp8, "unit": "samples/s", "ms_per_step": ms_fp8 / args.steps,
                     "form": "tcgen05 sum contractions (forward, element flows) in e4m3 with per-row weight scales, "
                             "the rest in split bf16"},
            "ll_error_vs_fp64": ll_err,
            "param_flow_rel_err_vs_fp64": {"samples": 16, "measure": "max |pf - pf_fp64| / max |pf_fp64|", **pf_err},
            "e2e": {"value": e2e_value, "unit": "samples/s", "h2d_bytes_per_step": B * SIDE * SIDE * 8,
                    "d2h_bytes_per_step": B * 4},
            "gpu_launches": kernels_per_step * args.steps,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
    if group is not None:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result), flush=True)


if __name__ == "__main__":
    main()
