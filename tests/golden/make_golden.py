"""Generate the golden fixtures in this directory by running the reference PyJuice.

Run from the repository root in a container that holds the reference sources, with
``PYJUICE_REF_SRC`` set to the reference's ``src`` directory:

    python tests/golden/make_golden.py [tiny] [hclt64] [hclt784]

The reference executes on CPU through Triton's interpreter (``ref_shim.py``) in its
plain FP32 mode (``force_use_fp32=True``). Outputs (``.npz``) hold the compiled index
tensors (or their SHA-256 digests for the large circuit), the initial parameters and
the results of one forward / backward / ``mini_batch_em`` step:

* ``tiny.npz``      the DAG of ``tests/circuits.py:build_tiny_dag`` (partitions, block-sparse
                    edges, pass-through insertion, tied sums and inputs), B = 64;
* ``hclt64.npz``    HCLT, 64 variables x 4 categories, 16 latents, block size 16, B = 512,
                    data from a seeded random tree Bayesian network;
* ``hclt784.npz``   HCLT, 28x28 variables x 256 categories, 128 latents, block size 32:
                    structure, index digests and the log-likelihoods of 8 samples;
* ``em_tiny.npz``    the tiny circuit with a tenth of its parameters zeroed: one step with
                    ``keep_zero_params=True``, and the reference's normalisation of a seeded
                    parameter vector with pseudocount 0.3;
* ``alg_tiny.npz``   the tiny circuit under MPE, GeneralLL(0.5), log-space flows and negated
                    parameter flows: log-likelihoods, node values, node flows, parameter flows;
* ``query_tiny.npz`` the tiny circuit's queries: marginals and the hard-evidence conditional
                    with a per-sample missing mask, the soft-evidence conditional, and
                    input-layer flows with a per-variable missing mask;
* ``io_tiny.npz``    ``.jpc`` files both ways: the bytes of the reference's file of the tiny
                    circuit, and the reference's parameters and log-likelihoods after loading
                    a file saved by pyjuice_b200;
* ``io_dists.npz``  ``.jpc`` files both ways for the four-variable circuit over Bernoulli,
                    Gaussian, DiscreteLogistic and SoftEvidenceCategorical inputs: the bytes of
                    the reference's files, and what the reference loads from ours;
* ``tdp_tiny.npz``   flows of the evidence-free pass (all variables missing) on the tiny
                    circuit: per sample, its top-down probabilities;
* ``structures.npz`` compiled layouts, parameters and log-likelihoods of the reference's PD
                    (3 x 3 grid) and homogeneous HMM (length 6) generators; flows and one EM
                    step of the HMM (tied transitions and emissions);
* ``dists.npz``      Bernoulli, Gaussian and DiscreteLogistic input layers (four-variable
                    circuit): one FP32 forward / backward / EM step;
* ``samples_{tiny,hclt64}.npz``  256 samples the reference's ``queries.sample`` drew on the
                    circuits and parameters of ``tiny.npz`` / ``hclt64.npz`` with every
                    ``tl.rand`` draw replaced by a table lookup by (node, sample)
                    (``ref_shim.install_uniform_table``).
"""

from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ref_shim import load_reference  # noqa: E402

juice = load_reference()
import torch  # noqa: E402
import networkx as nx  # noqa: E402
import pyjuice.nodes.distributions as dists  # noqa: E402
from pyjuice.structures.hclt import mutual_information_chunked, chow_liu_tree  # noqa: E402
from pyjuice.structures.compilation import BayesianTreeToHiddenRegionGraph  # noqa: E402

from circuits import build_tiny_dag  # noqa: E402
from pyjuice_b200.synthetic import gaussian_field_data, tree_bayes_net_data  # noqa: E402


def digest(t: torch.Tensor) -> str:
    return hashlib.sha256(t.detach().cpu().long().contiguous().numpy().tobytes()).hexdigest()


def collect_layout(pc, out: dict, full: bool = True):
    """Index tensors of every layer, flattened into ``out``."""
    gi = 0
    for group in pc.inner_layer_groups:
        for li, layer in enumerate(group):
            pre = f"g{gi}_l{li}_"
            if layer.is_sum():
                names = ["nids", "cids", "pids", "pfids", "chids", "parids", "parpids"]
                out[pre + "nid_range"] = np.array(layer._layer_nid_range)
                out[pre + "pid_range"] = np.array(layer._layer_pid_range)
                out[pre + "pfid_range"] = np.array(layer._layer_pfid_range)
                out[pre + "cs_block_sizes"] = np.array(layer.cs_block_sizes)
            else:
                names = ["nids", "cids", "u_cids", "parids"]
                out[pre + "nid_range"] = np.array(layer._layer_nid_range)
            for n in names:
                tl = getattr(layer, "partitioned_" + n)
                out[pre + n + "_count"] = np.array(len(tl))
                for p, t in enumerate(tl):
                    if full:
                        out[f"{pre}{n}_{p}"] = t.detach().cpu().numpy()
                    else:
                        out[f"{pre}{n}_{p}_sha"] = np.array(digest(t))
                        out[f"{pre}{n}_{p}_shape"] = np.array(tuple(t.shape))
        gi += 1
    il = pc.input_layer_group[0]
    for n in ("vids", "s_pids", "s_pfids", "s_mids", "nids", "source_nids", "node_id2source_id"):
        t = getattr(il, n)
        if full:
            out["in_" + n] = t.detach().cpu().numpy()
        else:
            out["in_" + n + "_sha"] = np.array(digest(t))
    out["num_nodes"] = np.array(pc.num_nodes)
    out["num_elements"] = np.array(pc.num_elements)
    out["num_sum_params"] = np.array(pc.num_sum_params)
    out["num_param_flows"] = np.array(pc.num_param_flows)
    out["num_groups"] = np.array(len(pc.inner_layer_groups))
    out["root_range"] = np.array(pc._root_node_range)


def run_step(pc, x, out: dict, keep_buffers: bool):
    """forward (FP32) -> backward (default flags) -> mini_batch_em(0.1, 0.1)."""
    out["params0"] = pc.params.detach().cpu().numpy().copy()
    out["in_params0"] = pc.input_layer_group[0].params.detach().cpu().numpy().copy()
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, force_use_fp32=True)
    out["lls"] = lls.detach().cpu().numpy()
    if keep_buffers:
        out["node_mars"] = pc.node_mars.detach().cpu().numpy().copy()
    lls.mean().backward()
    if keep_buffers:
        out["node_flows"] = pc.node_flows.detach().cpu().numpy().copy()
    out["param_flows"] = pc.param_flows.detach().cpu().numpy().copy()
    out["in_param_flows"] = pc.input_layer_group[0].param_flows.detach().cpu().numpy().copy()
    pc.mini_batch_em(step_size=0.1, pseudocount=0.1)
    out["params1"] = pc.params.detach().cpu().numpy().copy()
    out["in_params1"] = pc.input_layer_group[0].params.detach().cpu().numpy().copy()


def hclt_tree(x: torch.Tensor, num_bins=32, sigma=0.5 / 32, chunk_size=64):
    mi = mutual_information_chunked(x, x, num_bins, sigma, chunk_size=chunk_size).detach().cpu().numpy()
    T = chow_liu_tree(mi)
    root = nx.center(T)[0]
    clt = nx.bfs_tree(T, root)
    seq = list(nx.dfs_postorder_nodes(T, root))
    children = {int(v): [int(c) for c in clt.successors(v)] for v in clt.nodes}
    return mi, T, root, seq, children


def pack_tree(out, mi, root, seq, children):
    out["tree_mi"] = mi.astype(np.float32)
    out["tree_root"] = np.array(root)
    out["tree_seq"] = np.array(seq)
    ch_flat, ch_off = [], [0]
    for v in range(len(seq)):
        ch_flat.extend(children.get(v, []))
        ch_off.append(len(ch_flat))
    out["tree_children"] = np.array(ch_flat, dtype=np.int64)
    out["tree_children_off"] = np.array(ch_off, dtype=np.int64)


def make_tiny():
    torch.manual_seed(1)
    root = build_tiny_dag(juice, dists)
    pc = juice.compile(root, max_tied_ns_per_parflow_block=1, verbose=False)
    out = {}
    collect_layout(pc, out, full=True)
    gen = torch.Generator().manual_seed(2)
    x = torch.randint(0, 4, (64, 6), generator=gen)
    out["x"] = x.numpy()
    run_step(pc, x, out, keep_buffers=True)
    np.savez_compressed(os.path.join(HERE, "tiny.npz"), **out)


def make_hclt64():
    data = tree_bayes_net_data(num_vars=64, num_cats=4, num_samples=8192, seed=0)
    mi, T, root, seq, children = hclt_tree(data.float())
    torch.manual_seed(3)
    with juice.set_block_size(16):
        r = BayesianTreeToHiddenRegionGraph(T, root, 16, dists.Categorical, {"num_cats": 4}, num_root_ns=1,
                                            block_size=16)
    pc = juice.compile(r, verbose=False)
    out = {}
    pack_tree(out, mi, root, seq, children)
    collect_layout(pc, out, full=True)
    x = data[:512]
    out["x"] = x.numpy()
    run_step(pc, x, out, keep_buffers=False)
    np.savez_compressed(os.path.join(HERE, "hclt64.npz"), **out)


def make_hclt784():
    data = gaussian_field_data(8192, side=28, num_cats=256, length_scale=3.0, seed=0)
    mi, T, root, seq, children = hclt_tree(data.float())
    torch.manual_seed(4)
    r = BayesianTreeToHiddenRegionGraph(T, root, 128, dists.Categorical, {"num_cats": 256}, num_root_ns=1,
                                        block_size=32)
    t = time.time()
    pc = juice.compile(r, verbose=False)
    print("hclt784 compile", time.time() - t, flush=True)
    out = {}
    pack_tree(out, mi, root, seq, children)
    collect_layout(pc, out, full=False)
    # parameters regenerable from a seed (the layouts are identical, see test_compile_golden)
    import pyjuice_b200 as mine
    from pyjuice_b200.nodes.distributions import Categorical
    from pyjuice_b200.structures import hclt_from_tree
    from circuits import seeded_params
    mpc = mine.compile(hclt_from_tree(seq, children, root, 128, input_dist=Categorical(num_cats=256), block_size=32))
    il = pc.input_layer_group[0]
    p, q = seeded_params(mpc._em_pbase.tolist(), mpc._em_nch.tolist(), mpc._em_bs.tolist(), mpc.num_sum_params,
                         il.vids.size(0), 256, seed=784)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(p))
        il.params.copy_(torch.from_numpy(q))
    out["param_seed"] = np.array(784)
    x = data[:8]
    out["x"] = x.numpy()
    t = time.time()
    lls = pc(x, force_use_fp32=True)
    print("hclt784 forward", time.time() - t, flush=True)
    out["lls"] = lls.detach().cpu().numpy()
    np.savez_compressed(os.path.join(HERE, "hclt784.npz"), **out)


def make_em_variants():
    """The tiny circuit with some sum and input parameters set to zero: one forward /
    backward, then ``mini_batch_em(0.1, 0.1, keep_zero_params=True)``; and the reference's
    sum-to-one normalisation (``TensorCircuit._normalize_parameters``, pseudocount 0.3) of a
    seeded positive parameter vector."""
    fx = dict(np.load(os.path.join(HERE, "tiny.npz")))
    torch.manual_seed(1)
    pc = juice.compile(build_tiny_dag(juice, dists), max_tied_ns_per_parflow_block=1, verbose=False)
    p0 = fx["params0"].copy()
    q0 = fx["in_params0"].copy()
    rng = np.random.default_rng(5)
    nd = pc.num_dummy_params
    zs = nd + rng.choice(p0.shape[0] - nd, size=(p0.shape[0] - nd) // 10, replace=False)
    p0[zs] = 0.0
    q0[rng.choice(q0.shape[0], size=q0.shape[0] // 10, replace=False)] = 0.0
    out = dict(params0=p0, in_params0=q0, x=fx["x"])
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(p0))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(q0))
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(torch.from_numpy(fx["x"]), force_use_fp32=True)
    lls.mean().backward()
    out["param_flows"] = pc.param_flows.detach().cpu().numpy().copy()
    out["in_param_flows"] = pc.input_layer_group[0].param_flows.detach().cpu().numpy().copy()
    pc.mini_batch_em(step_size=0.1, pseudocount=0.1, keep_zero_params=True)
    out["params1_keep_zero"] = pc.params.detach().cpu().numpy().copy()
    out["in_params1_keep_zero"] = pc.input_layer_group[0].params.detach().cpu().numpy().copy()
    raw = np.exp(-4.0 * rng.random(p0.shape[0])).astype(np.float32)
    raw[:nd] = 0.0
    t = torch.from_numpy(raw.copy())
    pc._normalize_parameters(t, pseudocount=0.3)
    out["norm_in"] = raw
    out["norm_out"] = t.numpy().copy()
    np.savez_compressed(os.path.join(HERE, "em_tiny.npz"), **out)


def make_alg_variants():
    """The tiny circuit under the other propagation algorithms and flow modes (FP32 forms):
    MPE forward + backward, GeneralLL(alpha = 0.5) forward + backward, log-space LL flows and
    negated LL parameter flows (``allow_modify_flows=False`` throughout)."""
    fx = dict(np.load(os.path.join(HERE, "tiny.npz")))
    torch.manual_seed(1)
    pc = juice.compile(build_tiny_dag(juice, dists), max_tied_ns_per_parflow_block=1, verbose=False)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(fx["params0"]))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(fx["in_params0"]))
    x = torch.from_numpy(fx["x"])
    out = {}
    cases = {"mpe": (dict(propagation_alg="MPE"), dict()),
             "gll": (dict(propagation_alg="GeneralLL", alpha=0.5), dict()),
             "logspace": (dict(), dict(logspace_flows=True)),
             "negate": (dict(), dict(negate_pflows=True))}
    for name, (fw_kw, bw_kw) in cases.items():
        pc.init_param_flows(flows_memory=0.0)
        with torch.no_grad():
            lls = pc(x, force_use_fp32=True, **fw_kw)
        pc.backward(inputs=x, allow_modify_flows=False, force_use_fp32=True, **fw_kw, **bw_kw)
        out[name + "_lls"] = lls.detach().cpu().numpy().copy()
        out[name + "_node_mars"] = pc.node_mars.detach().cpu().numpy().copy()
        out[name + "_node_flows"] = pc.node_flows.detach().cpu().numpy().copy()
        out[name + "_param_flows"] = pc.param_flows.detach().cpu().numpy().copy()
        out[name + "_in_param_flows"] = pc.input_layer_group[0].param_flows.detach().cpu().numpy().copy()
    np.savez_compressed(os.path.join(HERE, "alg_tiny.npz"), **out)


def make_query_variants():
    """Queries on the tiny circuit: marginals with a per-sample missing mask, the conditional
    query with hard evidence (missing mask, target variables) and with soft evidence (rows of
    a seeded Dirichlet(1)), and the input-layer parameter flows of a backward pass with a
    per-variable missing mask."""
    fx = dict(np.load(os.path.join(HERE, "tiny.npz")))
    torch.manual_seed(1)
    pc = juice.compile(build_tiny_dag(juice, dists), max_tied_ns_per_parflow_block=1, verbose=False)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(fx["params0"]))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(fx["in_params0"]))
    x = torch.from_numpy(fx["x"])
    rng = np.random.default_rng(9)
    B, V = x.shape
    mask = rng.random((B, V)) < 0.3
    out = dict(mask=mask)
    out["marginal_lls"] = juice.queries.marginal(pc, data=x, missing_mask=torch.from_numpy(mask)).detach().numpy().copy()
    out["cond_hard"] = juice.queries.conditional(pc, data=x, missing_mask=torch.from_numpy(mask),
                                                 target_vars=[0, 2, 5]).detach().numpy().copy()
    out["cond_hard_full"] = juice.queries.conditional(pc, data=x, missing_mask=torch.from_numpy(mask)).detach().numpy().copy()
    soft = rng.dirichlet(np.ones(4), size=(B, V)).astype(np.float32)
    out["soft"] = soft
    out["cond_soft"] = juice.queries.conditional(pc, data=torch.from_numpy(soft.copy())).detach().numpy().copy()
    out["soft_lls"] = pc.node_mars[pc._root_node_range[0]:pc._root_node_range[1]].detach().numpy().T.copy()
    vmask = np.zeros(V, dtype=bool)
    vmask[[1, 4]] = True
    out["vmask"] = vmask
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, missing_mask=torch.from_numpy(vmask), force_use_fp32=True)
    out["vmask_lls"] = lls.detach().numpy().copy()
    lls.mean().backward()
    out["vmask_param_flows"] = pc.param_flows.detach().numpy().copy()
    out["vmask_in_param_flows"] = pc.input_layer_group[0].param_flows.detach().numpy().copy()
    np.savez_compressed(os.path.join(HERE, "query_tiny.npz"), **out)


def make_io_variants():
    """.jpc files in both directions on the tiny circuit: the reference saves its circuit
    (parameters of tiny.npz; the file bytes are stored), and the reference loads a file that
    pyjuice_b200 saved from its own build of the same circuit and evaluates it (FP32)."""
    import tempfile
    import pyjuice_b200 as mine
    from pyjuice_b200.nodes import distributions as mdists
    fx = dict(np.load(os.path.join(HERE, "tiny.npz")))
    torch.manual_seed(1)
    pc = juice.compile(build_tiny_dag(juice, dists), max_tied_ns_per_parflow_block=1, verbose=False)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(fx["params0"]))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(fx["in_params0"]))
    out = {}
    with tempfile.TemporaryDirectory() as d:
        juice.save(os.path.join(d, "ref.jpc"), pc)
        with open(os.path.join(d, "ref.jpc"), "rb") as f:
            out["ref_jpc"] = np.frombuffer(f.read(), dtype=np.uint8).copy()
        mpc = mine.compile(build_tiny_dag(mine, mdists), max_tied_ns_per_parflow_block=1)
        with torch.no_grad():
            mpc.params.copy_(torch.from_numpy(fx["params0"]))
            mpc.input_layer_group[0].params.copy_(torch.from_numpy(fx["in_params0"]))
        mine.save(os.path.join(d, "ours.jpc"), mpc)
        rpc = juice.compile(juice.load(os.path.join(d, "ours.jpc")), max_tied_ns_per_parflow_block=1, verbose=False)
        out["ref_loads_ours_params"] = rpc.params.detach().cpu().numpy().copy()
        out["ref_loads_ours_lls"] = rpc(torch.from_numpy(fx["x"]), force_use_fp32=True).detach().cpu().numpy().copy()
    np.savez_compressed(os.path.join(HERE, "io_tiny.npz"), **out)


def make_io_dists():
    """.jpc files both ways for circuits.build_dist_dag over each non-Categorical input
    distribution: the reference saves its circuit (input parameters of dists.npz where it has
    them; file bytes stored), and the reference loads the file pyjuice_b200 saved from the
    same circuit and parameters (its parameters stored, and its FP32 log-likelihoods of the
    dists.npz data for the three distributions that need no evidence)."""
    import tempfile
    from circuits import build_dist_dag
    import pyjuice_b200 as mine
    from pyjuice_b200.nodes import distributions as mdists
    dfx = dict(np.load(os.path.join(HERE, "dists.npz")))
    kinds = (("bern", "Bernoulli", {}), ("gauss", "Gaussian", {"mu": 0.0, "sigma": 1.0}),
             ("dlog", "DiscreteLogistic", {"val_range": (-2.0, 2.0), "num_cats": 8}),
             ("poe", "SoftEvidenceCategorical", {"num_cats": 6}))
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, cls, kw in kinds:
            torch.manual_seed(11)
            pc = juice.compile(build_dist_dag(juice, lambda: getattr(dists, cls)(**kw)), verbose=False)
            if name + "_in_params0" in dfx:
                with torch.no_grad():
                    pc.params.copy_(torch.from_numpy(dfx[name + "_params0"]))
                    pc.input_layer_group[0].params.copy_(torch.from_numpy(dfx[name + "_in_params0"]))
            out[name + "_params"] = pc.params.detach().numpy().copy()
            out[name + "_in_params"] = pc.input_layer_group[0].params.detach().numpy().copy()
            juice.save(os.path.join(d, name + "_ref.jpc"), pc)
            with open(os.path.join(d, name + "_ref.jpc"), "rb") as f:
                out[name + "_ref_jpc"] = np.frombuffer(f.read(), dtype=np.uint8).copy()
            torch.manual_seed(11)
            mpc = mine.compile(build_dist_dag(mine, lambda: getattr(mdists, cls)(**kw)))
            with torch.no_grad():
                mpc.params.copy_(torch.from_numpy(out[name + "_params"]))
                mpc.input_layer_group[0].params.copy_(torch.from_numpy(out[name + "_in_params"]))
            mine.save(os.path.join(d, name + "_ours.jpc"), mpc)
            rpc = juice.compile(juice.load(os.path.join(d, name + "_ours.jpc")), verbose=False)
            out[name + "_ref_loads_ours_params"] = rpc.params.detach().numpy().copy()
            out[name + "_ref_loads_ours_in_params"] = rpc.input_layer_group[0].params.detach().numpy().copy()
            if name != "poe":
                x = torch.from_numpy(dfx[name + "_x"])
                out[name + "_ref_loads_ours_lls"] = rpc(x, force_use_fp32=True).detach().numpy().copy()
    np.savez_compressed(os.path.join(HERE, "io_dists.npz"), **out)


def make_tdp_variants():
    """Flows of the evidence-free pass on the tiny circuit: every variable missing, root flow
    1 per sample (``pc(x, missing_mask=all)``, ``lls.mean().backward()``). Per sample these are
    the top-down probabilities that ``eval_top_down_probs`` computes; that function itself
    (and ``mini_batch_em(step_size_rescaling=True)``, which calls it) ends in a
    segmentation fault under Triton's CPU interpreter, so its own outputs cannot be
    recorded here."""
    fx = dict(np.load(os.path.join(HERE, "tiny.npz")))
    torch.manual_seed(1)
    pc = juice.compile(build_tiny_dag(juice, dists), max_tied_ns_per_parflow_block=1, verbose=False)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(fx["params0"]))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(fx["in_params0"]))
    x = torch.from_numpy(fx["x"][:4])
    out = {}
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, missing_mask=torch.ones(x.shape[1], dtype=torch.bool), force_use_fp32=True)
    out["lls"] = lls.detach().numpy().copy()
    lls.mean().backward()
    out["node_flows"] = pc.node_flows.detach().numpy().copy()
    out["param_flows"] = pc.param_flows.detach().numpy().copy()
    out["in_param_flows"] = pc.input_layer_group[0].param_flows.detach().numpy().copy()
    np.savez_compressed(os.path.join(HERE, "tdp_tiny.npz"), **out)


def make_structures():
    """Compiled layouts of the reference's PD and HMM generators, with parameters and the
    FP32 log-likelihoods of seeded data:
    * PD over a 3 x 3 grid, split interval 1, 32 latents (block size 16), 4 categories, at
      most 2 product blocks per sum block (so the random block choice is exercised), seed 7;
    * a homogeneous HMM of length 6, 32 latents, 10 symbols, seeded Dirichlet(1) alpha /
      beta / gamma (tied transition and emission vectors)."""
    from pyjuice.structures import PD, HMM
    out = {}
    torch.manual_seed(7)
    root = PD((3, 3), 32, split_intervals=1, max_prod_block_conns=2, input_node_params={"num_cats": 4})
    torch.manual_seed(8)
    pc = juice.compile(root, verbose=False)
    lay = {}
    collect_layout(pc, lay, full=True)
    out.update({"pd_" + k: v for k, v in lay.items()})
    out["pd_params"] = pc.params.detach().numpy().copy()
    out["pd_in_params"] = pc.input_layer_group[0].params.detach().numpy().copy()
    x = torch.from_numpy(np.random.default_rng(1).integers(0, 4, size=(16, 9)))
    out["pd_x"] = x.numpy()
    out["pd_lls"] = pc(x, force_use_fp32=True).detach().numpy().copy()
    rng = np.random.default_rng(2)
    alpha = torch.from_numpy(rng.dirichlet(np.ones(32), size=32).astype(np.float32))
    beta = torch.from_numpy(rng.dirichlet(np.ones(10), size=32).astype(np.float32))
    gamma = torch.from_numpy(rng.dirichlet(np.ones(32)).astype(np.float32))
    out["hmm_alpha"], out["hmm_beta"], out["hmm_gamma"] = alpha.numpy(), beta.numpy(), gamma.numpy()
    torch.manual_seed(9)
    pc = juice.compile(HMM(6, 32, 10, homogeneous=True, alpha=alpha, beta=beta, gamma=gamma), verbose=False)
    lay = {}
    collect_layout(pc, lay, full=True)
    out.update({"hmm_" + k: v for k, v in lay.items()})
    out["hmm_params"] = pc.params.detach().numpy().copy()
    out["hmm_in_params"] = pc.input_layer_group[0].params.detach().numpy().copy()
    x = torch.from_numpy(rng.integers(0, 10, size=(16, 6)))
    out["hmm_x"] = x.numpy()
    pc.init_param_flows(flows_memory=0.0)
    lls = pc(x, force_use_fp32=True)
    out["hmm_lls"] = lls.detach().numpy().copy()
    lls.mean().backward()
    out["hmm_param_flows"] = pc.param_flows.detach().numpy().copy()
    out["hmm_in_param_flows"] = pc.input_layer_group[0].param_flows.detach().numpy().copy()
    pc.mini_batch_em(step_size=0.5, pseudocount=0.01)
    out["hmm_params1"] = pc.params.detach().numpy().copy()
    out["hmm_in_params1"] = pc.input_layer_group[0].params.detach().numpy().copy()
    np.savez_compressed(os.path.join(HERE, "structures.npz"), **out)


def make_dist_variants():
    """Bernoulli, Gaussian and DiscreteLogistic input layers on a four-variable circuit
    (circuits.build_dist_dag): FP32 forward, backward and mini_batch_em(0.3, 0.1) by the
    reference, with seeded parameters and data (bool data for Bernoulli, N(0, 1.5) data for
    Gaussian, bin indices 0..7 for DiscreteLogistic over 8 bins of [-2, 2])."""
    from circuits import build_dist_dag
    out = {}
    rng = np.random.default_rng(21)
    for name, factory, data in (
            ("bern", lambda: dists.Bernoulli(), torch.from_numpy(rng.random((32, 4)) < 0.4)),
            ("gauss", lambda: dists.Gaussian(mu=0.0, sigma=1.0),
             torch.from_numpy((1.5 * rng.standard_normal((32, 4))).astype(np.float32))),
            ("dlog", lambda: dists.DiscreteLogistic(val_range=(-2.0, 2.0), num_cats=8),
             torch.from_numpy(rng.integers(0, 8, size=(32, 4)).astype(np.float32)))):
        torch.manual_seed(11)
        pc = juice.compile(build_dist_dag(juice, factory), verbose=False)
        out[name + "_params0"] = pc.params.detach().numpy().copy()
        out[name + "_in_params0"] = pc.input_layer_group[0].params.detach().numpy().copy()
        out[name + "_x"] = data.numpy()
        pc.init_param_flows(flows_memory=0.0)
        lls = pc(data, force_use_fp32=True)
        out[name + "_lls"] = lls.detach().numpy().copy()
        lls.mean().backward()
        out[name + "_param_flows"] = pc.param_flows.detach().numpy().copy()
        out[name + "_in_param_flows"] = pc.input_layer_group[0].param_flows.detach().numpy().copy()
        pc.mini_batch_em(step_size=0.3, pseudocount=0.1)
        out[name + "_params1"] = pc.params.detach().numpy().copy()
        out[name + "_in_params1"] = pc.input_layer_group[0].params.detach().numpy().copy()
    np.savez_compressed(os.path.join(HERE, "dists.npz"), **out)


SAMPLE_SEED = 20261204  # seed of the uniform table (oracle.pc_oracle.uniform_table)
SAMPLE_S = 256


def make_samples(name: str):
    """Samples the reference draws when every ``tl.rand`` draw of node n in sample s is
    ``uniform_table(SAMPLE_SEED)[n, s]``: the circuit and parameters of fixture ``name``,
    ``juice.queries.sample(pc, SAMPLE_S)``."""
    from ref_shim import install_uniform_table
    from oracle import pc_oracle as orc
    fx = dict(np.load(os.path.join(HERE, name + ".npz")))
    if name == "tiny":
        torch.manual_seed(1)
        root = build_tiny_dag(juice, dists)
        pc = juice.compile(root, max_tied_ns_per_parflow_block=1, verbose=False)
    else:
        seq = [int(v) for v in fx["tree_seq"]]
        off, flat = fx["tree_children_off"], fx["tree_children"]
        T = nx.Graph()
        T.add_nodes_from(range(len(seq)))
        for v in range(len(seq)):
            for c in flat[off[v]:off[v + 1]]:
                T.add_edge(v, int(c))
        with juice.set_block_size(16):
            r = BayesianTreeToHiddenRegionGraph(T, int(fx["tree_root"]), 16, dists.Categorical, {"num_cats": 4},
                                                num_root_ns=1, block_size=16)
        pc = juice.compile(r, verbose=False)
    with torch.no_grad():
        pc.params.copy_(torch.from_numpy(fx["params0"]))
        pc.input_layer_group[0].params.copy_(torch.from_numpy(fx["in_params0"]))
    table = orc.uniform_table(SAMPLE_SEED, pc.num_nodes, SAMPLE_S)
    install_uniform_table(juice, table)
    samples = juice.queries.sample(pc, SAMPLE_S)
    out = dict(uniform_seed=np.array(SAMPLE_SEED), num_samples=np.array(SAMPLE_S),
               samples=samples.detach().cpu().numpy().astype(np.int64), num_nodes=np.array(pc.num_nodes))
    np.savez_compressed(os.path.join(HERE, f"samples_{name}.npz"), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["tiny", "hclt64", "hclt784", "samples_tiny", "samples_hclt64", "em_tiny", "alg_tiny", "query_tiny", "io_tiny", "tdp_tiny", "structures", "dists", "io_dists"]
    for w in which:
        t = time.time()
        {"tiny": make_tiny, "hclt64": make_hclt64, "hclt784": make_hclt784,
         "samples_tiny": lambda: make_samples("tiny"), "samples_hclt64": lambda: make_samples("hclt64"),
         "em_tiny": make_em_variants, "alg_tiny": make_alg_variants, "query_tiny": make_query_variants,
         "io_tiny": make_io_variants, "tdp_tiny": make_tdp_variants, "structures": make_structures,
         "dists": make_dist_variants, "io_dists": make_io_dists}[w]()
        print(w, "done in", round(time.time() - t, 1), "s", flush=True)
