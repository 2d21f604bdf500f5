"""Data-parallel EM on two CPU ranks (gloo): the flow all-reduce makes the sharded step
equal to the single-process step on the whole batch. Flows are computed by the oracle,
so the host-side exchange logic is tested without a GPU."""

import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_fixture


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    from helpers import build_fixture_circuit, load_fixture_params
    from oracle import pc_oracle as orc
    from pyjuice_b200.distributed import allreduce_param_flows, broadcast_parameters

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        fx = load_fixture("hclt64")
        pc = build_fixture_circuit("hclt64", fx)
        load_fixture_params(pc, fx)
        if rank == 1:
            with torch.no_grad():
                pc.params.mul_(0.0)  # broadcast must restore rank 0's parameters
        broadcast_parameters(pc, src=0)
        lay = orc.layout_from_circuit(pc)
        p = pc.params.detach().numpy().astype(np.float64)
        q = pc.input_layer_group[0].params.detach().numpy().astype(np.float64)
        x = fx["x"][rank * 64:(rank + 1) * 64]
        nm, ems, _ = orc.forward(lay, p, q, x)
        _, pf, ipf = orc.backward(lay, p, x, nm, ems)
        pc.param_flows = torch.from_numpy(pf)
        pc.input_layer_group[0].param_flows = torch.from_numpy(ipf)
        allreduce_param_flows(pc)
        p1, q1 = orc.em_update(lay, p, pc.param_flows.numpy(), q, pc.input_layer_group[0].param_flows.numpy(),
                               0.1, 0.1)
        out_q.put((rank, p1, q1))
    finally:
        dist.destroy_process_group()


def test_two_rank_em_equals_full_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, p1, q1 = q.get(timeout=300)
        res[r] = (p1, q1)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks hold identical parameters after the step
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    # and they equal the single-process step on the union batch
    import sys
    from helpers import build_fixture_circuit, load_fixture_params
    from oracle import pc_oracle as orc
    fx = load_fixture("hclt64")
    pc = build_fixture_circuit("hclt64", fx)
    load_fixture_params(pc, fx)
    lay = orc.layout_from_circuit(pc)
    p = pc.params.detach().numpy().astype(np.float64)
    qq = pc.input_layer_group[0].params.detach().numpy().astype(np.float64)
    x = fx["x"][:128]
    nm, ems, _ = orc.forward(lay, p, qq, x)
    _, pf, ipf = orc.backward(lay, p, x, nm, ems)
    p1, q1 = orc.em_update(lay, p, pf, qq, ipf, 0.1, 0.1)
    assert np.allclose(res[0][0], p1, rtol=1e-10, atol=1e-12)
    assert np.allclose(res[0][1], q1, rtol=1e-10, atol=1e-12)
