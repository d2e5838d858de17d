"""World-size-2 gloo test of the replica path bench.py uses under torchrun:
each rank runs an independent filter (here the CPU oracle stands in for the
device work), timing is reduced as the max over ranks and units as the sum."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    sys.path.insert(0, os.path.join(root, "ssmproblems.jl_b200"))
    import torch
    import oracle as O
    from gfb200 import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    m, ys = W.lgssm_1d(seed=1, T=20)
    om = O.LGModel(m.prior.mu0, m.prior.Sigma0, m.dyn.A, m.dyn.b, m.dyn.Q, m.obs.H, m.obs.c, m.obs.R)
    r = O.pf_run(om, 2048, ys, threshold=0.5, seed=100 + rank)   # replica: own seed
    elapsed = torch.tensor([0.1 * (rank + 1)], dtype=torch.float64)
    dist.all_reduce(elapsed, op=dist.ReduceOp.MAX)
    units = torch.tensor([2048.0 * 20], dtype=torch.float64)
    dist.all_reduce(units, op=dist.ReduceOp.SUM)
    lls = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(lls, torch.tensor([r["ll"]], dtype=torch.float64))
    if rank == 0:
        q.put((float(elapsed.item()), float(units.item()), [float(x.item()) for x in lls]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    elapsed, units, lls = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert elapsed == pytest.approx(0.2)
    assert units == 2 * 2048 * 20
    assert lls[0] != lls[1] and all(np.isfinite(lls))
