"""Multi-process path: the step does not shard, so N GPUs run N independent
replicas (ensemble members / seeds) and only the timing and the per-replica
results are gathered.  Checked here with world_size 2 on the gloo backend,
each rank running the CPU oracle as its replica."""
import os

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from iwrepo_b200 import config as cf
    from oracle import Oracle, set_threads
    set_threads(1)
    cfg = cf.Config(nx=16, ny=16, nzloc=9, nsubd=3, dt=1e-3).validate()
    o = Oracle(cfg)
    o.init_mode1(0.05, 1e-4, 1000 + rank)  # per-rank seed, as bench.py
    o.step(2)
    ke = torch.tensor([o.diag()["ke"]], dtype=torch.float64)
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)  # stand-in per-rank time
    kes = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(kes, ke)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        q.put(([float(k) for k in kes], float(t)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    kes, tmax = q.get(timeout=120)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert tmax == 2.0  # value is taken over the slowest rank
    assert kes[0] != kes[1]  # different seeds -> independent replicas
    assert np.allclose(kes, kes[0], rtol=1e-3)  # same wave, different noise
