"""The multi-GPU path of bench.py is N independent replicas: every rank steps
its own seeded packing, nothing is exchanged on the data path, and the job
time is the maximum over ranks.  This runs that host logic with two gloo
ranks on CPU, the FP64 oracle standing in for the engine.
"""
import os
import sys
import time

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench
    import pyoracle
    from grains3dgpu_b200 import scenes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    scene = scenes.polydisperse_superquadrics(seed=bench.replica_seed(rank), n=3000)
    s = scenes.System(pyoracle.load_oracle(), scene)
    t0 = time.perf_counter()
    s.step(2)
    elapsed = time.perf_counter() - t0 + 0.05 * rank  # ranks finish at different times
    t_max = bench.max_over_ranks(elapsed, torch, world, "cpu")
    value = bench.aggregate(world, scene.n, 2, t_max)
    first = torch.tensor(scene.transforms[0, 9:], dtype=torch.float64)
    firsts = [torch.zeros(3, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(firsts, first)
    out.put((rank, elapsed, t_max, value, [f.numpy() for f in firsts]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, e0, m0, v0, f0), (_, e1, m1, v1, f1) = res
    assert m0 == m1 == max(e0, e1)              # every rank reports the slowest rank
    assert v0 == v1 == 2 * 3000 * 2 / m0        # whole-job particle-steps/s
    assert not np.allclose(f0[0], f0[1])        # the replicas are different packings
