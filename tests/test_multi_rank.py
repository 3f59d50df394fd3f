"""Multi-rank logic of bench.py on CPU: two gloo ranks (world size 2) on 127.0.0.1.

Each rank owns an independent batch (its own seed, so disjoint simulations and no data-path
collective); the whole-job figures are the sum of the ranks' cells and the max of their elapsed
times, exchanged once outside the timed region.
"""
import os
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sides, re = bench.batched_cavity_params(256, bench.rank_seed(rank))
        cells = int(np.sum(sides.astype(np.int64) ** 2))
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        total, ms_max = bench.job_totals(cells, ms, world, torch.device("cpu"))
        out[rank] = (cells, total, ms_max, tuple(int(s) for s in sides[:8]))
    finally:
        dist.destroy_process_group()


def test_two_rank_job_totals_gloo():
    import random
    world = 2
    port = 29500 + random.randint(0, 2000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    (c0, t0, m0, s0), (c1, t1, m1, s1) = res[0], res[1]
    assert t0 == t1 == c0 + c1          # whole-job cells
    assert m0 == m1 == 15.0             # max over ranks
    assert s0 != s1                     # independent batches per rank


def test_single_rank_totals_are_local():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_totals(123, 4.5, 1, torch.device("cpu")) == (123, 4.5)
    assert bench.rank_seed(0) == 6
