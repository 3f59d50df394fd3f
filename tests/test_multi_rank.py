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


def _stepping_worker(rank, world, port, out):
    """Each rank builds its own seeded sub-batch of the batched-cavity workload (the smallest simulations of
    its rank's seed, so the CPU oracle steps them in seconds), advances it by two PISO steps, and exchanges
    only the totals (one all_gather outside the stepping)."""
    import time
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench
    import piso_oracle as po
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sides, re = bench.batched_cavity_params(256, bench.rank_seed(rank))
        pick = np.argsort(sides)[:3]
        t0 = time.perf_counter()
        cells = 0
        fingerprint = []
        for i in pick:
            s = int(sides[i])
            d = po.ODomain(2, 1.0 / re[i])
            bi = d.create_block(coords=bench.cavity_coords(s))
            d.close_all(bi)
            d.close_boundary(bi, "-y", np.array([[1.0, 0.0]]))
            d.prepare()
            for _ in range(2):
                po.piso_step(d, 0.5 / s, adv_tol=1e-10, p_tol=1e-10)
            cells += s * s
            fingerprint.append(float(np.abs(d.velocity_global()).sum()))
        ms = (time.perf_counter() - t0) * 1e3
        total, ms_max = bench.job_totals(cells, ms, world, torch.device("cpu"))
        out[rank] = (cells, total, ms, ms_max, tuple(int(sides[i]) for i in pick), tuple(fingerprint))
    finally:
        dist.destroy_process_group()


def test_two_ranks_step_their_own_batches_gloo():
    import random
    world = 2
    port = 29500 + random.randint(2001, 4000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_stepping_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    (c0, t0, ms0, mm0, s0, f0), (c1, t1, ms1, mm1, s1, f1) = res[0], res[1]
    assert t0 == t1 == c0 + c1                 # whole-job cells: every rank's own simulations
    assert mm0 == mm1 == max(ms0, ms1)         # time of the slowest rank
    assert s0 != s1 and f0 != f1               # independent simulations, no shared data
    assert all(np.isfinite(f0)) and all(np.isfinite(f1)) and min(f0 + f1) > 0
