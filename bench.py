"""Benchmark of the B200 PISO step: cell-steps/s of a batched workload (one JSON line on rank 0).

Workloads (``--workload``):

* ``batched_cavities_256`` (default): 256 independent 2D lid-driven cavities, side
  s_i = round(exp(U(ln 32, ln 256))) (seed 6), Re_i = exp(U(ln 100, ln 5000)), viscosity 1/Re_i,
  lid speed 1, unit box, dt_i = 0.5 h_i (CFL 0.5), 2 correctors, BiCGStab advection and CG pressure
  solves to 1e-6 (RMS residual), FP32 fields with FP64 Krylov reductions, all simulations advanced
  by one launch per stage and the step replayed as a CUDA graph.
* ``lid_cavity_64``: the reference's minimal lid-driven cavity, 64x64, Re 1000, dt 0.01.

A "step" is one PISO time step of every simulation in the workload; ``value`` is the whole-job
throughput in cell-steps/s with all state resident in HBM.  ``e2e`` measures the same step through
the public API with the state uploaded from pinned host buffers and downloaded again every step.
``--impl reference`` times the reference algorithm's CPU restatement (the FP64 oracle; the reference
itself has no CPU implementation of the step) on a bounded sample of the same workload.

Multi-GPU (torchrun): every rank advances its own batch (seed + rank), no collective on the data
path ("weak" scaling); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "PISO cell-steps/s fwd & fwd+bwd, batched vs plain, at stated err, 1 B200"


# ------------------------------------------------------------------------------------------ workloads

def cavity_coords(n):
    xs = np.linspace(0.0, 1.0, n + 1)
    Y, X = np.meshgrid(xs, xs, indexing="ij")
    return np.stack([X, Y])[None]


def batched_cavity_params(num=256, seed=6):
    rng = np.random.default_rng(seed)
    sides = np.rint(np.exp(rng.uniform(np.log(32), np.log(256), num))).astype(int)
    re = np.exp(rng.uniform(np.log(100), np.log(5000), num))
    return sides, re


def make_cavity_domain(n, viscosity, dtype, device="cuda"):
    import torch
    from pict_b200 import PISOtorch
    dom = PISOtorch.Domain(2, torch.tensor([viscosity], dtype=dtype), name="cavity%d" % n, dtype=dtype,
                           device=device, passiveScalarChannels=0)
    coords = torch.tensor(cavity_coords(n), dtype=dtype, device=device).contiguous()
    blk = dom.CreateBlock(vertexCoordinates=coords, name="cavity")
    blk.CloseAllBoundaries()
    blk.CloseBoundary("-y", torch.tensor([[1.0, 0.0]], dtype=dtype, device=device))
    dom.PrepareSolve()
    return dom


def extras_pass():
    """Device time of the operators around the step, CUDA events over 20 calls after 3 warm-ups, FP32: the
    Smagorinsky viscosity and the passive scalar matrix / right-hand side on a 1024^2 cavity (seeded
    velocity and scalar), and a 3x3 multi-block convolution (16 -> 16 channels, batch 4) over a 2x2 grid of
    connected 512^2 blocks (its padding gather and the convolutions)."""
    import torch
    from pict_b200 import PISOtorch as P
    from pict_b200.multiblock_cnn import MultiblockConv
    dt, dev, n = torch.float32, "cuda", 1024
    dom = P.Domain(2, torch.tensor([1e-3], dtype=dt), name="extras", dtype=dt, device=torch.device(dev),
                   passiveScalarChannels=1)
    g = torch.Generator().manual_seed(0)
    vel = (torch.rand((1, 2, n, n), generator=g) - 0.5).to(dev, dt).contiguous()
    sc = torch.rand((1, 1, n, n), generator=g).to(dev, dt).contiguous()
    coords = torch.tensor(cavity_coords(n), dtype=dt, device=dev).contiguous()
    blk = dom.CreateBlock(velocity=vel, passiveScalar=sc, vertexCoordinates=coords, name="cavity")
    blk.CloseAllBoundaries()
    dom.PrepareSolve()
    ts = torch.tensor([0.5 / n], dtype=dt)
    coef = torch.tensor([0.17 ** 2], dtype=dt)

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    for key, fn in [("sgs_smagorinsky", lambda: P.SGSviscosityIncompressibleSmagorinsky(dom, coef)),
                    ("scalar_matrix", lambda: P.SetupAdvectionMatrix(dom, ts, 0, True, 0)),
                    ("scalar_rhs", lambda: P.SetupAdvectionScalar(dom, ts, 0))]:
        ms = timed(fn)
        out[key] = {"ms": ms, "cells": n * n, "cells_per_s": n * n / (ms * 1e-3)}
    m = 512
    grid = P.Domain(2, torch.tensor([1e-3], dtype=dt), name="grid", dtype=dt, device=torch.device(dev),
                    passiveScalarChannels=0)
    bl = [grid.CreateBlockWithSize(P.Int4(m, m, 1, 2), name="b%d" % i) for i in range(4)]
    for b in bl:
        b.CloseAllBoundaries()
    bl[0].ConnectBlock("+x", bl[1], "-x", "-y")
    bl[0].ConnectBlock("+y", bl[2], "-y", "-x")
    bl[1].ConnectBlock("+y", bl[3], "-y", "-x")
    bl[2].ConnectBlock("+x", bl[3], "-x", "-y")
    conv = MultiblockConv(grid, "ZERO", 16, 16, 3, device=dev, dtype=dt)
    xs = [torch.randn((4, 16, m, m), generator=g).to(dev) for _ in range(4)]
    with torch.no_grad():
        ms_pad = timed(lambda: conv.pad(xs))
        ms_all = timed(lambda: conv(xs))
    out["multiblock_conv"] = {"ms": ms_all, "ms_padding": ms_pad, "cells": 4 * m * m, "batch": 4, "channels": 16,
                              "cells_per_s": 4 * 4 * m * m / (ms_all * 1e-3)}
    print(json.dumps({"extras": out, "dtype": "f32", "unit": "ms per call"}), flush=True)


def channel_arrays(nx, ny, nz, seed=2, stretch=2.0, u_center=20.0, amp=0.1, modes=12):
    """3D channel on [0, 4 pi] x [-1, 1] x [0, 4 pi / 3]: vertex coordinates [1, 3, nz+1, ny+1, nx+1]
    (uniform in x and z, tanh-stretched in y with factor `stretch`) and the initial velocity
    [1, 3, nz, ny, nx]: laminar profile u = u_center (1 - y^2) plus the curl of a seeded random vector
    potential (`modes` Fourier modes in x and z times (1 - y^2)^2, vanishing at the walls), scaled to
    `amp` * u_center."""
    rng = np.random.default_rng(seed)
    lx, lz = 4 * np.pi, 4 * np.pi / 3
    xv = np.linspace(0, lx, nx + 1)
    s = np.linspace(-1.0, 1.0, ny + 1)
    yv = np.tanh(stretch * s) / np.tanh(stretch)
    zv = np.linspace(0, lz, nz + 1)
    Z, Y, X = np.meshgrid(zv, yv, xv, indexing="ij")
    coords = np.stack([X, Y, Z])[None]
    xc, yc, zc = 0.5 * (xv[1:] + xv[:-1]), 0.5 * (yv[1:] + yv[:-1]), 0.5 * (zv[1:] + zv[:-1])
    Zc, Yc, Xc = np.meshgrid(zc, yc, xc, indexing="ij")
    w = (1 - Yc ** 2) ** 2
    dw = -4 * Yc * (1 - Yc ** 2)
    dpsi = np.zeros((3, 3) + Xc.shape)  # dpsi[c][axis]
    for c in range(3):
        for _ in range(modes):
            kx = 2 * np.pi / lx * rng.integers(1, 5)
            kz = 2 * np.pi / lz * rng.integers(1, 5)
            a, ph = rng.standard_normal(), rng.uniform(0, 2 * np.pi)
            arg = kx * Xc + kz * Zc + ph
            dpsi[c][0] += -a * kx * np.sin(arg) * w
            dpsi[c][1] += a * np.cos(arg) * dw
            dpsi[c][2] += -a * kz * np.sin(arg) * w
    up = np.stack([dpsi[2][1] - dpsi[1][2], dpsi[0][2] - dpsi[2][0], dpsi[1][0] - dpsi[0][1]])
    up *= amp * u_center / max(np.abs(up).max(), 1e-30)
    vel = up.copy()
    vel[0] += u_center * (1 - Yc ** 2)
    return coords, vel[None]


def make_channel_domain(nx, ny, nz, dtype, device="cuda", viscosity=1.0 / 180.0):
    """Periodic channel (x, z periodic, no-slip walls at y = +-1) driven by the constant pressure
    gradient 1 (u_tau = 1, Re_tau = 1 / viscosity) as a static velocity source."""
    import torch
    from pict_b200 import PISOtorch
    coords, vel = channel_arrays(nx, ny, nz)
    dom = PISOtorch.Domain(3, torch.tensor([viscosity], dtype=dtype), name="channel", dtype=dtype,
                           device=device, passiveScalarChannels=0)
    blk = dom.CreateBlock(velocity=torch.tensor(vel, dtype=dtype, device=device).contiguous(),
                          vertexCoordinates=torch.tensor(coords, dtype=dtype, device=device).contiguous(),
                          name="channel")
    blk.MakePeriodic("x")
    blk.MakePeriodic("z")
    blk.CloseBoundary("-y")
    blk.CloseBoundary("+y")
    blk.setVelocitySource(torch.tensor([[1.0, 0.0, 0.0]], dtype=dtype, device=device))
    dom.PrepareSolve()
    return dom


def channel_dt(nx, u_center=20.0):
    return 0.5 * (4 * np.pi / nx) / u_center


def build_workload(name, rank=0, dtype=None):
    import torch
    dtype = torch.float32 if dtype is None else dtype
    if name == "batched_cavities_256":
        sides, re = batched_cavity_params(256, rank_seed(rank))
        doms = [make_cavity_domain(int(s), 1.0 / r, dtype) for s, r in zip(sides, re)]
        dts = [0.5 / s for s in sides]
        return dict(domains=doms, dts=dts, sides=sides, re=re, tol=1e-6, correctors=2, refine_tol=5e-10, adv_tol=5e-7)
    if name == "lid_cavity_64":
        doms = [make_cavity_domain(64, 1e-3, dtype)]
        return dict(domains=doms, dts=[0.01], sides=np.array([64]), re=np.array([1000.0]), tol=1e-6, correctors=2)
    if name == "channel3d_192":
        doms = [make_channel_domain(192, 96, 96, dtype)]
        return dict(domains=doms, dts=[channel_dt(192)], sides=None, re=None, tol=1e-6, correctors=2,
                    kind="channel", refine_tol=1e-10)
    raise KeyError(name)


# ------------------------------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.m = 0

    def start(self, wait=5.0):
        """Start sampling every 50 ms and wait (up to `wait` s) for the first sample, so that the timed region
        that follows is covered."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < wait:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.m = len(self.lines)

    def need(self, k=2):
        """True while fewer than k samples were read since the timed region started."""
        return self.proc is not None and len(self.lines) - self.m < k

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.m:]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def keep_busy(sampler, work, limit_s=3.0):
    """After a timed region shorter than the sampling interval: repeat untimed `work` (the same steps) until
    two clock samples under load were read, so the clocks reported are those of the loaded GPU."""
    import torch
    t0 = time.time()
    while sampler.need(2) and time.time() - t0 < limit_s:
        work()
        torch.cuda.synchronize()


# ------------------------------------------------------------------------------------------ helpers

def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def oracle_step_rate(sides, re, dts, n_sims, steps, tol=1e-6):
    """Time the FP64 oracle PISO step on the first `n_sims` simulations (CPU, single thread)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import piso_oracle as po
    cells = 0
    t_total = 0.0
    for s, r, dt in list(zip(sides, re, dts))[:n_sims]:
        d = po.ODomain(2, 1.0 / r)
        b = d.create_block(coords=cavity_coords(int(s)))
        d.close_all(b)
        d.close_boundary(b, "-y", np.array([[1.0, 0.0]]))
        d.prepare()
        po.piso_step(d, dt, adv_tol=tol, p_tol=tol)  # warm-up step (not timed)
        t0 = time.perf_counter()
        for _ in range(steps):
            po.piso_step(d, dt, adv_tol=tol, p_tol=tol)
        t_total += time.perf_counter() - t0
        cells += int(s) * int(s) * steps
    return cells / t_total, t_total, cells


def _oracle_cavity_worker(side, re, dt, steps, tol, barrier, queue):
    """One process of oracle_parallel_rate: builds its cavity, takes one untimed step, waits for the
    others, then times `steps` FP64 oracle steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import piso_oracle as po
    d = po.ODomain(2, 1.0 / re)
    b = d.create_block(coords=cavity_coords(int(side)))
    d.close_all(b)
    d.close_boundary(b, "-y", np.array([[1.0, 0.0]]))
    d.prepare()
    po.piso_step(d, dt, adv_tol=tol, p_tol=tol)
    barrier.wait(timeout=600)
    t0 = time.perf_counter()
    for _ in range(steps):
        po.piso_step(d, dt, adv_tol=tol, p_tol=tol)
    queue.put((int(side) * int(side) * steps, time.perf_counter() - t0))


def oracle_parallel_rate(sides, re, dts, steps, procs, tol=1e-6):
    """The FP64 oracle on several host cores: one process per simulation (spawned, one BLAS thread each),
    all timed together after a barrier, each taking about the same number of cell-steps (at least `steps`
    steps).  Returns (cell-steps/s over the wall time of the slowest process, that wall time, cell-steps)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    n = min(len(sides), procs)
    barrier = ctx.Barrier(n)
    queue = ctx.Queue()
    # every process gets about the same work: the largest simulation takes `steps` steps, smaller ones
    # proportionally more, so that the cores stay busy until the end of the timed region
    cmax = max(int(sides[i]) ** 2 for i in range(n))
    nsteps = [max(steps, int(round(steps * cmax / int(sides[i]) ** 2))) for i in range(n)]
    ps = [ctx.Process(target=_oracle_cavity_worker, args=(int(sides[i]), float(re[i]), float(dts[i]), nsteps[i], tol,
                                                          barrier, queue)) for i in range(n)]
    for p in ps:
        p.start()
    res = [queue.get(timeout=1800) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    cells = sum(c for c, _ in res)
    wall = max(t for _, t in res)
    return cells / wall, wall, cells


def sample_indices(sides, k):
    """k simulations at evenly spaced size quantiles (a representative bounded sample)."""
    order = np.argsort(sides)
    if len(order) <= k:
        return order
    q = [(j + 0.5) / k for j in range(k)]
    return order[[int(x * len(order)) for x in q]]


def precision_kwargs(args, wl=None):
    """mixed: FP32 stencils / vectors, FP64 reductions and one FP64 refinement sweep of every pressure
    solve to an RMS residual of 1e-9, pressure solves warm-started from the latest pressure and (unless
    --warm-advection 0) advection solves from the current velocity; fp32: the single FP32 pressure solve
    from zero (the reference's order)."""
    if args.precision == "mixed":
        rt = getattr(args, "refine_tol", 0.0) or (wl or {}).get("refine_tol", 1e-9)
        return {"pressure_refine": 1, "refine_tol": rt,
                "warm_start_pressure": "increment" if getattr(args, "warm_pressure", 2) == 2 else True,
                "refine_solver": args.refine_solver, "pressure_first_solve": bool(args.first_solve),
                "mg_iterations": args.mg_iterations,
                "warm_start_advection": "increment" if args.warm_advection == 2 else bool(args.warm_advection)}
    return {}


def adv_tol(args, wl):
    """RMS residual target of the advection solves: --adv-tol, else (mixed precision) the workload's adv_tol,
    else its solver tolerance."""
    if getattr(args, "adv_tol", 0.0):
        return args.adv_tol
    if args.precision == "mixed" and wl.get("adv_tol"):
        return wl["adv_tol"]
    return wl["tol"]


def rank_seed(rank):
    """Seed of rank r's batch: every rank advances its own independent simulations."""
    return 6 + rank


def job_totals(cells, ms, world, device):
    """(cells of all ranks, max elapsed ms over ranks): one all_gather outside the timed region."""
    import torch
    if world <= 1:
        return cells, ms
    import torch.distributed as dist
    mine = torch.tensor([float(cells), float(ms)], dtype=torch.float64, device=device)
    allv = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(allv, mine)
    allv = torch.stack(allv).cpu()
    return int(allv[:, 0].sum().item()), float(allv[:, 1].max().item())


# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) over algorithmic bytes of one captured
# launch of the batched workload (profiles/k_cg1_batched_cavities_256.md)
# ncu DRAM bytes / algorithmic bytes on captured launches (profiles/), per solver group: the persistent
# CG on the channel, the finest-level multigrid PCG kernels and k_bicgstab on the cavity batch
NCU_TRAFFIC_RATIO = {"cg": 14.27e9 / 20.12e9, "mg": 420.2e6 / 477.0e6, "bicg": 3.205e9 / 4.424e9}


def cg_algorithmic_bytes(dims, esz):
    """Algorithmic bytes per cell and CG iteration: read K coefficients, r, p_old; write p_new, q
    (phase 1); read x, p, q, r; write x, r (phase 2)."""
    K = 2 * dims + 1
    return esz * (K + 10)


# ------------------------------------------------------------------------------------------ arms

def run_reference(args, rank, world):
    if rank != 0:
        return
    w = args.workload
    if w == "channel3d_192":
        times, cells = [], 0
        for _ in range(args.steps):
            rate, t, c = oracle_channel_rate(48, 24, 24, 1)
            times.append(t)
            cells = c
        value = cells * len(times) / sum(times)
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w, "sample": "channel 48x24x24 (1/4 resolution), one PISO step per timed step"},
            "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": 1, "kind": "port",
                             "sample": "channel 48x24x24 x %d steps, FP64 NumPy/SciPy restatement" % args.steps},
            "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    if w == "cylinder_street":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import piso_oracle as po
        from pict_b200.cylinder_street import TIME_STEP, street_spec
        spec = street_spec()
        od = _oracle_street(po, spec)
        for _ in range(args.warmup):
            po.advective_outflow(od, spec["outflow"], spec["char_vel"], TIME_STEP, tol=1e-5)
            po.piso_step(od, TIME_STEP, adv_tol=1e-6, p_tol=1e-6)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            po.advective_outflow(od, spec["outflow"], spec["char_vel"], TIME_STEP, tol=1e-5)
            po.piso_step(od, TIME_STEP, adv_tol=1e-6, p_tol=1e-6)
            times.append(time.perf_counter() - t0)
        value = od.N * len(times) / sum(times)
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w, "sample": "the full street, one PISO step with the outflow update per timed step"},
            "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": 1, "kind": "port",
                             "sample": "full street x %d steps, FP64 NumPy/SciPy restatement" % args.steps},
            "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    if w == "batched_cavities_256":
        sides, re = batched_cavity_params(256, 6)
        dts = [0.5 / s for s in sides]
    else:
        sides, re, dts = np.array([64]), np.array([1000.0]), [0.01]
    # bounded sample on every host core (up to 64): one simulation per core at evenly spaced size quantiles,
    # each process taking `steps` oracle steps of its simulation, all timed together
    procs = max(1, min(os.cpu_count() or 1, 64))
    sel = sample_indices(sides, procs)
    value, wall, cells = oracle_parallel_rate(sides[sel], re[sel], [dts[i] for i in sel], args.steps, procs)
    n_sample = min(len(sel), procs)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w, "sample": "%d simulations at size quantiles (sides %d..%d), one process each, "
                                            "%d PISO steps of the largest and as many cell-steps in the others" % (
                                                n_sample, int(min(sides[sel])), int(max(sides[sel])), args.steps)},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": n_sample, "kind": "port",
                         "sample": "%d simulations x %d steps in %d processes, FP64 NumPy/SciPy restatement "
                                   "(the reference has no CPU implementation of the step)" % (
                                       n_sample, args.steps, n_sample)},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_pict(args, rank, world):
    import torch
    import torch.distributed as dist
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    wl = build_workload(args.workload, rank)
    doms = wl["domains"]
    batch = BatchDomain(doms, time_steps=wl["dts"])
    batch.pack_state()  # block fields as views of two contiguous tensors: one host copy per field
    kw = dict(time_step=float(wl["dts"][0]), corrector_steps=wl["correctors"], advection_tol=adv_tol(args, wl),
              pressure_tol=wl["tol"], max_iterations=5000, **precision_kwargs(args, wl))
    tuned = None
    if args.autotune:
        from pict_b200.autotune import autotune
        best, table = autotune(batch, kw)
        kw.update(p_group_size=best["p_group_size"], adv_group_size=best["adv_group_size"],
                  cg_variant=best["cg_variant"])
        tuned = {"best": {k: best[k] for k in ("tile_cells", "p_group_size", "cg_variant", "ms_per_step")},
                 "candidates": len(table)}
    else:
        kw.update(p_group_size=args.group_size, adv_group_size=args.group_size)
    st = PISOStepper(batch, **kw)
    cells = batch.getTotalSize()
    # warm-up (eager), then capture one step as a CUDA graph; the algorithmic bytes of every warm-up
    # CG launch are recorded so that an ncu capture of launch k (-k regex:k_cg -s k -c 1) can be set
    # against them (the step is deterministic)
    esz = 4 if batch.getDtype() == torch.float32 else 8
    per_cell = cg_algorithmic_bytes(batch.getSpatialDims(), esz)
    n_s = np.diff(batch._sim_cells.cpu().numpy())
    warm_cg_bytes = []
    for _ in range(args.warmup):
        st.step()
        _, p_inf = st.check()
        for p in p_inf:
            its = np.array([i.usedIterations for i in p])
            warm_cg_bytes.append(float(np.sum((its + 1) * n_s) * per_cell))
    torch.cuda.synchronize()
    G = graph_steps(args)
    if not args.no_graph:
        st.capture(steps=G)
    torch.cuda.synchronize()

    def run_steps(k):
        if args.no_graph:
            for _ in range(k):
                st.step()
        else:
            for _ in range(k // G):
                st.replay()

    run_steps(max(args.warmup, 3) * G)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(dev.index)
    sampler.start()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("piso_timed_steps")  # lets a profiler select exactly the timed launches
    e0.record()
    run_steps(args.steps)
    e1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    keep_busy(sampler, lambda: run_steps(G))
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    adv_infos, p_infos = st.check()
    total_cells, ms_max = job_totals(cells, ms, world, dev)
    value = total_cells * args.steps / (ms_max * 1e-3)

    # roofline of the dominant kernel (persistent CG): eager pass with events around each CG launch
    roof = roofline_pass(st, batch, args, dev)
    roof["warmup_launch_algorithmic_bytes"] = warm_cg_bytes

    # end-to-end through the public API with host buffers (a one-step graph: the state crosses the
    # host between steps)
    if not args.no_graph and G != 1:
        st.capture(steps=1)
    e2e = e2e_pass(st, batch, args, dev, cells, world)

    # the same batched step in plain FP32 (pressure solves from zero to the workload tolerance, no
    # refinement): faster, at the error reported under fp32_step.err
    cavities = wl.get("kind", "cavity") == "cavity"
    fp32 = fp32_pass(batch, wl, args, dev, cells, world) if (args.precision == "mixed" and not args.skip_fp32
                                                            and cavities) else None

    # forward + backward (adjoint) through the checkpointed rollout
    fb = fwd_bwd_pass(st, batch, args, dev, cells, world) if (not args.skip_bwd and cavities) else None

    # plain: the same step one simulation at a time (single-domain stepper, CUDA graph), sampled
    plain = plain_pass(wl, args) if (rank == 0 and not args.skip_plain and cavities) else None

    # accuracy: two smallest simulations, FP32 GPU vs FP64 oracle with tight solves; adjoint vs FD
    if rank == 0 and not args.skip_err:
        err = accuracy_check(wl, args) if cavities else channel_accuracy_check(wl, args)
    else:
        err = None
    if err is not None and not args.skip_bwd and cavities:
        err["viscosity_grad"] = grad_check(wl)
        err["viscosity_grad_timed_precision"] = grad_check_mixed(wl, args)

    # the reference's own CUDA build on this GPU (stock operators, one simulation at a time)
    ref_cuda = reference_cuda_pass(wl) if (rank == 0 and not args.skip_ref_cuda and cavities) else None

    # the other configurations, timed briefly so that their throughput is in this line
    extras = extras_pass_default(args) if (rank == 0 and not args.skip_extras and cavities) else None

    # CPU baseline (bounded sample, rank 0)
    cpu = None
    if rank == 0 and not args.skip_cpu and not cavities:
        rate, tt, c = oracle_channel_rate(48, 24, 24, 1)
        cpu = {"value": rate, "unit": "cell-steps/s", "cores": 1, "kind": "port",
               "sample": "channel 48x24x24 (same setup at 1/4 resolution), 1 PISO step (FP64 NumPy/SciPy "
                         "restatement, %.1f s)" % tt}
    elif rank == 0 and not args.skip_cpu:
        sel = sample_indices(wl["sides"], 4)
        n_s = len(sel)
        rate, tt, c = oracle_step_rate(wl["sides"][sel], wl["re"][sel], [wl["dts"][i] for i in sel], n_s, 2)
        cpu = {"value": rate, "unit": "cell-steps/s", "cores": 1, "kind": "port",
               "sample": "sides %s x 2 PISO steps each (FP64 NumPy/SciPy restatement, %.1f s)" % (
                   [int(wl["sides"][i]) for i in sel], tt)}
    iters_ref = [[max(i.usedIterations for i in r) for r in row] for row in st.refine_infos()]
    # RMS residual of the FP32 correction solve relative to its right-hand side is what the iteration cap bounds
    res_ref = [[max(float(i.finalResidual) for i in r) for r in row] for row in st.refine_infos()]
    iters_adv = [i.usedIterations for i in adv_infos]
    iters_p = [[i.usedIterations for i in p] for p in p_infos]
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "simulations": len(doms), "cells_per_gpu": cells,
                       "pass": "forward", "solver_tol": wl["tol"], "advection_tol": st.adv_tol,
                       "correctors": wl["correctors"],
                       "precision": args.precision + (" (FP32 fields and Krylov vectors, FP64 reductions, one FP64 "
                                                      "refinement sweep of each pressure solve to %g RMS (multigrid-preconditioned CG corrections on near-isotropic grids, at most %d iterations, each system stopping at the target), warm-started pressure solves" % (st.refine_tol, st.mg_iterations) + (" (later correctors from the previous corrector's pressure plus the previous step's corrector increment)" if st.pressure_increment else "") + (", advection solves from the current velocity plus the previous step's advection increment" if args.warm_advection == 2 else (", advection solves from the current velocity" if args.warm_advection else "")) + ")"
                                                      if args.precision == "mixed" else " (FP32, FP64 reductions)"),
                       "cuda_graph": not args.no_graph, "cuda_graph_steps": None if args.no_graph else G,
                       "l2": "working set > L2 (126 MB), no flush",
                       "autotune": tuned, "tile_cells": batch.tile_cells,
                       "parallelism": "independent batches per GPU" if world > 1 else "single GPU"},
            "clocks": clocks,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "fwd_bwd": fb,
            "fp32_step": fp32,
            "plain": plain,
            "reference_cuda": ref_cuda,
            "extras": extras,
            "gpu_launches": st.kernels_per_step() * args.steps,
            "err": err,
            "solver_iterations": {"advection_max": int(max(iters_adv)), "advection_mean": float(np.mean(iters_adv)),
                                  "pressure_max": [int(max(p)) for p in iters_p],
                                  "pressure_mean": [float(np.mean(p)) for p in iters_p],
                                  "refinement_max": iters_ref, "refinement_final_residual_max": res_ref},
        }
        print(json.dumps(line), flush=True)


def graph_steps(args):
    """Steps per captured CUDA graph: --graph-steps when it divides --steps, else 1."""
    g = max(1, int(args.graph_steps))
    return g if args.steps % g == 0 else 1


def street_stepper(dtype=None, tol=1e-6, graph=0, warm=False):
    """The full cylinder street (27,648 cells, FP32), projected to a divergence-free start through the
    drop-in Simulation, and its fused stepper with the device outflow update; the solves start from zero
    like the reference's driver.  warm: the pressure solves start from the latest pressure and the advection
    solves from the velocity plus the extrapolated increment (same tolerances; about 65 instead of 200 CG
    iterations per correction, but the FP32 pressure then ends 2.3e-2 instead of 5.0e-3 from the FP64
    oracle after 10 steps: the absolute 1e-6 tolerance leaves more of the warm start's smooth error)."""
    import torch
    from pict_b200.cylinder_street import TIME_STEP, build_street, street_prep_fn, street_spec
    from pict_b200.engine import PISOStepper
    from pict_b200.PISOtorch_simulation import Simulation
    dom, info = build_street(street_spec(), dtype=torch.float32 if dtype is None else dtype)
    sim = Simulation(domain=dom, time_step=TIME_STEP, prep_fn=street_prep_fn(info), corrector_steps=2,
                     advection_tol=tol, pressure_tol=tol, non_orthogonal=False)
    sim.make_divergence_free()
    warm_kw = dict(warm_start_pressure=True, warm_start_advection="increment") if warm else {}
    st = PISOStepper(dom, time_step=TIME_STEP, advection_tol=tol, pressure_tol=tol, outflow=info["outflow"],
                     outflow_velocity=info["char_vel"], **warm_kw)
    return dom, info, st


def _graph_rate(st, cells, steps, g):
    import torch
    for _ in range(3):
        st.step()
    st.check()
    st.capture(steps=g)
    st.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps // g):
        st.replay()
    e1.record()
    torch.cuda.synchronize()
    st.check()
    ms = e0.elapsed_time(e1)
    return cells * steps / (ms * 1e-3), ms / steps


def extras_pass_default(args):
    """Brief timings of the other configurations on this GPU (CUDA events over graph replays):
    the cylinder street (FP32, 200 steps) and the 192 x 96 x 96 channel (this run's precision, 10 steps)."""
    import torch
    out = {}
    dom, info, st = street_stepper()
    rate, ms = _graph_rate(st, dom.getTotalSize(), 200, 50)
    out["cylinder_street"] = {"value": rate, "unit": "cell-steps/s", "ms_per_step": ms, "cells": dom.getTotalSize(),
                              "steps": 200, "precision": "FP32, FP64 reductions, solves to 1e-6 from zero",
                              "workload": "bench.py --workload cylinder_street"}
    del st, dom
    dom, info, st = street_stepper(warm=True)
    rate, ms = _graph_rate(st, dom.getTotalSize(), 200, 50)
    out["cylinder_street_warm_start"] = {"value": rate, "unit": "cell-steps/s", "ms_per_step": ms, "steps": 200,
                                         "precision": "FP32, FP64 reductions, solves to 1e-6 from warm starts "
                                                      "(pressure 2.3e-2 from the FP64 oracle after 10 steps, "
                                                      "5.0e-3 from zero)"}
    del st, dom
    wl = build_workload("channel3d_192")
    d = wl["domains"][0]
    from pict_b200.engine import PISOStepper
    st = PISOStepper(d, time_step=float(wl["dts"][0]), corrector_steps=wl["correctors"], advection_tol=wl["tol"],
                     pressure_tol=wl["tol"], max_iterations=5000, **precision_kwargs(args, wl))
    rate, ms = _graph_rate(st, d.getTotalSize(), 10, 5)
    out["channel3d_192"] = {"value": rate, "unit": "cell-steps/s", "ms_per_step": ms, "cells": d.getTotalSize(),
                            "steps": 10, "precision": args.precision + ", pressure refined to %g" % wl["refine_tol"],
                            "workload": "bench.py --workload channel3d_192"}
    del st, d, wl
    torch.cuda.empty_cache()
    return out


def run_street(args, rank, world):
    """The cylinder street as its own bench line: the fused FP32 step with the device outflow update,
    replayed as a CUDA graph; e2e with every block's velocity and pressure through pinned host buffers
    each step; roofline of the solver groups; error against the FP64 oracle after 10 steps; CPU baseline
    of the oracle step; optionally the Strouhal number from a longer run."""
    import torch
    import torch.distributed as dist
    from pict_b200.cylinder_street import TIME_STEP, build_street, cylinder_forces, street_spec, strouhal
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    dom, info, st = street_stepper()
    cells = dom.getTotalSize()
    for _ in range(args.warmup):
        st.step()
    st.check()
    G = graph_steps(args)
    if not args.no_graph:
        st.capture(steps=G)

    def run_steps(k):
        if args.no_graph:
            for _ in range(k):
                st.step()
        else:
            for _ in range(k // G):
                st.replay()

    run_steps(3 * G)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(dev.index)
    sampler.start()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    run_steps(args.steps)
    e1.record()
    torch.cuda.synchronize()
    keep_busy(sampler, lambda: run_steps(G))
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    adv, ps = st.check()
    ms = e0.elapsed_time(e1)
    total_cells, ms_max = job_totals(cells, ms, world, dev)
    value = total_cells * args.steps / (ms_max * 1e-3)
    roof = roofline_pass(st, dom, args, dev)
    # e2e: all block fields in and out through pinned host buffers every step
    if not args.no_graph and G != 1:
        st.capture(steps=1)
    dev_state = [t for b in dom.getBlocks() for t in (b.velocity, b.pressure)]
    host_state = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in dev_state]
    for h, t in zip(host_state, dev_state):
        h.copy_(t)
    torch.cuda.synchronize()
    nbytes = sum(h.numel() * h.element_size() for h in host_state)
    k = max(1, min(args.steps, 50))
    e0.record()
    for _ in range(k):
        for h, t in zip(host_state, dev_state):
            t.copy_(h, non_blocking=True)
        st.step() if args.no_graph else st.replay()
        for h, t in zip(host_state, dev_state):
            h.copy_(t, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_cells, e2e_ms = job_totals(cells, e0.elapsed_time(e1), world, dev)
    e2e = {"value": e2e_cells * k / (e2e_ms * 1e-3), "unit": "cell-steps/s", "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": nbytes, "steps": k}
    shedding = None
    if args.shedding_steps > 0 and rank == 0:
        lift, drag = [], []
        for s in range(args.shedding_steps // 10):
            for _ in range(10):
                st.step()
            fx, fy = cylinder_forces(dom, info)
            drag.append(fx)
            lift.append(fy)
        st.check()
        stn = strouhal(lift, TIME_STEP, every=10)
        shedding = {"steps": args.shedding_steps, "strouhal": stn, "drag_coefficient_mean_last_half":
                    float(2 * np.mean(drag[len(drag) // 2:])), "lift_coefficient_amplitude_last_half":
                    float(2 * (np.max(lift[len(lift) // 2:]) - np.min(lift[len(lift) // 2:])) / 2)}
    err = cpu = None
    if rank == 0 and not args.skip_err:
        err = street_accuracy_check()
    if rank == 0 and not args.skip_cpu:
        cpu = street_oracle_rate()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "cylinder_street", "cells_per_gpu": cells, "blocks": dom.getNumBlocks(),
                           "pass": "forward", "solver_tol": 1e-6, "correctors": 2, "dt": TIME_STEP,
                           "precision": "FP32 fields and Krylov vectors, FP64 reductions, solves from zero",
                           "cuda_graph": not args.no_graph, "cuda_graph_steps": None if args.no_graph else G,
                           "l2": "working set < L2: latency-bound, no flush (inputs re-read from L2)",
                           "parallelism": "independent replicas per GPU" if world > 1 else "single GPU"},
                "clocks": clocks, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "err": err,
                "shedding": shedding, "gpu_launches": st.kernels_per_step() * args.steps,
                "solver_iterations": {"advection_max": int(max(i.usedIterations for i in adv)),
                                      "pressure_max": [int(max(i.usedIterations for i in p)) for p in ps]}}
        print(json.dumps(line), flush=True)


def street_accuracy_check(steps=10):
    """FP32 street step against the FP64 oracle (1e-10 solves: tighter ones stall at the FP64 floor of the
    full street's pressure system) on the full street after `steps` steps from the same projected state."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import piso_oracle as po
    from pict_b200.cylinder_street import TIME_STEP, street_spec
    spec = street_spec()
    dom, info, st = street_stepper()
    od = _oracle_street(po, spec)
    u = np.concatenate([b.velocity.double().cpu().numpy().reshape(2, -1) for b in dom.getBlocks()], axis=1)
    od.set_velocity_global(u)
    ob, of = info["outflow"][0]
    od.blocks[ob].boundaries[of].velocity = dom.getBlock(ob).getBoundary(of).velocity.double().cpu().numpy()
    for _ in range(steps):
        st.step()
        po.advective_outflow(od, info["outflow"], spec["char_vel"], TIME_STEP, tol=1e-5)
        po.piso_step(od, TIME_STEP, adv_tol=1e-10, p_tol=1e-10)
    st.check()
    u = np.concatenate([b.velocity.double().cpu().numpy().reshape(2, -1) for b in dom.getBlocks()], axis=1)
    p = np.concatenate([b.pressure.double().cpu().numpy().reshape(-1) for b in dom.getBlocks()])
    ur, pr = od.velocity_global(), od.pressure_global()
    return {"steps": steps, "velocity_rel_max": float(np.abs(u - ur).max() / np.abs(ur).max()),
            "pressure_rel_max": float(np.abs(p - pr).max() / np.abs(pr).max()),
            "reference": "FP64 oracle, solver tol 1e-10, from the same projected state"}


def _oracle_street(po, spec):
    od = po.ODomain(2, spec["viscosity"])
    for b in spec["blocks"]:
        od.create_block(coords=b["coords"], velocity=b["velocity"])
    for op in spec["ops"]:
        if op[0] == "close_all":
            od.close_all(op[1])
        elif op[0] == "connect":
            od.connect(op[1], op[2], op[3], op[4], *op[5:])
        elif op[0] == "close":
            od.close_boundary(op[1], op[2], op[3])
    od.prepare()
    return od


def street_oracle_rate(steps=2):
    """FP64 oracle steps of the full street (CPU, one core), tolerances as the GPU step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import piso_oracle as po
    from pict_b200.cylinder_street import TIME_STEP, street_spec
    spec = street_spec()
    od = _oracle_street(po, spec)
    po.advective_outflow(od, spec["outflow"], spec["char_vel"], TIME_STEP, tol=1e-5)
    po.piso_step(od, TIME_STEP, adv_tol=1e-6, p_tol=1e-6)
    t0 = time.perf_counter()
    for _ in range(steps):
        po.advective_outflow(od, spec["outflow"], spec["char_vel"], TIME_STEP, tol=1e-5)
        po.piso_step(od, TIME_STEP, adv_tol=1e-6, p_tol=1e-6)
    t = time.perf_counter() - t0
    n = od.N
    return {"value": n * steps / t, "unit": "cell-steps/s", "cores": 1, "kind": "port",
            "sample": "full street, %d PISO steps with the outflow update (FP64 NumPy/SciPy restatement, %.1f s)" % (steps, t)}


def solver_bytes_per_cell(kind, dims, esz, nrhs=1):
    """Algorithmic bytes per cell and iteration (each array once per pass at minimal fused traffic).

    cg: read K coefficients, r, w, s, p, x; write x, p, s, r, w.
    bicg: per component 2K + 17 values (two stencil sweeps and the vector updates of one iteration).
    mg: one preconditioned CG iteration as the fused kernels move it on the finest level: SpMV with
        the direction update (read K coefficients, z, p_old; write p, q: K + 4), restriction with the
        x/r update (read r, q, x, p, K coefficients; write r, x and the coarse right-hand side:
        K + 6 + 2^-D), prolongation with post-smoothing and the r.z partials (read K coefficients, r,
        the coarse iterate; write z: K + 2 + 2^-D); every coarser level restricts (K + 1 + 2^-D) and
        prolongs (K + 2 + 2^-D), the coarse levels summing to 1/3 (2D) or 1/7 (3D) of the finest.
    """
    K = 2 * dims + 1
    if kind == "cg":
        return esz * (K + 10)
    if kind == "bicg":
        return esz * (2 * K + 17) * nrhs
    c = 0.5 ** dims
    coarse = 1.0 / 3.0 if dims == 2 else 1.0 / 7.0
    return esz * ((K + 4) + (K + 6 + c) + (K + 2 + c) + coarse * ((K + 1 + c) + (K + 2 + c)))


def roofline_pass(st, batch, args, dev):
    """Per solver group (persistent BiCGStab, persistent CG, multigrid PCG): algorithmic bytes of the
    launches (iterations x cells of each system x bytes per cell and iteration) over their CUDA-event
    time.  The group with the largest time is reported as the dominant kernel."""
    import torch
    from pict_b200 import PISOtorch as P
    esz = 4 if batch.getDtype() == torch.float32 else 8
    D = batch.getSpatialDims()
    steps = max(1, min(args.steps, 5))
    events = [st.step_with_events() for _ in range(steps)]
    torch.cuda.synchronize()
    n_s = np.diff(batch._sim_cells.cpu().numpy())
    peak, kind_peak = measured_peaks()
    groups = {}
    for evs in events:
        for kind, lst in evs.items():
            g = groups.setdefault(kind, {"ms": 0.0, "bytes": 0.0, "launches": 0})
            for (a, b, info) in lst:
                g["ms"] += a.elapsed_time(b)
                infos = P.decode_infos(info)
                if kind == "bicg":
                    its = np.array([i.usedIterations for i in infos]).reshape(-1, D).max(axis=1)
                    per = solver_bytes_per_cell("bicg", D, esz, nrhs=D)
                else:
                    its = np.array([i.usedIterations for i in infos])
                    per = solver_bytes_per_cell(kind, D, esz)
                g["bytes"] += float(np.sum((np.maximum(its, 0) + 1) * n_s) * per)
                g["launches"] += 1
    if st._mg is not None and "mg" in groups and groups["mg"]["launches"] > 0:
        # the multigrid solve is ~400 short launches: time it as a captured CUDA graph, as it runs in the
        # step's graph (eager timing would measure launch overhead)
        ss = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        run = lambda: st._mg.solve(st.desc, st._res, st._corr, st.mg_iterations, st.refine_tol, st.info_r[0][0],
                                   st._mg_ws, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            run()
        torch.cuda.current_stream().wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            run()
        graph.replay()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 5
        e0.record()
        for _ in range(reps):
            graph.replay()
        e1.record()
        torch.cuda.synchronize()
        ms1 = e0.elapsed_time(e1) / reps
        g = groups["mg"]
        per_launch_bytes = g["bytes"] / g["launches"]
        g["eager_ms"] = g["ms"]
        g["ms"] = ms1 * g["launches"]
        del graph
    names = {"cg": "k_cg1" if st.p_params.variant == 1 else "k_cg", "bicg": "k_bicgstab",
             "mg": "multigrid PCG (k_mg_* V-cycle + k_pcg_* kernels)"}
    table = []
    for kind, g in groups.items():
        if g["launches"] == 0 or g["ms"] <= 0:
            continue
        ach = g["bytes"] / (g["ms"] * 1e-3) / 1e9
        table.append({"kernel": names[kind], "group": kind, "ms_per_step": g["ms"] / steps,
                      "achieved": ach, "frac": ach / peak,
                      "algorithmic_bytes_per_launch": g["bytes"] / g["launches"],
                      "avg_launch_ms": g["ms"] / g["launches"],
                      "bytes_per_cell_iteration": solver_bytes_per_cell(kind, D, esz, nrhs=D)})
    table.sort(key=lambda r: -r["ms_per_step"])
    top = dict(table[0])
    ratio = NCU_TRAFFIC_RATIO.get(top["group"])
    top.update({"bound": "hbm", "peak": peak, "peak_kind": kind_peak, "unit": "GB/s",
                "traffic": None if ratio is None else ratio * top["algorithmic_bytes_per_launch"],
                "traffic_note": None if ratio is None else
                "ncu dram bytes / algorithmic bytes on one captured launch (profiles/), scaled to the average launch",
                "groups": table})
    return top


def e2e_pass(st, batch, args, dev, cells, world, chunks=8):
    """The step with the batch state crossing the host every step: each step's result (all blocks' velocity
    and pressure) is read back into pinned host buffers, and the next step's input is uploaded from them.
    The state moves in `chunks` slices per field: the upload of a slice for the next step starts as soon as
    its download is done, on a second stream, so uploads overlap the remaining downloads (PCIe is full
    duplex); the step waits for every upload."""
    import torch
    # the batch state (all blocks' velocity and pressure) lives in two contiguous device tensors
    # (BatchDomain.pack_state), so each direction is `chunks` copies per field per step
    dev_state = [batch.velocity_arena, batch.pressure_arena]
    host_state = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in dev_state]
    for h, t in zip(host_state, dev_state):
        h.copy_(t)
    torch.cuda.synchronize()
    h2d = sum(h.numel() * h.element_size() for h in host_state)
    pieces = []
    for h, t in zip(host_state, dev_state):
        hv, tv = h.view(-1), t.view(-1)
        n = tv.numel()
        for a in range(chunks):
            sl = slice(a * n // chunks, (a + 1) * n // chunks)
            pieces.append((hv[sl], tv[sl]))
    main = torch.cuda.current_stream()
    up = torch.cuda.Stream()
    steps = max(1, min(args.steps, 20))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for h, t in pieces:
        t.copy_(h, non_blocking=True)
    for k in range(steps):
        if args.no_graph:
            st.step()
        else:
            st.replay()
        downs = []
        for h, t in pieces:
            h.copy_(t, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(main)
            downs.append(ev)
        if k + 1 < steps:
            with torch.cuda.stream(up):
                for (h, t), ev in zip(pieces, downs):
                    up.wait_event(ev)
                    t.copy_(h, non_blocking=True)
            main.wait_stream(up)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    total_cells, ms_max = job_totals(cells, ms, world, dev)
    return {"value": total_cells * steps / (ms_max * 1e-3), "unit": "cell-steps/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": h2d, "steps": steps,
            "copies": "%d slices per field and direction; uploads on a second stream overlap the downloads" % chunks}


def fp32_pass(batch, wl, args, dev, cells, world):
    import torch
    from pict_b200.engine import PISOStepper
    blocks = batch.getBlocks()
    saved = [(b.velocity.clone(), b.pressure.clone()) for b in blocks]
    st = PISOStepper(batch, time_step=float(wl["dts"][0]), corrector_steps=wl["correctors"], advection_tol=wl["tol"],
                     pressure_tol=wl["tol"], max_iterations=5000)
    for _ in range(3):
        st.step()
    st.capture(steps=1)
    for _ in range(3):
        st.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        st.replay()
    e1.record()
    torch.cuda.synchronize()
    st.check()
    ms = e0.elapsed_time(e1)
    for b, (v, p) in zip(blocks, saved):
        b.velocity.copy_(v)
        b.pressure.copy_(p)
    total_cells, ms_max = job_totals(cells, ms, world, dev)
    out = {"value": total_cells * args.steps / (ms_max * 1e-3), "unit": "cell-steps/s",
           "ms_per_step": ms_max / args.steps, "precision": "FP32, FP64 reductions, pressure solves from zero to %g" % wl["tol"]}
    if not args.skip_err:
        a = argparse.Namespace(**vars(args))
        a.precision = "fp32"
        out["err"] = accuracy_check(wl, a)
    return out


def adjoint_pressure_tol(batch, st):
    """Relative tolerance of the transposed pressure solves of the timed forward+backward: the forward
    pressure tolerance.  Where the stepper has no multigrid hierarchy the adjoint solve is the plain FP32 CG,
    which levels off between 1e-6 and 9e-5 on the largest cavities, so it stops at 1e-5 in FP32 there; the
    multigrid solve is refined in FP64 and reaches the forward tolerance."""
    import torch
    if st._mg is None and batch.getDtype() == torch.float32:
        return max(st.p_tol, 1e-5)
    return st.p_tol


def fwd_bwd_pass(st, batch, args, dev, cells, world):
    """Forward + backward of a checkpointed rollout: loss = mean over simulations of the final mean
    kinetic energy, gradient with respect to the initial velocity and every simulation's viscosity.

    Timed with the transposed solves relative to their right-hand sides (advection to the forward tolerance,
    pressure to adjoint_pressure_tol; the configuration whose gradient error err.viscosity_grad_timed_precision
    reports), and again with the
    reference's backward semantics (the same tolerances as absolute RMS residuals: for a loss this small
    the adjoint solves then stop almost at once, so that number is faster and less accurate)."""
    import torch
    from pict_b200 import PISOtorch as P
    from pict_b200.adjoint import PISOAdjoint, rollout
    R, K = args.fb_steps, args.checkpoint
    D = batch.getSpatialDims()
    n_s = torch.diff(batch._sim_cells.long()).to(dev)
    ns = n_s.numel()
    w = torch.repeat_interleave(1.0 / (ns * n_s.to(batch.getDtype())), n_s).repeat(D)
    rel = PISOAdjoint(st, relative_tolerance=True, adjoint_pressure_tol=adjoint_pressure_tol(batch, st))
    u0 = rel.velocity().clone()
    nu0 = batch._sim_visc.clone()

    def timed(adj):
        adj.use_graph = not args.no_graph

        def run():
            u0r = u0.clone().requires_grad_(True)
            nur = nu0.clone().requires_grad_(True)
            out = rollout(adj, u0r, R, [R], checkpoint_every=K, nu=nur)
            loss = 0.5 * (w * out[0] * out[0]).sum()
            loss.backward()
            return nur.grad

        run()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        g = run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        infos = P.decode_infos(adj.info)
        adv, pr = infos[:D * ns], infos[D * ns:]
        adj.set_velocity(u0)
        batch._sim_visc.copy_(nu0)
        total_cells, ms_max = job_totals(cells, ms, world, dev)
        return ms_max, total_cells, bool(torch.isfinite(g).all()), {
            "advection_max": int(max(i.usedIterations for i in adv)),
            "advection_mean": float(np.mean([i.usedIterations for i in adv])),
            "pressure_max": int(max(i.usedIterations for i in pr)),
            "pressure_mean": float(np.mean([i.usedIterations for i in pr]))}

    ms_max, total_cells, finite, its = timed(rel)
    ms_abs, _, _, its_abs = timed(PISOAdjoint(st))
    return {"value": total_cells * R / (ms_max * 1e-3), "unit": "cell-steps/s", "steps": R, "checkpoint_every": K,
            "ms": ms_max, "loss": "mean over simulations of the final mean kinetic energy",
            "adjoint_solves": "relative to their right-hand sides: advection to the forward tolerance %g, pressure "
                              "to %g by %s" % (rel.adv_params.tolerance, rel.p_tol, "multigrid-preconditioned CG"
                                               if rel.p_mg else "persistent CG"),
            "adjoint_iterations_last_step": its,
            "grad": "initial velocity and per-simulation viscosity", "grad_finite": finite,
            "absolute_adjoint_tolerances": {
                "value": total_cells * R / (ms_abs * 1e-3), "unit": "cell-steps/s", "ms": ms_abs,
                "adjoint_iterations_last_step": its_abs,
                "note": "the reference's backward semantics: the same tolerances as absolute RMS residuals"}}


def plain_pass(wl, args, k=8, steps=10, fb_steps=10, checkpoint=5):
    """The plain single-simulation FP32 step as the reference runs it: one domain per simulation, FP32
    with FP64 reductions, advection and pressure solves from zero to the workload tolerance, no
    refinement (CUDA graph), on k simulations at evenly spaced size quantiles, one after the other:
    sum(cells x steps) / sum(time).  Also the same simulations' forward + backward (checkpointed rollout
    of fb_steps steps, loss = final mean kinetic energy, gradient w.r.t. the initial velocity and the
    viscosity), and the plain step with this build's mixed precision for comparison."""
    import torch
    from pict_b200.adjoint import PISOAdjoint, rollout
    from pict_b200.engine import PISOStepper
    sel = sample_indices(wl["sides"], k)
    res = {}
    for mode in ("fp32", "mixed"):
        tot_cells, tot_ms, fb_cells, fb_ms = 0, 0.0, 0, 0.0
        for i in sel:
            s = int(wl["sides"][i])
            d = make_cavity_domain(s, 1.0 / wl["re"][i], torch.float32)
            kw = precision_kwargs(args, wl) if mode == "mixed" else {}
            stp = PISOStepper(d, time_step=float(wl["dts"][i]), advection_tol=wl["tol"], pressure_tol=wl["tol"], **kw)
            for _ in range(3):
                stp.step()
            stp.capture(steps=1)
            for _ in range(3):
                stp.replay()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                stp.replay()
            e1.record()
            torch.cuda.synchronize()
            stp.check()
            tot_ms += e0.elapsed_time(e1)
            tot_cells += s * s * steps
            if mode == "fp32" and not args.skip_bwd:
                adj = PISOAdjoint(stp)
                adj.use_graph = not args.no_graph
                u0 = adj.velocity().clone()
                nu0 = d._sim_visc.clone()
                w = 1.0 / (s * s)

                def run():
                    u0r = u0.clone().requires_grad_(True)
                    nur = nu0.clone().requires_grad_(True)
                    out = rollout(adj, u0r, fb_steps, [fb_steps], checkpoint_every=checkpoint, nu=nur)
                    (0.5 * w * (out[0] * out[0]).sum()).backward()
                run()
                torch.cuda.synchronize()
                e0.record()
                run()
                e1.record()
                torch.cuda.synchronize()
                fb_ms += e0.elapsed_time(e1)
                fb_cells += s * s * fb_steps
                adj.set_velocity(u0)
            del stp, d
        res[mode] = (tot_cells / (tot_ms * 1e-3), fb_cells / (fb_ms * 1e-3) if fb_ms > 0 else None)
    sample = "sides %s, one simulation at a time (its own domain and CUDA graph)" % [int(wl["sides"][i]) for i in sel]
    out = {"value": res["fp32"][0], "unit": "cell-steps/s", "steps": steps, "sample": sample,
           "precision": "FP32 fields and Krylov vectors, FP64 reductions, solves from zero to %g, no refinement" % wl["tol"],
           "fwd_bwd": None if res["fp32"][1] is None else
           {"value": res["fp32"][1], "unit": "cell-steps/s", "steps": fb_steps, "checkpoint_every": checkpoint,
            "loss": "final mean kinetic energy", "grad": "initial velocity and viscosity"},
           "mixed": {"value": res["mixed"][0], "unit": "cell-steps/s",
                     "precision": "this build's mixed precision (FP64 refinement of the pressure solves)"}}
    return out


def reference_cuda_pass(wl, k=8, timeout=300):
    """The reference's own CUDA build (oracle/_ref, compiled from its sources) timed on this GPU through
    its stock operators: the 64 x 64 lid cavity and the plain sample's simulations one at a time
    (oracle/time_ref_cuda.py, in a subprocess).  None when the build is absent."""
    ref = os.path.join(ROOT, "oracle", "_ref")
    if not (os.path.isdir(ref) and any(f.startswith("PISOtorch") and f.endswith(".so") for f in os.listdir(ref))):
        return None
    cmd = [sys.executable, os.path.join(ROOT, "oracle", "time_ref_cuda.py")]
    if wl.get("sides") is not None:
        sel = sample_indices(wl["sides"], k)
        cmd += ["--sides", ",".join(str(int(wl["sides"][i])) for i in sel),
                "--re", ",".join(repr(float(wl["re"][i])) for i in sel),
                "--dts", ",".join(repr(float(wl["dts"][i])) for i in sel)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode != 0 or not line:
            return {"error": "rc %d: %s" % (r.returncode, (r.stderr or r.stdout)[-300:])}
        return json.loads(line[-1])
    except subprocess.TimeoutExpired:
        return {"error": "timed out after %d s" % timeout}


def grad_check(wl, steps=3):
    """Viscosity gradient of the final mean kinetic energy of the two smallest simulations (FP64,
    solves to 1e-12): adjoint against central finite differences (relative step 1e-4)."""
    import torch
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    from pict_b200.adjoint import PISOAdjoint, rollout
    order = np.argsort(wl["sides"])[:2]
    doms = [make_cavity_domain(int(wl["sides"][i]), 1.0 / wl["re"][i], torch.float64) for i in order]
    b = BatchDomain(doms, time_steps=[wl["dts"][i] for i in order])
    st = PISOStepper(b, time_step=float(wl["dts"][order[0]]), advection_tol=1e-12, pressure_tol=1e-12)
    adj = PISOAdjoint(st)
    n_s = torch.diff(b._sim_cells.long()).cuda()
    w = torch.repeat_interleave(1.0 / n_s.double(), n_s).repeat(2)
    u0 = adj.velocity().clone()
    nu0 = b._sim_visc.clone()
    nur = nu0.clone().requires_grad_(True)
    out = rollout(adj, u0.clone(), steps, [steps], nu=nur)
    (0.5 * (w * out[0] * out[0]).sum()).backward()
    errs = []
    for s in range(2):
        def loss(e):
            nu = nu0.clone()
            nu[s] *= 1 + e
            b._sim_visc.copy_(nu)
            adj.set_velocity(u0)
            for _ in range(steps):
                st.step()
            st.check()
            u = adj.velocity()
            return float(0.5 * (w * u * u).sum())
        fd = (loss(1e-4) - loss(-1e-4)) / 2e-4
        ad = float(nur.grad[s] * nu0[s])
        errs.append(abs(ad - fd) / max(abs(fd), 1e-30))
    b._sim_visc.copy_(nu0)
    return {"rel_err_vs_fd_max": max(errs), "sims": [int(wl["sides"][i]) for i in order], "steps": steps,
            "dtype": "f64"}


def _oracle_channel(nx, ny, nz):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import piso_oracle as po
    coords, vel = channel_arrays(nx, ny, nz)
    d = po.ODomain(3, 1.0 / 180.0)
    bi = d.create_block(coords=coords, velocity=vel)
    d.make_periodic(bi, "x")
    d.make_periodic(bi, "z")
    d.close_boundary(bi, "-y")
    d.close_boundary(bi, "+y")
    d.blocks[bi].source = np.array([[1.0, 0.0, 0.0]])
    d.prepare()
    return po, d


def oracle_channel_rate(nx, ny, nz, steps):
    """FP64 oracle steps of the channel at a reduced resolution (CPU, one core)."""
    po, d = _oracle_channel(nx, ny, nz)
    dt = channel_dt(nx)
    po.piso_step(d, dt, adv_tol=1e-6, p_tol=1e-6)
    t0 = time.perf_counter()
    for _ in range(steps):
        po.piso_step(d, dt, adv_tol=1e-6, p_tol=1e-6)
    t = time.perf_counter() - t0
    return nx * ny * nz * steps / t, t, nx * ny * nz * steps


def channel_accuracy_check(wl, args, n=(96, 48, 48), steps=5):
    """Per-field relative error of the channel step (same settings, half resolution: the largest the FP64
    oracle steps in seconds) against the FP64 oracle with 1e-10 solves after `steps` steps, and the largest
    FP64 refinement residual (the discrete divergence the pressure solve leaves)."""
    import torch
    from pict_b200.engine import PISOStepper
    nx, ny, nz = n
    dom = make_channel_domain(nx, ny, nz, torch.float32)
    dt = channel_dt(nx)
    st = PISOStepper(dom, time_step=dt, advection_tol=wl["tol"], pressure_tol=wl["tol"],
                     **precision_kwargs(args, wl))
    res = 0.0
    for _ in range(steps):
        st.step()
        st.check()
        res = max(res, max(max(float(i.finalResidual) for i in r) for row in st.refine_infos() for r in row))
    po, d = _oracle_channel(nx, ny, nz)
    for _ in range(steps):
        po.piso_step(d, dt, adv_tol=1e-10, p_tol=1e-10)
    u = dom.getBlock(0).velocity.double().cpu().numpy().reshape(3, -1)
    p = dom.getBlock(0).pressure.double().cpu().numpy().reshape(-1)
    ur, pr = d.velocity_global(), d.pressure_global()
    return {"steps": steps, "grid": "%dx%dx%d" % n,
            "velocity_rel_max": float(np.abs(u - ur).max() / np.abs(ur).max()),
            "pressure_rel_max": float(np.abs(p - pr).max() / np.abs(pr).max()),
            "refinement_residual_max": res if st.pressure_refine > 0 else None,
            "reference": "FP64 oracle, solver tol 1e-10"}


_ORACLE_FIELDS = {}


def accuracy_picks(sides):
    """The smallest, the largest and the simulations at the 25/50/75 % size quantiles."""
    order = np.argsort(sides)
    n = len(order)
    return [int(order[min(n - 1, int(q * (n - 1) + 0.5))]) for q in (0.0, 0.25, 0.5, 0.75, 1.0)]


def accuracy_check(wl, args, steps=10):
    """Per-field relative error of the batched FP32 step (this run's precision settings) against the FP64
    oracle with 1e-12 solves after `steps` steps, per simulation, on the smallest and the largest
    simulation and those at the 25/50/75 % size quantiles (advanced together as one batch)."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import piso_oracle as po
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    picks = accuracy_picks(wl["sides"])
    doms = [make_cavity_domain(int(wl["sides"][i]), 1.0 / wl["re"][i], torch.float32) for i in picks]
    dts = [wl["dts"][i] for i in picks]
    b = BatchDomain(doms, time_steps=dts)
    st = PISOStepper(b, time_step=dts[0], advection_tol=adv_tol(args, wl), pressure_tol=wl["tol"],
                     **precision_kwargs(args, wl))
    for _ in range(steps):
        st.step()
    st.check()
    per = []
    for k, i in enumerate(picks):
        s = int(wl["sides"][i])
        key = (s, float(wl["re"][i]), float(dts[k]), steps)
        if key not in _ORACLE_FIELDS:  # the same simulations are checked for several precisions
            d = po.ODomain(2, 1.0 / wl["re"][i])
            bi = d.create_block(coords=cavity_coords(s))
            d.close_all(bi)
            d.close_boundary(bi, "-y", np.array([[1.0, 0.0]]))
            d.prepare()
            for _ in range(steps):
                po.piso_step(d, dts[k], adv_tol=1e-12, p_tol=1e-12)
            _ORACLE_FIELDS[key] = (d.velocity_global(), d.pressure_global())
        u = doms[k].getBlock(0).velocity.double().cpu().numpy().reshape(2, -1)
        p = doms[k].getBlock(0).pressure.double().cpu().numpy().reshape(-1)
        ur, pr = _ORACLE_FIELDS[key]
        per.append({"side": s, "re": float(wl["re"][i]),
                    "velocity_rel_max": float(np.abs(u - ur).max() / np.abs(ur).max()),
                    "pressure_rel_max": float(np.abs(p - pr).max() / np.abs(pr).max())})
    return {"steps": steps, "per_simulation": per, "sims": [q["side"] for q in per],
            "velocity_rel_max": max(q["velocity_rel_max"] for q in per),
            "pressure_rel_max": max(q["pressure_rel_max"] for q in per),
            "reference": "FP64 oracle, solver tol 1e-12; simulations at the size quantiles 0/25/50/75/100 %"}


def grad_check_mixed(wl, args, steps=3, eps=1e-4):
    """Viscosity gradient of the final mean kinetic energy through the timed precision (FP32 fields, FP64
    reductions and pressure refinement) against central finite differences of the FP64 step (solves to
    1e-12), on the two smallest simulations: the error of the FP32 adjoint itself."""
    import torch
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    from pict_b200.adjoint import PISOAdjoint, rollout
    order = np.argsort(wl["sides"])[:2]

    def batch(dtype):
        doms = [make_cavity_domain(int(wl["sides"][i]), 1.0 / wl["re"][i], dtype) for i in order]
        return BatchDomain(doms, time_steps=[wl["dts"][i] for i in order])
    b32 = batch(torch.float32)
    st32 = PISOStepper(b32, time_step=float(wl["dts"][order[0]]), advection_tol=wl["tol"], pressure_tol=wl["tol"],
                       **precision_kwargs(args, wl))
    # transposed solves relative to their right-hand side (the loss gradient is ~1e-3 per cell), the
    # pressure ones to the tolerance the timed forward+backward uses
    adj = PISOAdjoint(st32, relative_tolerance=True, adjoint_pressure_tol=adjoint_pressure_tol(b32, st32))
    n_s = torch.diff(b32._sim_cells.long()).cuda()
    w32 = torch.repeat_interleave(1.0 / n_s.float(), n_s).repeat(2)
    nu32 = b32._sim_visc.clone().requires_grad_(True)
    out = rollout(adj, adj.velocity().clone(), steps, [steps], nu=nu32)
    (0.5 * (w32 * out[0] * out[0]).sum()).backward()
    b64 = batch(torch.float64)
    st64 = PISOStepper(b64, time_step=float(wl["dts"][order[0]]), advection_tol=1e-12, pressure_tol=1e-12)
    adj64 = PISOAdjoint(st64)
    u0 = adj64.velocity().clone()
    nu0 = b64._sim_visc.clone()
    w = torch.repeat_interleave(1.0 / n_s.double(), n_s).repeat(2)
    errs = []
    for s in range(2):
        def loss(e):
            nu = nu0.clone()
            nu[s] *= 1 + e
            b64._sim_visc.copy_(nu)
            adj64.set_velocity(u0)
            for _ in range(steps):
                st64.step()
            st64.check()
            u = adj64.velocity()
            return float(0.5 * (w * u * u).sum())
        fd = (loss(eps) - loss(-eps)) / (2 * eps)
        ad = float(nu32.grad[s].double() * nu0[s])
        errs.append(abs(ad - fd) / max(abs(fd), 1e-30))
    return {"rel_err_vs_fd_max": max(errs), "sims": [int(wl["sides"][i]) for i in order], "steps": steps,
            "dtype": "f32 adjoint (timed precision) vs FP64 central differences (relative step %g)" % eps}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pict", choices=["pict", "reference"])
    ap.add_argument("--extras", action="store_true",
                    help="only time the operators around the step (scalar, SGS, multi-block convolution); own JSON line")
    ap.add_argument("--warm-advection", type=int, default=2,
                    help="mixed precision: start each advection solve from the current velocity (1), from it plus "
                         "the previous step's advection increment (2), or from zero (0)")
    ap.add_argument("--workload", default="batched_cavities_256",
                    choices=["batched_cavities_256", "lid_cavity_64", "channel3d_192", "cylinder_street"])
    ap.add_argument("--group-size", type=int, default=0)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-err", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32"])
    ap.add_argument("--refine-solver", default="auto", choices=["auto", "mg", "cg"],
                    help="solver of the refinement corrections (mixed precision)")
    ap.add_argument("--first-solve", type=int, default=0,
                    help="mixed precision: 1 = FP32 CG pressure solve before the refinement, 0 = refine from the "
                         "warm-start pressure")
    ap.add_argument("--mg-iterations", type=int, default=0,
                    help="cap of the multigrid PCG iterations per correction (each system stops once its RMS residual "
                         "meets the refinement target); 0: 8 where the finest level smooths with two sweeps, else 12")
    ap.add_argument("--mg-graph-loop", type=int, default=1,
                    help="1: the multigrid PCG loop as a conditional node of the captured step (stops at convergence); "
                         "0: the fixed launch sequence (what a profiler that cannot profile kernel nodes of graphs "
                         "with conditional nodes needs)")
    ap.add_argument("--warm-pressure", type=int, default=2,
                    help="mixed precision: refinement of corrector k >= 1 starts from corrector k-1's pressure (1) "
                         "or from it plus the previous step's corrector increment (2)")
    ap.add_argument("--adv-tol", type=float, default=0.0,
                    help="RMS residual target of the advection solves (0: the workload's)")
    ap.add_argument("--refine-tol", type=float, default=0.0,
                    help="RMS residual target of the FP64 pressure refinement (0: the workload's)")
    ap.add_argument("--skip-bwd", action="store_true")
    ap.add_argument("--skip-fp32", action="store_true")
    ap.add_argument("--autotune", type=int, default=1, help="1: pick tile size / CTA cap / CG variant by timing")
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-ref-cuda", action="store_true", help="skip timing the reference's own CUDA build")
    ap.add_argument("--skip-extras", action="store_true", help="skip the brief timings of the other configurations")
    ap.add_argument("--graph-steps", type=int, default=10,
                    help="steps per captured CUDA graph (1 if --steps is not a multiple)")
    ap.add_argument("--shedding-steps", type=int, default=0,
                    help="cylinder_street: further steps after the timed ones, lift recorded every 10 steps, for "
                         "the Strouhal number")
    ap.add_argument("--fb-steps", type=int, default=10, help="steps of the forward+backward rollout")
    ap.add_argument("--checkpoint", type=int, default=5, help="checkpoint interval of the rollout")
    args = ap.parse_args()
    if args.extras:
        extras_pass()
        return
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if not args.mg_graph_loop:
        from pict_b200 import _lib
        _lib.load().pict_mg_set_graph_loop(0)
    try:
        if args.workload == "cylinder_street":
            run_street(args, rank, world)
        else:
            run_pict(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
