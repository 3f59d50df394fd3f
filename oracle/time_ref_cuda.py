"""Timing of the reference's own CUDA build on the B200 (baseline measurement, not the product).

Imports the reference extension that ``oracle/build_ref.py`` compiled from the reference's sources into
``oracle/_ref`` and times the plain PISO step through its stock operators in the reference driver's
orthogonal order (Simulation._PISO_split_step, PISOtorch_simulation.py:1170-1312: SetupAdvectionMatrix,
SetupAdvectionVelocity, SolveLinear BiCGStab, then per corrector SetupPressureCorrection, SolveLinear
CG, mean removal, CopyPressureResultToBlocks, CorrectVelocity; CopyVelocityResultToBlocks), solves to
an RMS residual of 1e-6, FP32, wall clock with a device synchronisation on both sides:

* ``lid64``: the 64 x 64 lid-driven cavity (Re 1000, dt 0.01), --lid-steps steps;
* ``cavities``: lid-driven cavities of the given sides / Reynolds numbers / time steps, one simulation
  at a time (the reference has no batched step), --cavity-steps steps each.

Prints one JSON object.  Run by bench.py as a subprocess when oracle/_ref holds the build.

Usage:  python oracle/time_ref_cuda.py [--sides 38,49,...] [--re ...] [--dts ...]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "_ref"))

import torch  # noqa: E402


def cavity(R, n, viscosity, dtype=torch.float32):
    xs = np.linspace(0.0, 1.0, n + 1)
    Y, X = np.meshgrid(xs, xs, indexing="ij")
    coords = torch.tensor(np.stack([X, Y])[None], dtype=dtype, device="cuda").contiguous()
    dom = R.Domain(2, torch.tensor([viscosity], dtype=dtype), name="cavity", dtype=dtype, device=torch.device("cuda"),
                   passiveScalarChannels=0)
    blk = dom.CreateBlock(vertexCoordinates=coords, name="cavity")
    blk.CloseAllBoundaries()
    blk.CloseBoundary("-y", torch.tensor([[1.0, 0.0]], dtype=dtype, device="cuda"))
    dom.PrepareSolve()
    return dom


def _solve(R, A, rhs, use_bicg, tol, maxit=5000):
    x = torch.zeros_like(rhs)
    if bool(rhs.eq(0).all()):
        return x
    R.SolveLinear(A, rhs, x, torch.IntTensor([maxit]), torch.tensor([tol], dtype=rhs.dtype),
                  R.ConvergenceCriterion.NORM2_NORMALIZED, use_bicg, False, 0, False, False, False,
                  BiCGwithPreconditioner=False)
    return x


def step(R, dom, ts, tol, correctors=2):
    dom.UpdateDomainData()
    R.SetupAdvectionMatrix(dom, ts, 0)
    R.SetupAdvectionVelocity(dom, ts, 0, False)
    dom.setVelocityResult(_solve(R, dom.C, dom.velocityRHS, True, tol))
    dom.UpdateDomainData()
    for _ in range(correctors):
        R.SetupPressureCorrection(dom, ts, 0, False, timeStepNorm=False)
        p = _solve(R, dom.P, dom.pressureRHSdiv, False, tol)
        dom.setPressureResult(p - torch.mean(p))
        dom.UpdateDomainData()
        R.CopyPressureResultToBlocks(dom)
        R.CorrectVelocity(dom, ts, version=1, timeStepNorm=False)
    R.CopyVelocityResultToBlocks(dom)


def timed(R, n, viscosity, dt, steps, tol=1e-6, warmup=1):
    dom = cavity(R, n, viscosity)
    ts = torch.tensor([dt], dtype=torch.float32)
    for _ in range(warmup):
        step(R, dom, ts, tol)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        step(R, dom, ts, tol)
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lid-steps", type=int, default=20)
    ap.add_argument("--sides", default="")
    ap.add_argument("--re", default="")
    ap.add_argument("--dts", default="")
    ap.add_argument("--cavity-steps", type=int, default=3)
    args = ap.parse_args()
    import PISOtorch as R
    out = {"build": "reference extensions built from source (oracle/build_ref.py), FP32, solves to 1e-6 RMS",
           "timing": "wall clock, device synchronised, warm-up step excluded"}
    t = timed(R, 64, 1e-3, 0.01, args.lid_steps)
    out["lid64"] = {"cells": 4096, "steps": args.lid_steps, "seconds": t, "cell_steps_per_s": 4096 * args.lid_steps / t}
    if args.sides:
        sides = [int(v) for v in args.sides.split(",")]
        re = [float(v) for v in args.re.split(",")]
        dts = [float(v) for v in args.dts.split(",")]
        tot_t, tot_c = 0.0, 0
        for s, r, dt in zip(sides, re, dts):
            tot_t += timed(R, s, 1.0 / r, dt, args.cavity_steps)
            tot_c += s * s * args.cavity_steps
        out["cavities"] = {"sides": sides, "steps_each": args.cavity_steps, "seconds": tot_t,
                           "cell_steps_per_s": tot_c / tot_t, "order": "one simulation at a time"}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
