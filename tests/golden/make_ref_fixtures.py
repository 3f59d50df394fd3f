"""Generate golden fixtures from the reference's own CUDA build (run on a GPU machine).

The reference extension is compiled from its sources by ``oracle/build_ref.py`` into
``oracle/_ref/PISOtorch*.so``; this script imports that module, builds every setup of
``tests/setups.py`` through the reference's own ``PISOtorch`` API, runs its operators and its
Krylov solvers (``SolveLinear``) in the order of the reference driver's orthogonal PISO branch
(PISOtorch_simulation.py:1170-1312; solve wrapper PISOtorch_diff.py:245-293), and writes the
results as ``.npz`` fixtures.  ``tests/test_oracle_golden.py`` pins the FP64 oracle and the CUDA
path against them.  It also times the reference's CUDA step for the baseline table.

Usage (GPU machine):  python tests/golden/make_ref_fixtures.py --out <dir>
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))

import torch  # noqa: E402

DT = 0.05


def ref_module():
    import PISOtorch as R
    return R


def _np(t):
    return t.detach().double().cpu().numpy()


def solve(R, A, rhs, use_bicg, tol, maxit=5000):
    """_linear_solve_wrapper (PISOtorch_diff.py:245-293) without fallbacks."""
    x = torch.zeros_like(rhs)
    if rhs.eq(0).all():
        return x, []
    tol_t = torch.tensor([tol], dtype=rhs.dtype)
    infos = R.SolveLinear(A, rhs, x, torch.IntTensor([maxit]), tol_t, R.ConvergenceCriterion.NORM2_NORMALIZED,
                          use_bicg, False, 0, False, False, False, BiCGwithPreconditioner=False)
    return x, [(i.finalResidual, i.usedIterations, i.converged, i.isFiniteResidual) for i in infos]


def piso_step(R, dom, dt, tol, correctors=2):
    """Orthogonal branch of Simulation._PISO_split_step (PISOtorch_simulation.py:1170-1312)."""
    ts = torch.tensor([dt], dtype=dom.getDtype())
    infos = []
    dom.UpdateDomainData()
    R.SetupAdvectionMatrix(dom, ts, 0)
    R.SetupAdvectionVelocity(dom, ts, 0, False)
    x, inf = solve(R, dom.C, dom.velocityRHS, True, tol)
    infos += inf
    dom.setVelocityResult(x)
    dom.UpdateDomainData()
    for _ in range(correctors):
        R.SetupPressureCorrection(dom, ts, 0, False, timeStepNorm=False)
        p, inf = solve(R, dom.P, dom.pressureRHSdiv, False, tol)
        infos += inf
        p = p - torch.mean(p)
        dom.setPressureResult(p)
        dom.UpdateDomainData()
        R.CopyPressureResultToBlocks(dom)
        R.CorrectVelocity(dom, ts, version=1, timeStepNorm=False)
    R.CopyVelocityResultToBlocks(dom)
    return infos


def block_fields(dom):
    D = dom.getSpatialDims()
    u = np.concatenate([_np(b.velocity).reshape(D, -1) for b in dom.getBlocks()], axis=1)
    p = np.concatenate([_np(b.pressure).reshape(-1) for b in dom.getBlocks()])
    return u, p


def op_fixtures(R, name):
    from setups import build_product, case
    spec = case(name)
    out = {}
    dom = build_product(spec, torch.float64, module=R)
    ts = torch.tensor([DT], dtype=torch.float64)
    R.SetupAdvectionMatrix(dom, ts, 0)
    R.SetupAdvectionVelocity(dom, ts, 0, False)
    torch.cuda.synchronize()
    out["C_value"], out["C_index"], out["C_row"] = _np(dom.C.value), dom.C.index.cpu().numpy(), dom.C.row.cpu().numpy()
    out["A"] = _np(dom.A)
    out["velocityRHS"] = _np(dom.velocityRHS)
    N = dom.getTotalSize()
    D = spec["dims"]
    rng = np.random.default_rng(7)
    ustar = rng.standard_normal((D, N)) * 0.3
    dom.setVelocityResult(torch.tensor(ustar.reshape(-1), dtype=torch.float64, device="cuda"))
    dom.UpdateDomainData()
    R.SetupPressureCorrection(dom, ts, 0, False, timeStepNorm=False)
    torch.cuda.synchronize()
    out["ustar"] = ustar
    out["P_value"], out["P_index"], out["P_row"] = _np(dom.P.value), dom.P.index.cpu().numpy(), dom.P.row.cpu().numpy()
    out["pressureRHS"] = _np(dom.pressureRHS)
    out["pressureRHSdiv"] = _np(dom.pressureRHSdiv)
    rng = np.random.default_rng(11)
    p = rng.standard_normal(N)
    h = rng.standard_normal((D, N))
    dom.setPressureResult(torch.tensor(p, dtype=torch.float64, device="cuda"))
    dom.setPressureRHS(torch.tensor(h.reshape(-1), dtype=torch.float64, device="cuda"))
    dom.UpdateDomainData()
    R.CopyPressureResultToBlocks(dom)
    R.CorrectVelocity(dom, ts, version=1, timeStepNorm=False)
    torch.cuda.synchronize()
    out["corr_p"], out["corr_h"], out["corr_velocityResult"] = p, h, _np(dom.velocityResult)
    # full steps, FP64, tight tolerance
    dom2 = build_product(spec, torch.float64, module=R)
    infos = []
    for _ in range(4):
        infos += piso_step(R, dom2, 0.02, 1e-13)
    u, pp = block_fields(dom2)
    out["steps_dt"], out["steps_n"] = 0.02, 4
    out["steps_velocity"], out["steps_pressure"] = u, pp
    out["steps_infos"] = np.array(infos, dtype=np.float64) if infos else np.zeros((0, 4))
    return out


def lid_fixture(R, n, steps, dtype, tol, dt=0.01, viscosity=1e-3):
    from setups import build_product, lid_cavity
    spec = lid_cavity(n, viscosity=viscosity)
    dom = build_product(spec, dtype, module=R)
    torch.cuda.synchronize()
    infos = []
    t0 = time.perf_counter()
    for _ in range(steps):
        infos += piso_step(R, dom, dt, tol)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    u, p = block_fields(dom)
    return dict(velocity=u, pressure=p, infos=np.array(infos, dtype=np.float64), n=n, steps=steps, dt=dt,
                viscosity=viscosity, tol=tol, seconds=el)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--cases", nargs="*", default=None, help="only the operator fixtures of these setups")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    R = ref_module()
    from setups import ALL_CASES
    summary = {}
    for name in (ALL_CASES if args.cases is None else args.cases):
        fx = op_fixtures(R, name)
        np.savez_compressed(os.path.join(args.out, "ref_ops_%s.npz" % name), **fx)
        summary[name] = "ok"
        print("fixture", name, flush=True)
    if args.cases is not None:
        return
    timings = {}
    for (n, steps, dtype, tol, tag) in [(64, 100, torch.float32, 1e-6, "lid64_f32"), (64, 100, torch.float64, 1e-10, "lid64_f64")]:
        fx = lid_fixture(R, n, steps, dtype, tol)
        np.savez_compressed(os.path.join(args.out, "ref_%s.npz" % tag), **fx)
        timings[tag] = {"cells": n * n, "steps": steps, "seconds": fx["seconds"],
                        "cell_steps_per_s": n * n * steps / fx["seconds"]}
        print("fixture", tag, timings[tag], flush=True)
    if not args.quick:
        for n in (32, 128, 256):
            fx = lid_fixture(R, n, 5, torch.float32, 1e-6, dt=0.5 / n, viscosity=1e-3)
            timings["plain_cavity%d_f32" % n] = {"cells": n * n, "steps": 5, "seconds": fx["seconds"],
                                                 "cell_steps_per_s": n * n * 5 / fx["seconds"]}
            print("timing", n, timings["plain_cavity%d_f32" % n], flush=True)
    with open(os.path.join(args.out, "ref_timings.json"), "w") as f:
        json.dump(timings, f, indent=1)


if __name__ == "__main__":
    main()
