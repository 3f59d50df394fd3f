"""Cylinder-street fixtures from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``),
builds the cylinder street (pict_b200.cylinder_street) through the reference's own ``PISOtorch`` API and
runs it the way the reference's vortex-street samples do (vortex_street_sample.py:212-258,
vortex_street_torus_sample.py:169-233): the advective outflow update before every step (the samples'
prep_fn "PRE"; the update functions are this package's restatement, pinned to the reference's own
functions by tests/test_outflow_golden.py), Simulation.make_divergence_free first
(PISOtorch_simulation.py:985-1052, whose "PRE" update runs with time step 1), then the orthogonal
PISO step (PISOtorch_simulation.py:1170-1312) with the reference's operators and SolveLinear.

Written to ``--out``:
* ``ref_street16_f64.npz``: the reduced street (16 x 16 cells per quadrant, dx 0.5, 1728 cells) in
  FP64 with 1e-12 solves: operators at the initial state, the fields after the projection and after
  20 steps, the outflow face velocity and the solver reports;
* ``ref_street_full_f32.npz`` (unless --quick): the full street (27,648 cells) in FP32, --full-steps
  steps with 1e-6 solves, the force on the cylinder every 10 steps, the final fields and the
  reference's wall-clock time per step;
* ``ref_street_full_f64.npz`` (unless --quick): the same in FP64 with 1e-10 solves, --full64-steps steps.

Usage (GPU machine):  python tests/golden/make_ref_street_fixtures.py --out <dir> [--quick] [--full-steps N]
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
sys.path.insert(0, ROOT)

import torch  # noqa: E402

from make_ref_fixtures import block_fields, piso_step, ref_module, solve  # noqa: E402
from pict_b200.cylinder_street import build_street, cylinder_forces, outflow_bounds, street_spec  # noqa: E402
from pict_b200.PISOtorch_simulation import update_advective_boundaries  # noqa: E402

DT = 0.005


def _np(t):
    return t.detach().double().cpu().numpy()


def outflow_update(dom, info, dt):
    update_advective_boundaries(dom, outflow_bounds(dom, info), info["char_vel"],
                                torch.tensor([dt], dtype=dom.getDtype()).cuda())


def make_divergence_free(R, dom, info, tol, maxit=1000):
    """Simulation.make_divergence_free with one corrector, orthogonal (PISOtorch_simulation.py:985-1052)."""
    ts = torch.tensor([1.0], dtype=dom.getDtype())
    dom.setA(torch.ones_like(dom.A))
    outflow_update(dom, info, 1.0)
    dom.UpdateDomainData()
    R.CopyVelocityResultFromBlocks(dom)
    dom.setPressureRHS(dom.velocityResult)
    dom.UpdateDomainData()
    R.SetupPressureMatrix(dom, ts, 0, False)
    R.SetupPressureRHSdiv(dom, ts, 0, False, timeStepNorm=False)
    p, inf = solve(R, dom.P, dom.pressureRHSdiv, False, tol, maxit=maxit)
    p = p - torch.mean(p)
    dom.setPressureResult(p)
    dom.UpdateDomainData()
    R.CopyPressureResultToBlocks(dom)
    R.CorrectVelocity(dom, ts, version=1, timeStepNorm=False)
    R.CopyVelocityResultToBlocks(dom)
    return inf


def outflow_velocity(dom, info):
    return np.concatenate([_np(b.velocity).reshape(2, -1) for b in outflow_bounds(dom, info)], axis=1)


def reduced_fixture(R, steps=20, tol=1e-12):
    spec = street_spec(16, 16, 0.5)
    out = {}
    dom, info = build_street(spec, module=R, dtype=torch.float64)
    ts = torch.tensor([DT], dtype=torch.float64)
    R.SetupAdvectionMatrix(dom, ts, 0)
    R.SetupAdvectionVelocity(dom, ts, 0, False)
    torch.cuda.synchronize()
    out["C_value"], out["C_index"], out["C_row"] = _np(dom.C.value), dom.C.index.cpu().numpy(), dom.C.row.cpu().numpy()
    out["A"], out["velocityRHS"] = _np(dom.A), _np(dom.velocityRHS)
    N = dom.getTotalSize()
    ustar = np.random.default_rng(7).standard_normal((2, N)) * 0.3 + np.array([[1.0], [0.0]])
    dom.setVelocityResult(torch.tensor(ustar.reshape(-1), dtype=torch.float64, device="cuda"))
    dom.UpdateDomainData()
    R.SetupPressureCorrection(dom, ts, 0, False, timeStepNorm=False)
    torch.cuda.synchronize()
    out["ustar"] = ustar
    out["P_value"], out["pressureRHS"], out["pressureRHSdiv"] = _np(dom.P.value), _np(dom.pressureRHS), _np(dom.pressureRHSdiv)
    # projection and steps on a fresh domain
    dom, info = build_street(spec, module=R, dtype=torch.float64)
    out["proj_infos"] = np.array(make_divergence_free(R, dom, info, tol), dtype=np.float64)
    out["proj_velocity"], out["proj_pressure"] = block_fields(dom)
    out["proj_outflow"] = outflow_velocity(dom, info)
    infos = []
    for _ in range(steps):
        outflow_update(dom, info, DT)
        infos += piso_step(R, dom, DT, tol)
    out["steps"], out["dt"], out["tol"] = steps, DT, tol
    out["velocity"], out["pressure"] = block_fields(dom)
    out["outflow"] = outflow_velocity(dom, info)
    out["infos"] = np.array(infos, dtype=np.float64)
    return out


def full_fixture(R, steps, tol=1e-6, every=10, dtype=torch.float32):
    spec = street_spec()
    dom, info = build_street(spec, module=R, dtype=dtype)
    # the projection's iteration cap is the driver's 1000 (PISOtorch_simulation.py:985); tight FP64 solves
    # of the full street need more
    make_divergence_free(R, dom, info, tol, maxit=1000 if dtype == torch.float32 else 5000)
    forces, infos = [], []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(steps):
        outflow_update(dom, info, DT)
        infos += piso_step(R, dom, DT, tol)
        if (s + 1) % every == 0:
            forces.append(cylinder_forces(dom, info))
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    u, p = block_fields(dom)
    it = np.array(infos, dtype=np.float64)
    return dict(forces=np.array(forces), every=every, steps=steps, dt=DT, tol=tol, velocity=u, pressure=p,
                outflow=outflow_velocity(dom, info), seconds=el, cells=dom.getTotalSize(),
                iterations=it[:, 1] if len(it) else np.zeros(0), converged=it[:, 2] if len(it) else np.zeros(0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    ap.add_argument("--quick", action="store_true", help="only the reduced FP64 fixture")
    ap.add_argument("--full-steps", type=int, default=2000)
    ap.add_argument("--full64-steps", type=int, default=400)
    ap.add_argument("--only", default="", help="comma list of fixtures to write: street16,full,full64")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    R = ref_module()
    only = set(args.only.split(",")) if args.only else {"street16", "full", "full64"}
    if "street16" in only:
        fx = reduced_fixture(R)
        np.savez_compressed(os.path.join(args.out, "ref_street16_f64.npz"), **fx)
        print("fixture street16_f64: iterations", fx["infos"][:, 1].astype(int).tolist()[:12], flush=True)
    if args.quick:
        return
    runs = []
    if "full" in only:
        runs.append(("ref_street_full_f32.npz", args.full_steps, 1e-6, torch.float32))
    if "full64" in only:
        runs.append(("ref_street_full_f64.npz", args.full64_steps, 1e-10, torch.float64))
    for name, steps, tol, dtype in runs:
        fx = full_fixture(R, steps, tol=tol, dtype=dtype)
        np.savez_compressed(os.path.join(args.out, name), **fx)
        print("fixture %s: %d steps in %.1f s (%.2f ms/step), all converged: %s, last forces %s"
              % (name, fx["steps"], fx["seconds"], 1e3 * fx["seconds"] / fx["steps"], bool(fx["converged"].all()),
                 fx["forces"][-3:].tolist()), flush=True)


if __name__ == "__main__":
    main()
