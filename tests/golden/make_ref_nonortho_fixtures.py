"""Golden fixtures of the non-orthogonal terms (nonOrthoFlags) from the reference's own CUDA build.

Run on a GPU machine after ``oracle/build_ref.py`` has compiled the reference extension into
``oracle/_ref``.  For every setup of ``tests/setups.py:NONORTHO_CASES`` (skewed and distorted grids,
2D/3D, periodic, inflow, two connected blocks with and without an axis permutation) this records,
through the reference's own ``PISOtorch`` API:

* operators for each flag set of ``NONORTHO_FLAG_SETS``: the advection matrix C and A
  (SetupAdvectionMatrix), the velocity RHS of a given velocity result (SetupAdvectionVelocity), the
  pressure matrix P (SetupPressureMatrix) and h, div h plus the explicit terms of a given pressure
  result (SetupPressureRHS);
* 4 FP64 steps of the non-orthogonal branch of Simulation._PISO_split_step
  (PISOtorch_simulation.py:1194-1296) from rest, with every solver report (the non-orthogonal pressure
  system is slightly inconsistent, so CG only converges above a floor: the tests use the steps whose
  solves converged).

Usage:  python tests/golden/make_ref_nonortho_fixtures.py --out <dir>
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))

import torch  # noqa: E402

DT = 0.05
STEP_DT = 0.02
ADV_TOL = 1e-12
P_TOL = 1e-5


def _np(t):
    return t.detach().double().cpu().numpy()


def solve(R, A, rhs, use_bicg, tol, reset=0, maxit=5000):
    """_linear_solve_wrapper (PISOtorch_diff.py:245-293) without fallbacks."""
    x = torch.zeros_like(rhs)
    if rhs.eq(0).all():
        return x, []
    tol_t = torch.tensor([tol], dtype=rhs.dtype)
    infos = R.SolveLinear(A, rhs, x, torch.IntTensor([maxit]), tol_t, R.ConvergenceCriterion.NORM2_NORMALIZED,
                          use_bicg, False, reset, False, False, False, BiCGwithPreconditioner=False)
    return x, [(i.finalResidual, i.usedIterations, i.converged, i.isFiniteResidual) for i in infos]


def piso_step_nonortho(R, dom, dt, flags, correctors=2):
    """Non-orthogonal branch of Simulation._PISO_split_step (PISOtorch_simulation.py:1180-1296) with one
    non-orthogonal advection and pressure step, FD velocity corrector."""
    ts = torch.tensor([dt], dtype=dom.getDtype())
    infos = []
    dom.UpdateDomainData()
    R.SetupAdvectionMatrix(dom, ts, flags)
    R.CopyVelocityResultFromBlocks(dom)
    R.SetupAdvectionVelocity(dom, ts, flags, False)
    x, inf = solve(R, dom.C, dom.velocityRHS, True, ADV_TOL)
    infos += [("adv",) + i for i in inf]
    dom.setVelocityResult(x)
    dom.UpdateDomainData()
    for _ in range(correctors):
        R.SetupPressureMatrix(dom, ts, flags, False)
        R.SetupPressureRHS(dom, ts, flags, False, timeStepNorm=False)
        p, inf = solve(R, dom.P, dom.pressureRHSdiv, False, P_TOL, reset=100)
        infos += [("p",) + i for i in inf]
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


def rest_spec(name):
    """The setup started from rest (a uniform source drives the flows without a lid or inflow)."""
    from setups import case
    spec = case(name)
    for b in spec["blocks"]:
        b["velocity"] = np.zeros_like(b["velocity"])
    if name == "skewed_periodic2d":
        spec["blocks"][0]["source"] = np.array([[0.5, 0.1]])
    return spec


def fixtures(R, name):
    from setups import NONORTHO_FLAG_SETS, build_product, case
    spec = case(name)
    D = spec["dims"]
    out = {}
    for flags in NONORTHO_FLAG_SETS:
        dom = build_product(spec, torch.float64, module=R)
        N = dom.getTotalSize()
        ts = torch.tensor([DT], dtype=torch.float64)
        rng = np.random.default_rng(7)
        ures = rng.standard_normal((D, N)) * 0.3
        R.SetupAdvectionMatrix(dom, ts, flags)
        dom.setVelocityResult(torch.tensor(ures.reshape(-1), dtype=torch.float64, device="cuda"))
        dom.UpdateDomainData()
        R.SetupAdvectionVelocity(dom, ts, flags, False)
        torch.cuda.synchronize()
        k = "f%d_" % flags
        out[k + "ures"] = ures
        out[k + "C_value"], out[k + "C_index"], out[k + "C_row"] = (_np(dom.C.value), dom.C.index.cpu().numpy(),
                                                                   dom.C.row.cpu().numpy())
        out[k + "A"] = _np(dom.A)
        out[k + "velocityRHS"] = _np(dom.velocityRHS)
        ustar = rng.standard_normal((D, N)) * 0.3
        pres = rng.standard_normal(N)
        dom.setVelocityResult(torch.tensor(ustar.reshape(-1), dtype=torch.float64, device="cuda"))
        dom.setPressureResult(torch.tensor(pres, dtype=torch.float64, device="cuda"))
        dom.UpdateDomainData()
        R.SetupPressureMatrix(dom, ts, flags, False)
        R.SetupPressureRHS(dom, ts, flags, False, timeStepNorm=False)
        torch.cuda.synchronize()
        out[k + "ustar"], out[k + "pres"] = ustar, pres
        out[k + "P_value"], out[k + "P_index"], out[k + "P_row"] = (_np(dom.P.value), dom.P.index.cpu().numpy(),
                                                                   dom.P.row.cpu().numpy())
        out[k + "pressureRHS"] = _np(dom.pressureRHS)
        out[k + "pressureRHSdiv"] = _np(dom.pressureRHSdiv)
    dom2 = build_product(rest_spec(name), torch.float64, module=R)
    infos = []
    for _ in range(4):
        infos += piso_step_nonortho(R, dom2, STEP_DT, 25)
    u, p = block_fields(dom2)
    out["steps_flags"], out["steps_dt"], out["steps_n"], out["steps_p_tol"] = 25, STEP_DT, 4, P_TOL
    out["steps_velocity"], out["steps_pressure"] = u, p
    out["steps_infos"] = np.array([i[1:] for i in infos], dtype=np.float64) if infos else np.zeros((0, 4))
    out["steps_info_kind"] = np.array([0 if i[0] == "adv" else 1 for i in infos], dtype=np.int32)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    from setups import NONORTHO_CASES
    for name in NONORTHO_CASES:
        fx = fixtures(R, name)
        np.savez_compressed(os.path.join(args.out, "ref_nonortho_%s.npz" % name), **fx)
        conv = fx["steps_infos"][:, 2].all() if len(fx["steps_infos"]) else True
        print("fixture", name, "steps converged:", bool(conv), flush=True)


if __name__ == "__main__":
    main()
