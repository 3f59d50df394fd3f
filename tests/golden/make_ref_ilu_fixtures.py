"""ILU(0)-preconditioned BiCGStab fixtures from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``) and
records ``SolveLinear`` with ``useBiCG=True, BiCGwithPreconditioner=True`` (bicgstabSolveGPU,
extensions/bicgstab_solver_kernel.cu:47-395: csrilu02 factors of the matrix, two triangular solves per
preconditioner application) on the advection matrix of each setup of ``ILU_CASES`` with D seeded
right-hand sides, from x = 0, FP64 and FP32, plain and transposed (the adjoint's solve), and the
unpreconditioned solve of the same systems: solutions and result infos.
tests/test_gpu_ilu.py and tests/test_oracle_ilu.py compare this library's preconditioned BiCGStab and the
oracle's with them.

Usage (GPU machine):  python tests/golden/make_ref_ilu_fixtures.py --out <dir>
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

ILU_CASES = ["cavity2d_refined", "periodic2d", "twoblock2d_rotated", "channel3d", "distorted2d"]
MAXIT = 300


def _solve(R, A, b, tol, transpose, precond, maxit=MAXIT, conv="NORM2_NORMALIZED"):
    x = torch.zeros_like(b)
    infos = R.SolveLinear(A, b, x, torch.IntTensor([maxit]), torch.tensor([tol], dtype=b.dtype),
                          getattr(R.ConvergenceCriterion, conv), True, False, 0, transpose, False, False,
                          BiCGwithPreconditioner=precond)
    torch.cuda.synchronize()
    return x.double().cpu().numpy(), np.array([[i.finalResidual, i.usedIterations, float(i.converged),
                                                 float(i.isFiniteResidual)] for i in infos])


def ilu_fixture(R, name):
    from setups import build_product, case
    out = {}
    for dtype, tol, tag in ((torch.float64, 1e-10, "f64"), (torch.float32, 1e-6, "f32")):
        dom = build_product(case(name), dtype, module=R)
        ts = torch.tensor([0.05], dtype=dtype)
        R.SetupAdvectionMatrix(dom, ts, 0)
        torch.cuda.synchronize()
        D = dom.getSpatialDims()
        n = dom.C.getRows()
        rb = np.random.default_rng(90 + ILU_CASES.index(name)).standard_normal(D * n)
        b = torch.tensor(rb, dtype=dtype, device="cuda")
        out["b"] = rb
        for transpose in (False, True):
            for precond in (True, False):
                x, inf = _solve(R, dom.C, b, tol, transpose, precond)
                key = "%s_t%d_p%d" % (tag, int(transpose), int(precond))
                out["x_" + key], out["info_" + key] = x, inf
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    for name in ILU_CASES:
        fx = ilu_fixture(R, name)
        np.savez_compressed(os.path.join(args.out, "ref_ilu_%s.npz" % name), **fx)
        print("ilu fixture", name, {k: v[:, 1].astype(int).tolist() for k, v in fx.items() if k.startswith("info_")},
              flush=True)


if __name__ == "__main__":
    main()
