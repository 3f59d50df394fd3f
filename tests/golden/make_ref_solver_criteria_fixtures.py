"""CG convergence criteria and rank-deficient CG fixtures from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``) and records,
for the pressure matrix of each setup of ``CRITERIA_CASES`` (FP64, time step 0.05), ``SolveLinear`` with CG
(extensions/cg_solver_kernel.cu:114-456) for the ``ConvergenceCriterion`` values NORM2, NORM2_NORMALIZED,
ABS_SUM and ABS_MEAN (:77-110), without and with ``matrixRankDeficient`` (:240-298), from x = 0: the solution
and the result info.  ABS_MAX is left out: the reference reads the residual at the 1-based index that
``cublasITamax`` returns as if it were 0-based (:99-104), i.e. the entry after the largest one, and past the
end of the vector when the largest entry is the last (there the copy fails with "invalid argument" and the
process ends), so it has no usable result to record.  The fixture also holds the
matrix in CSR form and the right-hand sides, so that the oracle's CG runs on exactly the same system;
``criteria_fixture`` takes the module as an argument, so ``tests/test_gpu_solver_criteria.py`` runs it with
this library's module.

Usage (GPU machine):  python tests/golden/make_ref_solver_criteria_fixtures.py --out <dir>
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

CRITERIA_CASES = ["cavity2d_refined", "periodic2d", "twoblock2d_rotated", "channel3d"]
CRITERIA = [("NORM2", 1e-8), ("NORM2_NORMALIZED", 1e-9), ("ABS_SUM", 1e-7), ("ABS_MEAN", 1e-10)]
MAXIT = 300
# The rank-deficient operator makes CG nonlinear; where it does not converge its iterates depend on rounding
# (a relative change of 1e-15 in b changes the 300th iterate at order one), so those solves are also recorded
# after EARLY_MAXIT iterations, where they are still reproducible.
EARLY_MAXIT = 40
# BiCGStab (unpreconditioned) on the advection matrix with D seeded right-hand sides
BICG_CRITERIA = [("NORM2_NORMALIZED", 1e-10), ("ABS_SUM", 1e-8), ("ABS_MEAN", 1e-11)]


def rhs_vectors(n, seed):
    g = np.random.default_rng(seed)
    b = g.standard_normal(n)
    return b - b.mean(), b + 0.5  # a compatible right-hand side, and one with a mean


def criteria_fixture(R, name, csr=True):
    """Solutions and infos of every (criterion, rank-deficient) combination; with ``csr`` also the matrix
    (reference module only: its ``P`` is a CSR matrix)."""
    from setups import build_product, case
    dom = build_product(case(name), torch.float64, module=R)
    ts = torch.tensor([0.05], dtype=torch.float64)
    R.SetupAdvectionMatrix(dom, ts, 0)
    R.SetupPressureMatrix(dom, ts, 0, False)
    torch.cuda.synchronize()
    n = dom.P.getRows()
    b0, b1 = rhs_vectors(n, 7 + CRITERIA_CASES.index(name))
    out = {"b0": b0, "b1": b1}
    if csr:
        out["value"] = dom.P.value.cpu().numpy()
        out["index"] = dom.P.index.cpu().numpy()
        out["row"] = dom.P.row.cpu().numpy()
    for conv, tol in CRITERIA:
        for rd, maxit, suffix in ((False, MAXIT, ""), (True, MAXIT, ""), (True, EARLY_MAXIT, "_early")):
            b = b1 if rd else b0
            x = torch.zeros(n, dtype=torch.float64, device="cuda")
            infos = R.SolveLinear(dom.P, torch.tensor(b, device="cuda"), x, torch.IntTensor([maxit]),
                                  torch.tensor([tol], dtype=torch.float64), getattr(R.ConvergenceCriterion, conv),
                                  False, rd, 0, False, False, False)
            torch.cuda.synchronize()
            key = "%s_rd%d%s" % (conv, int(rd), suffix)
            out["x_" + key] = x.cpu().numpy()
            i = infos[0]
            out["info_" + key] = np.array([i.finalResidual, i.usedIterations, float(i.converged), float(i.isFiniteResidual)])
    D = dom.getSpatialDims()
    rb = np.random.default_rng(70 + CRITERIA_CASES.index(name)).standard_normal(D * n)
    out["b_bicg"] = rb
    if csr:
        out["value_C"] = dom.C.value.cpu().numpy()
        out["index_C"] = dom.C.index.cpu().numpy()
        out["row_C"] = dom.C.row.cpu().numpy()
    for conv, tol in BICG_CRITERIA:
        x = torch.zeros(D * n, dtype=torch.float64, device="cuda")
        infos = R.SolveLinear(dom.C, torch.tensor(rb, device="cuda"), x, torch.IntTensor([MAXIT]),
                              torch.tensor([tol], dtype=torch.float64), getattr(R.ConvergenceCriterion, conv),
                              True, False, 0, False, False, False, BiCGwithPreconditioner=False)
        torch.cuda.synchronize()
        out["x_bicg_" + conv] = x.cpu().numpy()
        out["info_bicg_" + conv] = np.array([[i.finalResidual, i.usedIterations, float(i.converged),
                                              float(i.isFiniteResidual)] for i in infos])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    for name in CRITERIA_CASES:
        np.savez_compressed(os.path.join(args.out, "ref_criteria_%s.npz" % name), **criteria_fixture(R, name))
        print("criteria fixture", name, flush=True)


if __name__ == "__main__":
    main()
