"""The oracle's CG with every convergence criterion and the rank-deficient operator against the reference's own
CUDA build on the same systems (fixtures from tests/golden/make_ref_solver_criteria_fixtures.py)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import piso_oracle as po

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["cavity2d_refined", "periodic2d", "twoblock2d_rotated", "channel3d"]
CRITERIA = [("NORM2", 1e-8), ("NORM2_NORMALIZED", 1e-9), ("ABS_SUM", 1e-7), ("ABS_MEAN", 1e-10)]
MAXIT = 300
EARLY_MAXIT = 40


def check_solve(x, info, f, key):
    """Compare a solve (x, (finalResidual, usedIterations, converged, ...)) with fixture entry ``key``.

    Converged solves: the same iteration (or one apart at the tolerance) and solutions equal to rounding.  The
    criterion is compared loosely (10 %): at convergence it is the norm of a recursively updated residual 1e-8
    to 1e-10 below the right-hand side, whose last digits follow the order of the sparse products.  Unconverged
    rank-deficient solves after the full iteration count are only checked for their status: that CG is
    nonlinear and its late iterates depend on rounding (a 1e-15 change of b changes them at order one).  The
    same solves stopped after a few iterations (keys ending in "_early") are compared strictly."""
    ref_info = f["info_" + key]
    ref_x = f["x_" + key]
    assert bool(info[2]) == bool(ref_info[2]), (key, info, ref_info)
    if bool(ref_info[2]):
        assert abs(int(info[1]) - int(ref_info[1])) <= 1, (key, info, ref_info)
        if int(info[1]) == int(ref_info[1]):
            assert abs(info[0] - ref_info[0]) <= 0.1 * abs(ref_info[0]), (key, info, ref_info)
            assert np.abs(x - ref_x).max() <= 1e-7 * np.abs(ref_x).max(), key
        else:
            assert np.abs(x - ref_x).max() <= 1e-5 * np.abs(ref_x).max(), key
    else:
        assert int(info[1]) == int(ref_info[1]), (key, info, ref_info)
        if key.endswith("_early"):
            assert abs(info[0] - ref_info[0]) <= 1e-6 * abs(ref_info[0]), (key, info, ref_info)
            assert np.abs(x - ref_x).max() <= 1e-7 * np.abs(ref_x).max(), key


BICG_CRITERIA = [("NORM2_NORMALIZED", 1e-10), ("ABS_SUM", 1e-8), ("ABS_MEAN", 1e-11)]


def check_bicg(x, infos, f, conv):
    """BiCGStab solves of the D components against the fixture: per component the same iteration (or one
    apart at the tolerance), convergence, and the solution to rounding."""
    ref = f["info_bicg_" + conv]
    ref_x = f["x_bicg_" + conv]
    n = ref_x.size // len(ref)
    for c, (inf, ri) in enumerate(zip(infos, ref)):
        assert bool(inf[2]) == bool(ri[2]) and abs(int(inf[1]) - int(ri[1])) <= 1, (conv, c, inf, ri)
        xs, rs = x[c * n:(c + 1) * n], ref_x[c * n:(c + 1) * n]
        assert np.abs(xs - rs).max() <= 1e-6 * np.abs(rs).max(), (conv, c)


@pytest.mark.parametrize("name", CASES)
def test_oracle_bicgstab_criteria_match_reference(name):
    with np.load(os.path.join(GOLDEN, "ref_criteria_%s.npz" % name)) as z:
        f = {k: z[k] for k in z.files}
    n = f["b0"].size
    C = sp.csr_matrix((f["value_C"], f["index_C"], f["row_C"]), shape=(n, n))
    D = f["b_bicg"].size // n
    for conv, tol in BICG_CRITERIA:
        xs, infos = [], []
        for c in range(D):
            x, inf = po.bicgstab(C, f["b_bicg"][c * n:(c + 1) * n], tol=tol, maxit=MAXIT, conv=conv)
            xs.append(x)
            infos.append((inf.finalResidual, inf.usedIterations, inf.converged))
        check_bicg(np.concatenate(xs), infos, f, conv)


@pytest.mark.parametrize("name", CASES)
def test_oracle_cg_criteria_match_reference(name):
    with np.load(os.path.join(GOLDEN, "ref_criteria_%s.npz" % name)) as z:
        f = {k: z[k] for k in z.files}
    n = f["b0"].size
    A = sp.csr_matrix((f["value"], f["index"], f["row"]), shape=(n, n))
    for conv, tol in CRITERIA:
        for rd, maxit, suffix in ((False, MAXIT, ""), (True, MAXIT, ""), (True, EARLY_MAXIT, "_early")):
            b = f["b1"] if rd else f["b0"]
            x, inf = po.cg(A, b, tol=tol, maxit=maxit, conv=conv, rank_deficient=rd)
            check_solve(x, (inf.finalResidual, inf.usedIterations, inf.converged), f,
                        "%s_rd%d%s" % (conv, int(rd), suffix))
