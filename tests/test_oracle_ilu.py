"""The ILU(0) oracle and the host-side level analysis (CPU).

* ilu0() is exact LU where the pattern admits no fill (tridiagonal), and in general reproduces A on its
  sparsity pattern ((L U)_ij = A_ij for every stored (i, j)), the defining property of ILU(0);
* the preconditioned BiCGStab oracle with the operator the reference's build applies (M = tril(A)^2)
  reproduces that build's preconditioned solves (tests/golden/ref_ilu_*.npz, made by
  tests/golden/make_ref_ilu_fixtures.py): iterations, final residuals, solutions; with ILU(0) it reaches
  the same solutions in fewer iterations;
* pict_ilu_analyze (host code of the C-ABI library, no device call) returns the diagonal and transposed
  positions and level orders that make every dependency of a row sit in an earlier level.
"""
import ctypes
import os

import numpy as np
import pytest
import scipy.sparse as sp

import piso_oracle as po
from setups import build_oracle, case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ILU_CASES = ["cavity2d_refined", "periodic2d", "twoblock2d_rotated", "channel3d", "distorted2d"]
DT = 0.05


def _advection_csr(name):
    od = build_oracle(case(name))
    coef, _ = po.advection_matrix(od, DT)
    return od, po.stencil_to_csr(od, coef)


def test_ilu0_is_exact_lu_without_fill():
    rng = np.random.default_rng(5)
    n = 40
    main = 4.0 + rng.random(n)
    off_l, off_u = rng.random(n - 1) - 0.5, rng.random(n - 1) - 0.5
    A = sp.diags([off_l, main, off_u], [-1, 0, 1], format="csr")
    A.sort_indices()
    f = po.ilu0(A.data, A.indices, A.indptr)
    F = sp.csr_matrix((f, A.indices, A.indptr), shape=A.shape).toarray()
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    assert np.abs(L @ U - A.toarray()).max() < 1e-14


@pytest.mark.parametrize("name", ILU_CASES)
def test_ilu0_reproduces_matrix_on_pattern(name):
    _, (val, idx, row) = _advection_csr(name)
    n = row.size - 1
    f = po.ilu0(val, idx, row)
    F = sp.csr_matrix((f, idx, row), shape=(n, n))
    L = sp.tril(F, -1) + sp.eye(n)
    U = sp.triu(F, 0)
    LU = (L @ U).tocsr()
    A = sp.csr_matrix((val, idx, row), shape=(n, n))
    on_pattern = np.asarray(LU[A.nonzero()]).ravel() - np.asarray(A[A.nonzero()]).ravel()
    assert np.abs(on_pattern).max() < 1e-13 * np.abs(val).max()
    # with fill-in dropped, L U differs from A off the pattern
    assert (LU - A).count_nonzero() > 0 or n < 8


def _ref_fixture(name):
    p = os.path.join(GOLDEN, "ref_ilu_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    return np.load(p)


@pytest.mark.parametrize("name", ILU_CASES)
def test_oracle_preconditioned_bicgstab_reproduces_reference(name):
    """The operator the reference's build applies (M = tril(A)^2) gives its solves: the same iteration
    counts, final residuals and solutions (FP64, plain and transposed)."""
    fx = _ref_fixture(name)
    od, (val, idx, row) = _advection_csr(name)
    n = row.size - 1
    D = od.dims
    b = fx["b"].reshape(D, n)
    for transpose in (False, True):
        ref = fx["x_f64_t%d_p1" % int(transpose)].reshape(D, n)
        info = fx["info_f64_t%d_p1" % int(transpose)]
        for c in range(D):
            x, io = po.bicgstab_ilu(val, idx, row, b[c], tol=1e-10, maxit=300, transpose=transpose,
                                    preconditioner="as_reference")
            assert io.converged and io.usedIterations == int(info[c, 1])
            assert abs(io.finalResidual - info[c, 0]) <= 1e-8 * info[c, 0]
            assert np.abs(x - ref[c]).max() <= 1e-12 * np.abs(ref[c]).max()


@pytest.mark.parametrize("name", ILU_CASES)
def test_oracle_ilu0_bicgstab_matches_reference_solution(name):
    fx = _ref_fixture(name)
    od, (val, idx, row) = _advection_csr(name)
    n = row.size - 1
    D = od.dims
    b = fx["b"].reshape(D, n)
    for transpose in (False, True):
        ref = fx["x_f64_t%d_p1" % int(transpose)].reshape(D, n)
        ref_unpre = fx["info_f64_t%d_p0" % int(transpose)]
        for c in range(D):
            x, info = po.bicgstab_ilu(val, idx, row, b[c], tol=1e-10, maxit=300, transpose=transpose,
                                      preconditioner="ilu0")
            assert info.converged
            # ILU(0) takes at most as many iterations as the unpreconditioned solve
            assert info.usedIterations <= int(ref_unpre[c, 1])
            assert np.abs(x - ref[c]).max() <= 1e-8 * np.abs(ref[c]).max()


def _analyze(row, idx):
    from pict_b200 import _lib
    lib = _lib.load()
    n, nnz = row.size - 1, idx.size
    rh, ih = row.astype(np.int32), idx.astype(np.int32)
    diag, tpos = np.empty(n, np.int32), np.empty(nnz, np.int32)
    of, ob = np.empty(n, np.int32), np.empty(n, np.int32)
    pf, pb = np.empty(n + 1, np.int32), np.empty(n + 1, np.int32)
    nlf, nlb = ctypes.c_int32(0), ctypes.c_int32(0)
    rc = lib.pict_ilu_analyze(n, rh.ctypes.data, ih.ctypes.data, diag.ctypes.data, tpos.ctypes.data, of.ctypes.data,
                              pf.ctypes.data, ob.ctypes.data, pb.ctypes.data, ctypes.byref(nlf), ctypes.byref(nlb))
    return rc, diag, tpos, of, pf[:nlf.value + 1], ob, pb[:nlb.value + 1]


@pytest.mark.parametrize("name", ILU_CASES)
def test_ilu_analyze_levels(name):
    _, (val, idx, row) = _advection_csr(name)
    rc, diag, tpos, of, pf, ob, pb = _analyze(row, idx)
    assert rc == 0
    n = row.size - 1
    rows_of = np.repeat(np.arange(n), np.diff(row))
    assert np.array_equal(idx[diag], np.arange(n))
    assert np.array_equal(idx[tpos], rows_of) and np.array_equal(rows_of[tpos], idx)
    for order, ptr, lower in ((of, pf, True), (ob, pb, False)):
        assert sorted(order.tolist()) == list(range(n))
        assert ptr[0] == 0 and ptr[-1] == n
        level = np.empty(n, np.int64)
        for l in range(ptr.size - 1):
            level[order[ptr[l]:ptr[l + 1]]] = l
        dep = (idx < rows_of) if lower else (idx > rows_of)
        assert np.all(level[idx[dep]] < level[rows_of[dep]])


def test_ilu_analyze_rejects_unsymmetric_pattern():
    A = sp.csr_matrix(np.array([[2.0, 1.0, 0.0], [0.0, 2.0, 0.0], [0.0, 1.0, 2.0]]))
    A.sort_indices()
    rc = _analyze(A.indptr, A.indices)[0]
    assert rc != 0
