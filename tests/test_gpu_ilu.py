"""Preconditioned BiCGStab on the device (GPU), through SolveLinear(useBiCG=True,
BiCGwithPreconditioner=True) and the C-ABI factorisation:

* the default preconditioner (BiCGPreconditioner.AS_REFERENCE, the operator the reference's build applies)
  reproduces the reference build's preconditioned solves (tests/golden/ref_ilu_*.npz): the same iteration
  counts (FP64; FP32 within one), solutions to 1e-10 (FP64), plain and transposed;
* ILU0: pict_ilu0_factor against the oracle's ilu0() on the advection matrices of five setups (FP64 to
  round-off); solutions against the reference's and the oracle's ILU(0) solve, with at most the oracle's
  iterations + 1;
* the preconditioned fallback of the linear-solve wrapper (PISOtorch_diff.py:276-286) and of
  Simulation.linear_solve: an unpreconditioned BiCGStab solve that stops unconverged at max_iter is repeated
  preconditioned and converges.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import piso_oracle as po
from setups import build_product, case, lid_cavity

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ILU_CASES = ["cavity2d_refined", "periodic2d", "twoblock2d_rotated", "channel3d", "distorted2d"]
DT = 0.05


def _np(t):
    return t.detach().double().cpu().numpy()


def _load(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip("fixture %s missing" % name)
    return np.load(p)


def _advection(name, dtype):
    from pict_b200 import PISOtorch as P
    pd = build_product(case(name), dtype)
    P.SetupAdvectionMatrix(pd, torch.tensor([DT], dtype=dtype), 0)
    return pd


def _solve(pd, b, tol, transpose, precond, maxit=300):
    from pict_b200 import PISOtorch as P
    x = torch.zeros_like(b)
    infos = P.SolveLinear(pd.C, b, x, torch.IntTensor([maxit]), torch.tensor([tol], dtype=b.dtype),
                          P.ConvergenceCriterion.NORM2_NORMALIZED, True, False, 0, transpose, False, False,
                          BiCGwithPreconditioner=precond)
    torch.cuda.synchronize()
    return x, infos


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("name", ILU_CASES)
def test_ilu0_factor_matches_oracle(name, dtype):
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    pd = _advection(name, dtype)
    plan = P._ilu_plan(pd)
    val = pd.C.value.contiguous()
    f = torch.empty_like(val)
    lib = _lib.load()
    rc = lib.pict_ilu0_factor(plan["n"], plan["nnz"], P._dtype_code(dtype), P._ptr(plan["row"]), P._ptr(plan["index"]),
                              P._ptr(plan["diag"]), P._ptr(plan["order_f"]), plan["ptr_f"].ctypes.data, plan["nlf"],
                              P._ptr(val), P._ptr(f), P._stream_ptr())
    torch.cuda.synchronize()
    assert rc == 0
    ref = po.ilu0(_np(val), plan["index"].cpu().numpy(), plan["row"].cpu().numpy())
    bound = 1e-13 if dtype == torch.float64 else 2e-6
    assert np.abs(_np(f) - ref).max() <= bound * np.abs(ref).max()


@pytest.fixture
def ilu0_mode():
    from pict_b200 import PISOtorch as P
    prev = P.SetBiCGPreconditioner(P.BiCGPreconditioner.ILU0)
    yield
    P.SetBiCGPreconditioner(prev)


@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("name", ILU_CASES)
def test_preconditioned_bicgstab_reproduces_reference(name, dtype, transpose):
    from pict_b200 import PISOtorch as P
    assert P.GetBiCGPreconditioner() == P.BiCGPreconditioner.AS_REFERENCE
    fx = _load("ref_ilu_%s.npz" % name)
    pd = _advection(name, dtype)
    D = pd.getSpatialDims()
    tag = "f64" if dtype == torch.float64 else "f32"
    tol = 1e-10 if dtype == torch.float64 else 1e-6
    b = torch.tensor(fx["b"], dtype=dtype, device="cuda")
    x, infos = _solve(pd, b, tol, transpose, True)
    assert all(i.converged and i.isFiniteResidual for i in infos)
    n = pd.C.getRows()
    xs = _np(x).reshape(D, n)
    key = "%s_t%d_p1" % (tag, int(transpose))
    ref = fx["x_" + key].reshape(D, n)
    rinfo = fx["info_" + key]
    for c in range(D):
        if dtype == torch.float64:
            assert infos[c].usedIterations == int(rinfo[c, 1])
            assert np.abs(xs[c] - ref[c]).max() <= 1e-10 * np.abs(ref[c]).max()
        else:
            assert abs(infos[c].usedIterations - int(rinfo[c, 1])) <= 1
            assert np.abs(xs[c] - ref[c]).max() <= 5e-5 * np.abs(ref[c]).max()


@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("name", ILU_CASES)
def test_ilu0_bicgstab_matches_reference_and_oracle(name, dtype, transpose, ilu0_mode):
    fx = _load("ref_ilu_%s.npz" % name)
    pd = _advection(name, dtype)
    D = pd.getSpatialDims()
    tag = "f64" if dtype == torch.float64 else "f32"
    tol = 1e-10 if dtype == torch.float64 else 1e-6
    b = torch.tensor(fx["b"], dtype=dtype, device="cuda")
    x, infos = _solve(pd, b, tol, transpose, True)
    assert all(i.converged and i.isFiniteResidual for i in infos)
    n = pd.C.getRows()
    xs = _np(x).reshape(D, n)
    ref = fx["x_%s_t%d_p1" % (tag, int(transpose))].reshape(D, n)
    val = _np(pd.C.value)
    idx, row = pd.C.index.cpu().numpy(), pd.C.row.cpu().numpy()
    bref = fx["b"].reshape(D, n)
    for c in range(D):
        xo, io = po.bicgstab_ilu(val, idx, row, bref[c], tol=tol, maxit=300, transpose=transpose,
                                 preconditioner="ilu0")
        scale = np.abs(ref[c]).max()
        bound = 1e-8 if dtype == torch.float64 else 5e-5
        assert np.abs(xs[c] - ref[c]).max() <= bound * scale
        assert np.abs(xs[c] - xo).max() <= bound * scale
        assert infos[c].usedIterations <= io.usedIterations + 1


def _shifted_laplacian(n=48):
    """The pressure matrix of an n x n lid-driven cavity with its diagonal scaled by 1.001 (nonsingular,
    condition number in the thousands) and a seeded right-hand side, FP64."""
    from pict_b200 import PISOtorch as P
    pd = build_product(lid_cavity(n, viscosity=1e-3), torch.float64)
    ts = torch.tensor([0.01], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupPressureCorrection(pd, ts)
    coef = pd.P.coef.clone()
    coef[0] *= 1.001
    M = P.StencilMatrix(pd, coef)
    g = torch.Generator().manual_seed(11)
    b = torch.randn(M.getRows(), generator=g, dtype=torch.float64).cuda()
    return pd, M, b


def test_preconditioned_fallback_recovers_a_failed_solve(ilu0_mode):
    from pict_b200 import PISOtorch as P
    from pict_b200 import PISOtorch_diff as PD
    from pict_b200.engine import LinsolveError
    pd, M, b = _shifted_laplacian()
    tol = 1e-9

    def iters(pre):
        x = torch.zeros_like(b)
        infos = P.SolveLinear(M, b, x, torch.IntTensor([2000]), torch.tensor([tol], dtype=torch.float64),
                              P.ConvergenceCriterion.NORM2_NORMALIZED, True, False, 0, False, False, False,
                              BiCGwithPreconditioner=pre)
        assert infos[0].converged
        return infos[0].usedIterations, x

    it_plain, _ = iters(False)
    it_pre, x_pre = iters(True)
    assert it_pre + 1 < it_plain
    maxit = it_pre + 1
    with pytest.raises(LinsolveError):
        PD.linear_solve_GPU(M, b, use_BiCG=True, tol=tol, max_iter=maxit, BiCG_with_preconditioner=False,
                            BiCG_precondition_fallback=False)
    x = PD.linear_solve_GPU(M, b, use_BiCG=True, tol=tol, max_iter=maxit, BiCG_with_preconditioner=False,
                            BiCG_precondition_fallback=True)
    assert torch.equal(x, x_pre)
    n = M.getRows()
    A = sp.csr_matrix((_np(M.value), M.index.cpu().numpy(), M.row.cpu().numpy()), shape=(n, n))
    r = _np(b) - A @ _np(x)
    assert np.sqrt(np.mean(r * r)) < tol


def test_simulation_fallback_flag_reaches_solve(ilu0_mode):
    """Simulation.linear_solve passes preconditionBiCG / BiCG_precondition_fallback to the solve
    (PISOtorch_simulation.py:896-903): a too-small iteration cap fails without the fallback and succeeds
    with it."""
    from pict_b200 import PISOtorch as P
    from pict_b200 import PISOtorch_simulation as S
    from pict_b200.engine import LinsolveError
    pd, M, b = _shifted_laplacian()
    x = torch.zeros_like(b)
    infos = P.SolveLinear(M, b, x, torch.IntTensor([2000]), torch.tensor([1e-9], dtype=torch.float64),
                          P.ConvergenceCriterion.NORM2_NORMALIZED, True, False, 0, False, False, False,
                          BiCGwithPreconditioner=True)
    maxit = infos[0].usedIterations + 1
    for fallback in (False, True):
        sim = S.Simulation(domain=pd, time_step=0.01, substeps=1, BiCG_precondition_fallback=fallback,
                           log_dir=None, save_domain_name=None)
        if fallback:
            y, ok = sim.linear_solve(M, b, use_BiCG=True, tol=1e-9, max_iter=maxit)
            assert ok and torch.equal(y, x)
        else:
            with pytest.raises(LinsolveError):
                sim.linear_solve(M, b, use_BiCG=True, tol=1e-9, max_iter=maxit)
