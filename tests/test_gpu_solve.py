"""Krylov solver parity (GPU): persistent CG / BiCGStab kernels vs the oracle's restatement of the
reference's host loops (extensions/cg_solver_kernel.cu:236-427, extensions/bicgstab_solver_kernel.cu:240-360) and vs a direct solve.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import piso_oracle as po
from setups import ALL_CASES, build_oracle, build_product, case

pytestmark = pytest.mark.gpu
DT = 0.05


def _np(t):
    return t.detach().double().cpu().numpy()


def _relerr(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", ALL_CASES)
@pytest.mark.parametrize("group_size", [1, 3])
def test_bicgstab_velocity(name, group_size):
    from pict_b200 import PISOtorch as P
    spec = case(name)
    od = build_oracle(spec)
    pd = build_product(spec, torch.float64)
    Cref, _ = po.advection_matrix(od, DT)
    rhs = po.advection_rhs(od, DT)
    Cm = po.stencil_to_scipy(od, Cref)
    ts = torch.tensor([DT], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupAdvectionVelocity(pd, ts, 0)
    x = torch.zeros_like(pd.velocityRHS)
    params = P._solve_params(spec["dims"], 1000, 1e-12, 1, True, False, x_zero=True, group_size=group_size)
    info = P.decode_infos(P.solve_stencil(pd, pd.C.coef, pd.velocityRHS, x, params))
    xs = _np(x).reshape(spec["dims"], -1)
    for c in range(spec["dims"]):
        xref, iref = po.bicgstab(Cm, rhs[c], tol=1e-12, maxit=1000)
        xd = spla.spsolve(Cm.tocsc(), rhs[c])
        assert info[c].converged and info[c].isFiniteResidual
        assert abs(info[c].usedIterations - iref.usedIterations) <= 1, (info[c], iref)
        assert _relerr(xs[c], xd) < 1e-9
        assert _relerr(xs[c], xref) < 1e-9


@pytest.mark.parametrize("name", ALL_CASES)
@pytest.mark.parametrize("group_size", [1, 4])
@pytest.mark.parametrize("variant", [0, 1])
def test_cg_pressure(name, group_size, variant):
    from pict_b200 import PISOtorch as P
    spec = case(name)
    od = build_oracle(spec)
    pd = build_product(spec, torch.float64)
    Cref, Aref = po.advection_matrix(od, DT)
    h = po.pressure_rhs(od, DT, Cref, Aref, od.velocity_global())
    div = po.divergence(od, h)
    Pm = po.stencil_to_scipy(od, po.pressure_matrix(od, Aref))
    ts = torch.tensor([DT], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.CopyVelocityResultFromBlocks(pd)
    P.SetupPressureCorrection(pd, ts)
    x = torch.zeros_like(pd.pressureRHSdiv)
    params = P._solve_params(1, 2000, 1e-12, 1, False, False, x_zero=True, group_size=group_size, variant=variant)
    info = P.decode_infos(P.solve_stencil(pd, pd.P.coef, pd.pressureRHSdiv, x, params))[0]
    xref, iref = po.cg(Pm, div, tol=1e-12, maxit=2000)
    assert info.converged and info.isFiniteResidual, info
    assert abs(info.usedIterations - iref.usedIterations) <= 2, (info, iref)
    # the Laplacian is singular on closed domains: compare mean-free solutions
    xg = _np(x)
    assert _relerr(xg - xg.mean(), xref - xref.mean()) < 1e-8


def test_solve_linear_api_and_transpose():
    from pict_b200 import PISOtorch as P
    spec = case("twoblock2d_rotated")
    od = build_oracle(spec)
    pd = build_product(spec, torch.float64)
    ts = torch.tensor([DT], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    Cref, _ = po.advection_matrix(od, DT)
    Cm = po.stencil_to_scipy(od, Cref)
    rng = np.random.default_rng(3)
    b = rng.standard_normal(2 * od.N)
    x = torch.zeros(2 * od.N, dtype=torch.float64, device="cuda")
    infos = P.SolveLinear(pd.C, torch.tensor(b, device="cuda"), x, torch.IntTensor([500]), torch.tensor([1e-12], dtype=torch.float64),
                          P.ConvergenceCriterion.NORM2_NORMALIZED, True, False, 0, False, False, False, False)
    assert len(infos) == 2 and all(i.converged for i in infos)
    xs = _np(x).reshape(2, -1)
    for c in range(2):
        assert _relerr(xs[c], spla.spsolve(Cm.tocsc(), b[c * od.N:(c + 1) * od.N])) < 1e-9
    # transposed solve (adjoint): A^T x = b
    x.zero_()
    infos = P.SolveLinear(pd.C, torch.tensor(b, device="cuda"), x, 500, 1e-12, useBiCG=True, transposeA=True,
                          BiCGwithPreconditioner=False)
    xs = _np(x).reshape(2, -1)
    for c in range(2):
        assert _relerr(xs[c], spla.spsolve(Cm.T.tocsc(), b[c * od.N:(c + 1) * od.N])) < 1e-9


def test_zero_rhs_and_nonconvergence_reports():
    from pict_b200 import PISOtorch as P
    spec = case("cavity2d")
    pd = build_product(spec, torch.float32)
    ts = torch.tensor([DT], dtype=torch.float32)
    P.SetupAdvectionMatrix(pd, ts, 0)
    x = torch.full_like(pd.velocityRHS, 3.0)
    zero = torch.zeros_like(pd.velocityRHS)
    infos = P.SolveLinear(pd.C, zero, x, 100, 1e-6, useBiCG=True, BiCGwithPreconditioner=False)
    assert all(i.converged for i in infos)
    assert float(x.abs().max()) == 0.0  # an all-zero RHS gives x = 0 (PISOtorch_diff.py:245-293)
    P.SetupAdvectionVelocity(pd, ts, 0)
    x = torch.zeros_like(pd.velocityRHS)
    infos = P.SolveLinear(pd.C, pd.velocityRHS, x, 1, 1e-30, useBiCG=True, BiCGwithPreconditioner=False)
    assert all((not i.converged) and i.usedIterations == 0 for i in infos)
    # non-finite input -> isFiniteResidual False, no hang
    rhs = pd.velocityRHS.clone()
    rhs[5] = float("nan")
    x = torch.zeros_like(rhs)
    infos = P.SolveLinear(pd.C, rhs, x, 50, 1e-6, useBiCG=True, BiCGwithPreconditioner=False)
    assert not infos[0].isFiniteResidual and not infos[0].converged
