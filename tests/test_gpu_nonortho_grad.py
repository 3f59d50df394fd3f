"""Gradients of the non-orthogonal terms (nonOrthoFlags) through the raw gradient operators (GPU).

Fixtures: tests/golden/ref_nonortho_grad_*.npz, generated on a B200 by
tests/golden/make_ref_nonortho_grad_fixtures.py from the reference's compiled module: each raw gradient
operator (SetupAdvectionMatrixGrad, SetupAdvectionVelocityGrad, SetupPressureMatrixGrad,
SetupPressureRHSdivGrad, SetupPressureRHSGrad) once, with seeded gradient inputs, on skewed and distorted
2D/3D grids with a per-cell block viscosity, for the flag sets 25, 27 and 19.  The same function runs
here with this library's module; FP64 results must agree to round-off.

Independent of the fixtures, dot-product tests check that the operators are the adjoints of the
forward operators: the forward terms are linear in the result fields, and the finite difference of
<out_bar, F(x)> along a random direction equals <x_bar, direction>.
"""
import os
import sys

import numpy as np
import pytest
import torch

from setups import NONORTHO_CASES, build_product

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_ref_nonortho_grad_fixtures as G  # noqa: E402


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64).reshape(-1), np.asarray(b, dtype=np.float64).reshape(-1)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", NONORTHO_CASES)
def test_nonortho_raw_grad_operators_match_reference(name):
    from pict_b200 import PISOtorch as P
    p = os.path.join(GOLDEN, "ref_nonortho_grad_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    fx = np.load(p)
    out = G.grad_ops_fixture(P, name)
    errs = {}
    for key in fx.files:
        assert key in out, key
        assert out[key].size == fx[key].size, key
        if np.abs(fx[key]).max() == 0 and np.abs(out[key]).max() == 0:
            continue
        errs[key] = _rel(out[key], fx[key])
    worst = sorted(errs.items(), key=lambda kv: -kv[1])[:6]
    print(name, {k: "%.1e" % v for k, v in worst})
    assert max(errs.values()) < 1e-10, worst


def _dot(a, b):
    return float((a.double().reshape(-1) * b.double().reshape(-1)).sum())


@pytest.mark.parametrize("flags", [25, 27, 19])
@pytest.mark.parametrize("name", ["distorted2d", "skewed_twoblock2d_rotated", "skewed_cavity3d", "skewed_inflow2d"])
def test_nonortho_rhs_gradients_are_adjoints(name, flags):
    """velocityRHS and pressureRHSdiv are affine in velocityResult / pressureResult: the gradient operators
    must return exactly the transposed linear maps."""
    from pict_b200 import PISOtorch as P
    from setups import case
    spec = case(name)
    pd = build_product(spec, torch.float64)
    D, N = pd.getSpatialDims(), pd.getTotalSize()
    ts = torch.tensor([0.05], dtype=torch.float64)
    g = torch.Generator(device="cpu").manual_seed(3 + flags)
    rnd = lambda n: torch.randn(n, generator=g, dtype=torch.float64).cuda()
    U, dU = rnd(D * N) * 0.3, rnd(D * N)
    P.SetupAdvectionMatrix(pd, ts, flags)

    def vrhs(u):
        pd.setVelocityResult(u.clone())
        pd.UpdateDomainData()
        P.SetupAdvectionVelocity(pd, ts, flags, False)
        return pd.velocityRHS.clone()

    rb = rnd(D * N)
    lin = _dot(rb, vrhs(U + dU) - vrhs(U))
    pd.setVelocityResult(U.clone())
    pd.setVelocityRHSGrad(rb)
    pd.CreateVelocityResultGrad()
    pd.CreateViscosityGrad()
    pd.CreateVelocityGradOnBlocks()
    pd.CreateVelocityGradOnBoundaries()
    pd.UpdateDomainData()
    P.SetupAdvectionVelocityGrad(pd, ts, flags, False)
    adj = _dot(pd.velocityResultGrad, dU)
    assert abs(lin - adj) <= 1e-11 * max(abs(lin), 1e-30) + 1e-13, (lin, adj)

    pd.setVelocityResult(U.clone())
    pd.UpdateDomainData()
    P.SetupPressureMatrix(pd, ts, flags, False)
    p0, dp = rnd(N), rnd(N)

    def prhs(p):
        pd.setPressureResult(p.clone())
        pd.UpdateDomainData()
        P.SetupPressureRHS(pd, ts, flags, False, timeStepNorm=False)
        return pd.pressureRHSdiv.clone()

    db = rnd(N)
    lin = _dot(db, prhs(p0 + dp) - prhs(p0))
    pd.setPressureResult(p0.clone())
    pd.setPressureRHSdivGrad(db)
    pd.CreatePressureRHSGrad()
    pd.CreatePressureResultGrad()
    pd.CreateAGrad()
    pd.UpdateDomainData()
    P.SetupPressureRHSdivGrad(pd, ts, flags, False, timeStepNorm=False)
    adj = _dot(pd.pressureResultGrad, dp)
    assert abs(lin - adj) <= 1e-11 * max(abs(lin), 1e-30) + 1e-13, (lin, adj)


@pytest.mark.parametrize("name", ["distorted2d", "skewed_twoblock2d", "skewed_channel3d"])
def test_nonortho_coefficient_gradients_match_central_differences(name):
    """Viscosity gradient of the advection matrix and A gradient of the pressure matrix and pressure RHS
    (orthogonal + non-orthogonal parts) against central differences of the forward operators."""
    from pict_b200 import PISOtorch as P
    flags = 25 | 2
    spec = G.viscous_spec(name)
    pd = build_product(spec, torch.float64)
    D, N = pd.getSpatialDims(), pd.getTotalSize()
    ts = torch.tensor([0.05], dtype=torch.float64)
    g = torch.Generator(device="cpu").manual_seed(9)
    rnd = lambda *s: torch.randn(*s, generator=g, dtype=torch.float64).cuda()
    nu0 = [b.viscosity.clone() for b in pd.getBlocks()]
    dnu = [rnd(*v.shape) * 1e-3 for v in nu0]
    Cb, Ab = rnd(pd.C.value.numel()), rnd(N)

    def cmat(eps):
        for b, v, d in zip(pd.getBlocks(), nu0, dnu):
            b.setViscosity(v + eps * d)
        pd.UpdateDomainData()
        P.SetupAdvectionMatrix(pd, ts, flags)
        return _dot(Cb, pd.C.value) + _dot(Ab, pd.A)

    eps = 1e-3
    fd = (cmat(eps) - cmat(-eps)) / (2 * eps)
    cmat(0.0)
    pd.CGrad.setValue(Cb)
    pd.setAGrad(Ab)
    pd.CreateViscosityGrad()
    pd.CreateVelocityGradOnBlocks()
    pd.CreateVelocityGradOnBoundaries()
    pd.UpdateDomainData()
    P.SetupAdvectionMatrixGrad(pd, ts, flags)
    an = sum(_dot(b.viscosityGrad, d) for b, d in zip(pd.getBlocks(), dnu))
    assert abs(fd - an) <= 1e-8 * abs(fd) + 1e-14, (fd, an)

    # pressure matrix + explicit pressure terms in A
    U, p = rnd(D * N) * 0.3, rnd(N)
    A0 = pd.A.clone()
    dA = rnd(N) * 1e-3 * A0.abs().max()
    Pb, db = rnd(pd.P.value.numel()), rnd(N)

    def pmat(eps):
        pd.setA(A0 + eps * dA)
        pd.setVelocityResult(U.clone())
        pd.setPressureResult(p.clone())
        pd.UpdateDomainData()
        P.SetupPressureMatrix(pd, ts, flags, False)
        P.SetupPressureRHSdiv(pd, ts, flags, False, timeStepNorm=False)
        return _dot(Pb, pd.P.value) + _dot(db, pd.pressureRHSdiv)

    fd = (pmat(eps) - pmat(-eps)) / (2 * eps)
    pmat(0.0)
    pd.PGrad.setValue(Pb)
    pd.CreateAGrad()
    pd.UpdateDomainData()
    P.SetupPressureMatrixGrad(pd, ts, flags, False)
    pd.setPressureRHSdivGrad(db)
    pd.CreatePressureRHSGrad()
    pd.CreatePressureResultGrad()
    pd.UpdateDomainData()
    P.SetupPressureRHSdivGrad(pd, ts, flags, False, timeStepNorm=False)
    an = _dot(pd.AGrad, dA)
    assert abs(fd - an) <= 1e-7 * abs(fd) + 1e-14, (fd, an)


@pytest.mark.parametrize("flags", [25, 27, 19])
@pytest.mark.parametrize("name", ["distorted2d", "skewed_twoblock2d_rotated", "skewed_cavity3d", "skewed_inflow2d"])
def test_nonortho_autograd_functions_match_central_differences(name, flags):
    """PISOtorch_diff's SetupAdvectionMatrix -> SetupAdvectionVelocity -> SetupPressureCorrection chain with
    non-orthogonal flags: the directional derivative of a weighted sum of all their outputs (C, A, velocity
    RHS, P, H/A, its divergence) along viscosity, velocity result and pressure result, against central
    differences (FP64; the operators are smooth, so only O(eps^2) and round-off separate the two)."""
    from pict_b200 import PISOtorch_diff as PD
    pd = build_product(G.viscous_spec(name), torch.float64)
    D, N = pd.getSpatialDims(), pd.getTotalSize()
    ts = torch.tensor([0.05], dtype=torch.float64)
    g = torch.Generator(device="cpu").manual_seed(100 + flags)
    rnd = lambda *s: torch.randn(*s, generator=g, dtype=torch.float64).cuda()
    blocks = pd.getBlocks()
    nu0 = [b.viscosity.detach().clone() for b in blocks]
    U0, p0 = rnd(D * N) * 0.3, rnd(N)
    dnu = [rnd(*v.shape) * 2e-3 for v in nu0]
    dU, dp = rnd(D * N) * 0.3, rnd(N)
    weights = []

    def run(eps, grad):
        nus = [(v + eps * d).requires_grad_(grad) for v, d in zip(nu0, dnu)]
        for b, v in zip(blocks, nus):
            b.setViscosity(v)
        U = (U0 + eps * dU).requires_grad_(grad)
        p = (p0 + eps * dp).requires_grad_(grad)
        pd.setVelocityResult(U)
        pd.setPressureResult(p)
        pd.UpdateDomainData()
        A, C = PD.SetupAdvectionMatrix(pd, ts, flags)
        rhs = PD.SetupAdvectionVelocity(pd, ts, flags)
        PD.SetupPressureCorrection(pd, ts, flags)
        outs = [C, A, rhs, pd.P.coef, pd.pressureRHS, pd.pressureRHSdiv]
        if not weights:
            weights.extend(rnd(*o.shape) for o in outs)
        L = sum((w * o).sum() for w, o in zip(weights, outs))
        return L, nus, U, p

    L, nus, U, p = run(0.0, True)
    L.backward()
    an = sum(_dot(v.grad, d) for v, d in zip(nus, dnu)) + _dot(U.grad, dU) + _dot(p.grad, dp)
    assert p.grad.abs().max() > 0  # the explicit pressure terms are tracked
    eps = 1e-4
    with torch.no_grad():
        fd = (float(run(eps, False)[0]) - float(run(-eps, False)[0])) / (2 * eps)
    assert abs(fd - an) <= 1e-7 * abs(fd), (fd, an)


PTOL = 1e-10


@pytest.mark.parametrize("name", ["skewed_cavity3d", "skewed_twoblock2d", "distorted2d"])
def test_differentiable_non_orthogonal_simulation_step(name):
    """Simulation(differentiable=True, non_orthogonal=True): one PISO step of the non-orthogonal branch
    through PISOtorch_diff, from rest with a lid or a source driving the flow; the gradient of <w, u>
    w.r.t. the initial velocity and the block viscosity, against central differences.

    The non-orthogonal matrix terms make P non-symmetric, so the pressure is solved with BiCGStab, to
    1e-10.  Next to walls the one-sided corner treatment leaves P's rows not exactly summing to zero: P
    is then regular but close to singular, and central differences of the solves carry noise of about
    1e-3 relative (they move by that much between eps 1e-3 and 1e-4).  The adjoint must agree with the
    closer of the two to 1e-3."""
    from make_ref_nonortho_fixtures import rest_spec
    from pict_b200.PISOtorch_simulation import Simulation
    g = torch.Generator(device="cpu").manual_seed(5)
    spec = G.viscous_spec(name, rest_spec(name))
    D = spec["dims"]

    def run(eps, du, dnu, grad):
        pd = build_product(spec, torch.float64)
        leaves = []
        for k, b in enumerate(pd.getBlocks()):
            v = (b.velocity.detach() + eps * du[k]).requires_grad_(grad)
            n = (b.viscosity.detach() + eps * dnu[k]).requires_grad_(grad)
            b.setVelocity(v)
            b.setViscosity(n)
            leaves.append((v, n))
        pd.UpdateDomainData()
        sim = Simulation(pd, time_step=0.02, corrector_steps=2, advection_tol=1e-12, pressure_tol=PTOL,
                         differentiable=grad, non_orthogonal=True, velocity_corrector="FD")
        sim.pressure_use_BiCG = True  # P is not symmetric with the non-orthogonal matrix terms
        assert sim._non_ortho_flags() == 25
        assert sim._PISO_split_step(1)
        u = torch.cat([b.velocity.reshape(D, -1) for b in pd.getBlocks()], dim=1)
        return u, leaves

    pd0 = build_product(spec, torch.float64)
    du = [torch.randn(b.velocity.shape, generator=g, dtype=torch.float64).cuda() for b in pd0.getBlocks()]
    dnu = [torch.randn(b.viscosity.shape, generator=g, dtype=torch.float64).cuda() * 1e-2 for b in pd0.getBlocks()]
    u, leaves = run(0.0, du, dnu, True)
    w = torch.randn(u.shape, generator=g, dtype=torch.float64).cuda()
    (w * u).sum().backward()
    an = sum(_dot(v.grad, a) + _dot(n.grad, b) for (v, n), a, b in zip(leaves, du, dnu))
    fds = []
    for eps in (1e-3, 1e-4):
        with torch.no_grad():
            up = run(eps, du, dnu, False)[0]
            um = run(-eps, du, dnu, False)[0]
        fds.append(_dot(w, up - um) / (2 * eps))
    rel = min(abs(fd - an) / abs(fd) for fd in fds)
    print(name, "fd %.10e / %.10e (eps 1e-3 / 1e-4) adjoint %.10e rel %.2e" % (fds[0], fds[1], an, rel))
    assert rel <= 1e-3, (fds, an)
