"""Gradients of the passive scalar operators (SetupAdvectionMatrixGrad with forPassiveScalar,
SetupAdvectionScalarGrad, CopyScalarResultGrad*) against the reference's own CUDA build (GPU).

Fixtures: tests/golden/ref_scalar_grad_*.npz from tests/golden/make_ref_scalar_grad_fixtures.py (seeded
gradient inputs, nonOrthoFlags 0, 25 and 27); the same function runs here with this library's module.
Independent of the fixtures, a dot-product test checks that the scalar RHS gradient is the adjoint of
the forward operator in the block scalar, the boundary scalars and the scalar result.
"""
import os
import sys

import numpy as np
import pytest
import torch

from setups import SCALAR_CASES, build_product, scalar_case

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_ref_scalar_grad_fixtures as G  # noqa: E402


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64).reshape(-1), np.asarray(b, dtype=np.float64).reshape(-1)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", SCALAR_CASES)
def test_scalar_grad_operators_match_reference(name):
    from pict_b200 import PISOtorch as P
    p = os.path.join(GOLDEN, "ref_scalar_grad_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    fx = np.load(p)
    out = G.scalar_grad_fixture(P, name)
    errs = {}
    for key in fx.files:
        assert key in out, key
        assert out[key].size == fx[key].size, key
        if np.abs(fx[key]).max() == 0 and np.abs(out[key]).max() == 0:
            continue
        errs[key] = _rel(out[key], fx[key])
    worst = sorted(errs.items(), key=lambda kv: -kv[1])[:5]
    print(name, {k: "%.1e" % v for k, v in worst})
    assert max(errs.values()) < 1e-10, worst


def _dot(a, b):
    return float((a.double().reshape(-1) * b.double().reshape(-1)).sum())


@pytest.mark.parametrize("flags", [0, 27])
@pytest.mark.parametrize("name", ["scalar_cavity2d", "scalar_inflow2d", "scalar_skewed_cavity3d"])
def test_scalar_rhs_gradient_is_the_adjoint(name, flags):
    """scalarRHS is linear in the block scalar, the boundary scalars and the scalar result: the gradient
    operator must return the transposed maps."""
    from pict_b200 import PISOtorch as P
    pd = build_product(scalar_case(name), torch.float64)
    C, N = pd.getPassiveScalarChannels(), pd.getTotalSize()
    ts = torch.tensor([0.05], dtype=torch.float64)
    g = torch.Generator(device="cpu").manual_seed(7 + flags)
    rnd = lambda *s: torch.randn(*s, generator=g, dtype=torch.float64).cuda()
    blocks = pd.getBlocks()
    fixed = [(b, bnd) for b in blocks for bnd in b.boundaries if isinstance(bnd, P.FixedBoundary)]
    s0 = [b.passiveScalar.clone() for b in blocks]
    sb0 = [bnd.passiveScalar.clone() for _, bnd in fixed]
    r0 = rnd(C * N)
    ds = [rnd(*x.shape) for x in s0]
    dsb = [rnd(*x.shape) for x in sb0]
    dr = rnd(C * N)

    def rhs(eps):
        for b, x, d in zip(blocks, s0, ds):
            b.setPassiveScalar(x + eps * d)
        for (_, bnd), x, d in zip(fixed, sb0, dsb):
            bnd.setPassiveScalar(x + eps * d)
        pd.setScalarResult(r0 + eps * dr)
        pd.UpdateDomainData()
        P.SetupAdvectionScalar(pd, ts, flags)
        return pd.scalarRHS.clone()

    w = rnd(C * N)
    lin = _dot(w, rhs(1.0) - rhs(0.0))
    pd.setScalarRHSGrad(w)
    pd.CreateScalarResultGrad()
    pd.CreatePassiveScalarGradOnBlocks()
    pd.CreatePassiveScalarGradOnBoundaries()
    pd.CreateVelocityGradOnBoundaries()
    pd.CreateViscosityGrad()
    pd.UpdateDomainData()
    P.SetupAdvectionScalarGrad(pd, ts, flags)
    adj = sum(_dot(b.passiveScalarGrad, d) for b, d in zip(blocks, ds))
    adj += sum(_dot(bnd.passiveScalarGrad, d) for (_, bnd), d in zip(fixed, dsb))
    adj += _dot(pd.scalarResultGrad, dr)
    assert abs(lin - adj) <= 1e-11 * abs(lin), (lin, adj)


@pytest.mark.parametrize("name", ["scalar_cavity2d", "scalar_inflow2d", "scalar_twoblock2d_rotated"])
def test_differentiable_simulation_scalar_gradients(name):
    """Simulation(differentiable=True) with passive scalar advection: the gradient of <w, s> after one step
    w.r.t. the initial block scalar, the initial velocity and the scalar (or domain) viscosity, against
    central differences (FP64, solves to 1e-12)."""
    from pict_b200.PISOtorch_simulation import Simulation
    spec = scalar_case(name)
    g = torch.Generator(device="cpu").manual_seed(3)

    def run(eps, ds, du, dnu, grad):
        pd = build_product(spec, torch.float64)
        leaves = []
        for k, b in enumerate(pd.getBlocks()):
            s = (b.passiveScalar.detach() + eps * ds[k]).requires_grad_(grad)
            v = (b.velocity.detach() + eps * du[k]).requires_grad_(grad)
            b.setPassiveScalar(s)
            b.setVelocity(v)
            leaves += [s, v]
        if pd.passiveScalarViscosity is not None:
            nu = (pd.passiveScalarViscosity.detach() + eps * dnu).requires_grad_(grad)
            pd.setScalarViscosity(nu)
            leaves.append(nu)
        pd.UpdateDomainData()
        sim = Simulation(pd, time_step=0.05, corrector_steps=2, advection_tol=1e-12, pressure_tol=1e-12,
                         differentiable=grad, non_orthogonal=False, advect_passive_scalar=True)
        assert sim._PISO_split_step(1)
        C = pd.getPassiveScalarChannels()
        return torch.cat([b.passiveScalar.reshape(C, -1) for b in pd.getBlocks()], dim=1), leaves

    pd0 = build_product(spec, torch.float64)
    ds = [torch.randn(b.passiveScalar.shape, generator=g, dtype=torch.float64).cuda() for b in pd0.getBlocks()]
    du = [torch.randn(b.velocity.shape, generator=g, dtype=torch.float64).cuda() * 0.1 for b in pd0.getBlocks()]
    sv = pd0.passiveScalarViscosity
    dnu = None if sv is None else torch.randn(sv.shape, generator=g, dtype=torch.float64).cuda() * 1e-3
    s, leaves = run(0.0, ds, du, dnu, True)
    w = torch.randn(s.shape, generator=g, dtype=torch.float64).cuda()
    (w * s).sum().backward()
    dirs = []
    for k in range(len(ds)):
        dirs += [ds[k], du[k]]
    if dnu is not None:
        dirs.append(dnu)
    an = sum(_dot(l.grad, d) for l, d in zip(leaves, dirs))
    eps = 1e-5
    with torch.no_grad():
        fd = (_dot(w, run(eps, ds, du, dnu, False)[0]) - _dot(w, run(-eps, ds, du, dnu, False)[0])) / (2 * eps)
    print(name, fd, an)
    assert abs(fd - an) <= 1e-6 * abs(fd), (fd, an)
