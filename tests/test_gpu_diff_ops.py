"""Operator-level differentiation (GPU): ``pict_b200.PISOtorch_diff`` behind
``Simulation(differentiable=True)`` (the reference's differentiable driver path,
PISOtorch_simulation.py:1054-1327 with PISOtorch_diff.py) against the fused, finite-difference-checked
rollout adjoint of ``pict_b200.adjoint`` on the same setups (FP64, solves to 1e-12).
"""
import pytest
import torch

from setups import build_product, case

pytestmark = pytest.mark.gpu
DT = 0.05
STEPS = 2


def _global(blocks, attr):
    D = blocks[0].velocity.shape[1]
    return torch.cat([getattr(b, attr).reshape(D, -1) for b in blocks], dim=1).reshape(-1)


@pytest.mark.parametrize("name", ["cavity2d", "twoblock2d_rotated", "periodic2d", "channel3d"])
def test_differentiable_simulation_matches_rollout_adjoint(name):
    from pict_b200.PISOtorch_simulation import Simulation
    from pict_b200.engine import PISOStepper
    from pict_b200.adjoint import PISOAdjoint, rollout
    g = torch.Generator(device="cpu").manual_seed(11)
    # operator-level autograd through the differentiable Simulation
    pd = build_product(case(name), torch.float64)
    blocks = pd.getBlocks()
    leaves = []
    for b in blocks:
        v = b.velocity.detach().clone().requires_grad_(True)
        b.setVelocity(v)
        leaves.append(v)
    nu = pd.viscosity.detach().clone().requires_grad_(True)
    pd.setViscosity(nu)
    pd.UpdateDomainData()
    N, D = pd.getTotalSize(), pd.getSpatialDims()
    w = torch.randn(D * N, generator=g, dtype=torch.float64).cuda()
    sim = Simulation(pd, time_step=DT, corrector_steps=2, advection_tol=1e-12, pressure_tol=1e-12,
                     differentiable=True, non_orthogonal=False)
    sim.run(iterations=STEPS)
    uT = _global(pd.getBlocks(), "velocity")
    (w * uT).sum().backward()
    g_ops = torch.cat([l.grad.reshape(D, -1) for l in leaves], dim=1).reshape(-1)
    g_nu_ops = float(nu.grad.reshape(-1)[0])
    # fused rollout adjoint on a fresh copy of the setup
    pd2 = build_product(case(name), torch.float64)
    st = PISOStepper(pd2, time_step=DT, advection_tol=1e-12, pressure_tol=1e-12)
    adj = PISOAdjoint(st)
    u0 = adj.velocity().clone().requires_grad_(True)
    nu2 = pd2._sim_visc.clone().requires_grad_(True)
    out = rollout(adj, u0, STEPS, [STEPS], nu=nu2)
    assert torch.allclose(out[0].detach(), uT.detach(), rtol=1e-9, atol=1e-11)
    (w * out[0]).sum().backward()
    scale = float(u0.grad.abs().max())
    assert float((g_ops - u0.grad).abs().max()) <= 1e-6 * scale
    assert abs(g_nu_ops - float(nu2.grad[0])) <= 1e-6 * abs(float(nu2.grad[0]))


def test_linear_solve_gpu_gradients():
    """linear_solve_GPU: d/d rhs and d/d matrix coefficients against finite differences (FP64)."""
    from pict_b200 import PISOtorch as P
    from pict_b200 import PISOtorch_diff as PD
    pd = build_product(case("twoblock2d_rotated"), torch.float64)
    ts = torch.tensor([DT], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupAdvectionVelocity(pd, ts, 0)
    g = torch.Generator(device="cpu").manual_seed(2)
    coef = pd.C.coef.detach().clone().requires_grad_(True)
    rhs = pd.velocityRHS.detach().clone().requires_grad_(True)
    w = torch.randn(rhs.numel(), generator=g, dtype=torch.float64).cuda()
    pd.C.setCoef(coef)
    x = PD.linear_solve_GPU(pd.C, rhs, use_BiCG=True, tol=1e-13)
    (w * x).sum().backward()
    dc = torch.randn(coef.shape, generator=g, dtype=torch.float64).cuda() * (coef.detach() != 0)
    dr = torch.randn(rhs.shape, generator=g, dtype=torch.float64).cuda()

    def L(e):
        with torch.no_grad():
            pd.C.setCoef(coef.detach() + e * dc)
            xx = PD.linear_solve_GPU(pd.C, rhs.detach() + e * dr, use_BiCG=True, tol=1e-13)
        return float((w * xx).sum())
    eps = 1e-6
    fd = (L(eps) - L(-eps)) / (2 * eps)
    ad = float((coef.grad * dc).sum() + (rhs.grad * dr).sum())
    assert abs(fd - ad) <= 1e-5 * abs(fd)


@pytest.mark.parametrize("name", ["cavity2d", "twoblock2d_rotated"])
def test_time_step_normalized_pressure_has_the_same_gradients(name):
    """Simulation(differentiable=True, pressure_time_step_normalized=True) solves for dt * p instead of p:
    the same step, so the gradients through the timeStepNorm operators (SetupPressureCorrection,
    CorrectVelocity) equal those of the plain form."""
    from pict_b200.PISOtorch_simulation import Simulation
    g = torch.Generator(device="cpu").manual_seed(12)
    grads = []
    for ts_norm in (False, True):
        pd = build_product(case(name), torch.float64)
        leaves = []
        for b in pd.getBlocks():
            v = b.velocity.detach().clone().requires_grad_(True)
            b.setVelocity(v)
            leaves.append(v)
        nu = pd.viscosity.detach().clone().requires_grad_(True)
        pd.setViscosity(nu)
        pd.UpdateDomainData()
        N, D = pd.getTotalSize(), pd.getSpatialDims()
        if not grads:
            w = torch.randn(D * N, generator=g, dtype=torch.float64).cuda()
        sim = Simulation(pd, time_step=DT, corrector_steps=2, advection_tol=1e-12, pressure_tol=1e-12,
                         differentiable=True, non_orthogonal=False, pressure_time_step_normalized=ts_norm)
        sim.run(iterations=STEPS)
        (w * _global(pd.getBlocks(), "velocity")).sum().backward()
        grads.append((torch.cat([l.grad.reshape(D, -1) for l in leaves], dim=1).reshape(-1), float(nu.grad.sum())))
    scale = float(grads[0][0].abs().max())
    assert float((grads[0][0] - grads[1][0]).abs().max()) <= 1e-7 * scale
    assert abs(grads[0][1] - grads[1][1]) <= 1e-7 * abs(grads[0][1])


@pytest.mark.parametrize("name", ["cavity2d", "twoblock2d_rotated", "channel3d"])
def test_apply_pressure_gradient_is_differentiable_in_the_pressure(name):
    """SetupAdvectionVelocity(apply_pressure_gradient=True) subtracts dt grad p: its gradient with respect
    to the blocks' pressure matches central differences (the term is linear in p), and the other
    gradients equal those without the term."""
    from pict_b200 import PISOtorch as P
    from pict_b200 import PISOtorch_diff as PD
    g = torch.Generator(device="cpu").manual_seed(13)
    pd = build_product(case(name), torch.float64)
    ts = torch.tensor([DT], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    blocks = pd.getBlocks()
    p0 = [torch.randn(b.pressure.shape, generator=g, dtype=torch.float64).cuda() for b in blocks]
    w = None

    def run(pressures, apply, with_grad):
        nonlocal w
        vs = []
        for b, p in zip(blocks, pressures):
            b.setPressure(p)
            v = b.velocity.detach().clone().requires_grad_(with_grad)
            b.setVelocity(v)
            vs.append(v)
        pd.UpdateDomainData()
        rhs = PD.SetupAdvectionVelocity(pd, ts, 0, apply_pressure_gradient=apply)
        if w is None:
            w = torch.randn(rhs.shape, generator=g, dtype=torch.float64).cuda()
        loss = (w * rhs).sum()
        if with_grad:
            loss.backward()
        return float(loss), vs

    leaves = [p.clone().requires_grad_(True) for p in p0]
    _, vs = run(leaves, True, True)
    gp = [l.grad.clone() for l in leaves]
    gv = [v.grad.clone() for v in vs]
    _, vs0 = run([p.clone() for p in p0], False, True)
    for a, b in zip(gv, vs0):
        assert torch.allclose(a, b.grad, rtol=1e-12, atol=1e-14)
    assert max(float(x.abs().max()) for x in gp) > 0
    eps = 1e-3
    for k in range(3):
        d = [torch.randn(p.shape, generator=g, dtype=torch.float64).cuda() for p in p0]
        lp, _ = run([p + eps * e for p, e in zip(p0, d)], True, False)
        lm, _ = run([p - eps * e for p, e in zip(p0, d)], True, False)
        fd = (lp - lm) / (2 * eps)
        an = sum(float((gg * e).sum()) for gg, e in zip(gp, d))
        assert abs(fd - an) <= 1e-8 * max(abs(fd), 1e-30)
