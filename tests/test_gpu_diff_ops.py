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
