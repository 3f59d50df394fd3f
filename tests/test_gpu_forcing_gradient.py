"""Differentiable forcing (GPU): 128x128 periodic box, viscosity 1e-3, smooth random initial velocity
(spectrum ~ k^-3, k <= 8, seed 3) made divergence-free, 50 PISO steps, loss = mean squared error to
target velocities at steps 10, 20, ..., 50 produced by a hidden forcing (seed 4, same spectrum).
Gradient with respect to the per-cell forcing [1, 2, 128, 128] through the checkpointed adjoint
(checkpoints every 10 steps), checked against central finite differences on 16 seeded random unit
directions (seed 5, step 1e-3 of the forcing scale) and against the operator-level PISOtorch_diff
gradient of the differentiable Simulation.  FP64 with solves to 1e-12.
"""
import numpy as np
import pytest
import torch

from setups import build_product, forcing_box, spectral_field

pytestmark = pytest.mark.gpu
N = 128
STEPS = 50
REC = [10, 20, 30, 40, 50]
DT = 0.5 / N


@pytest.fixture(scope="module")
def problem():
    from pict_b200.PISOtorch_simulation import Simulation
    from pict_b200.engine import PISOStepper
    from pict_b200.adjoint import PISOAdjoint
    pd = build_product(forcing_box(N), torch.float64)
    sim = Simulation(pd, time_step=DT, pressure_tol=1e-12, advection_tol=1e-12, non_orthogonal=False)
    sim.make_divergence_free()
    st = PISOStepper(pd, time_step=DT, advection_tol=1e-12, pressure_tol=1e-12)
    adj = PISOAdjoint(st)
    adj.check_solves = True
    u0 = adj.velocity().clone()
    f_star = torch.tensor(0.5 * spectral_field(N, 4).reshape(-1), dtype=torch.float64, device="cuda")
    targets = run(adj, u0, f_star)
    return pd, adj, u0, f_star, targets


def run(adj, u0, f):
    adj.set_source(f)
    adj.set_velocity(u0)
    outs = []
    for t in range(1, STEPS + 1):
        adj.st.step()
        if t in REC:
            outs.append(adj.velocity().clone())
    adj.st.check()
    return outs


def loss_of(outs, targets):
    return sum(((o - t) ** 2).mean() for o, t in zip(outs, targets))


def test_forcing_gradient_matches_finite_differences(problem):
    from pict_b200.adjoint import rollout
    pd, adj, u0, f_star, targets = problem
    src = torch.zeros_like(f_star).requires_grad_(True)
    outs = rollout(adj, u0, STEPS, REC, checkpoint_every=10, src=src)
    loss_of(outs, targets).backward()
    g = src.grad.clone()
    gen = torch.Generator(device="cpu").manual_seed(5)
    eps = 1e-3 * float(f_star.abs().max())
    errs = []
    for _ in range(16):
        d = torch.randn(g.numel(), generator=gen, dtype=torch.float64).cuda()
        d /= d.norm()
        lp = float(loss_of(run(adj, u0, eps * d), targets))
        lm = float(loss_of(run(adj, u0, -eps * d), targets))
        fd = (lp - lm) / (2 * eps)
        ad = float((g * d).sum())
        errs.append(abs(ad - fd) / max(abs(fd), 1e-30))
    print("forcing gradient vs FD on 16 directions: max rel err %.2e" % max(errs))
    assert max(errs) < 1e-4


def test_forcing_gradient_matches_operator_level_diff(problem):
    from pict_b200.PISOtorch_simulation import Simulation
    from pict_b200.adjoint import rollout
    pd, adj, u0, f_star, targets = problem
    src = torch.zeros_like(f_star).requires_grad_(True)
    outs = rollout(adj, u0, STEPS, REC, checkpoint_every=10, src=src)
    loss_of(outs, targets).backward()
    g_fused = src.grad.clone()
    # operator-level autograd through the differentiable Simulation on a fresh domain
    pd2 = build_product(forcing_box(N), torch.float64)
    blk = pd2.getBlock(0)
    blk.setVelocity(u0.reshape(blk.velocity.shape).clone())
    f = torch.zeros(blk.velocitySource.shape, dtype=torch.float64, device="cuda", requires_grad=True)
    blk.setVelocitySource(f)
    pd2.UpdateDomainData()
    sim = Simulation(pd2, time_step=DT, pressure_tol=1e-12, advection_tol=1e-12, differentiable=True,
                     non_orthogonal=False)
    outs2 = []
    for _ in REC:
        sim.run(iterations=10)
        outs2.append(pd2.getBlock(0).velocity.reshape(-1))
    loss_of(outs2, targets).backward()
    g_ops = f.grad.reshape(-1)
    assert float((g_ops - g_fused).abs().max()) <= 1e-6 * float(g_fused.abs().max())
