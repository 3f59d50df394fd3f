"""Adjoint of the PISO step (GPU): gradients of the checkpointed rollout against central finite
differences of the forward step, in FP64 with tight solves.

Loss L = sum(w * u^T) after T = 2 steps.  Checked directions: initial velocity, system viscosity,
per-cell block viscosity, velocity source (static and per cell), boundary velocity of fixed faces
(static and varying).  Setups cover transforms (stretched / distorted grids), periodic and connected
(rotated) blocks, inflow boundaries and 3D.
"""
import numpy as np
import pytest
import torch

from setups import build_product, case

pytestmark = pytest.mark.gpu
DT = 0.05
T = 2
TOL = 1e-13
ADJ_CASES = ["cavity2d", "distorted2d", "periodic2d", "fullperiodic2d", "inflow2d", "twoblock2d_rotated",
             "channel3d", "twoblock3d"]


def _setup(name, dtype=torch.float64, tol=TOL):
    from pict_b200.engine import PISOStepper
    from pict_b200.adjoint import PISOAdjoint
    pd = build_product(case(name), dtype)
    pd.CreateVelocityGradOnBoundaries()
    for b in pd.getBlocks():
        b.CreateViscosityGrad()
        b.CreateVelocitySourceGrad()
    pd.UpdateDomainData()
    st = PISOStepper(pd, time_step=DT, advection_tol=tol, pressure_tol=tol, max_iterations=5000)
    adj = PISOAdjoint(st)
    adj.check_solves = True
    return pd, st, adj


def _loss(adj, u0, w):
    adj.set_velocity(u0)
    for _ in range(T):
        adj.st.step()
    adj.st.check()
    return float((w * adj.velocity()).sum())


def _fd(fn, eps):
    return (fn(eps) - fn(-eps)) / (2 * eps)


def _close(a, b, rtol=1e-4):
    assert abs(a - b) <= rtol * max(abs(a), abs(b), 1e-12), (a, b)


@pytest.mark.parametrize("name", ADJ_CASES)
def test_rollout_gradients_match_finite_differences(name):
    from pict_b200.adjoint import rollout
    pd, st, adj = _setup(name)
    g = torch.Generator(device="cpu").manual_seed(7)
    u0 = adj.velocity().clone()
    N, D = adj.N, adj.D
    w = torch.randn(D * N, generator=g, dtype=torch.float64).cuda()
    # adjoint
    u0r = u0.clone().requires_grad_(True)
    nu = pd._sim_visc.clone().requires_grad_(True)
    out = rollout(adj, u0r, T, [T], checkpoint_every=1, nu=nu)
    (w * out[0]).sum().backward()
    gu, gnu = u0r.grad.clone(), nu.grad.clone()
    blocks = pd.getBlocks()
    # initial velocity
    v = torch.randn(D * N, generator=g, dtype=torch.float64).cuda()
    eps = 1e-4 * float(u0.abs().max().clamp(min=1.0))
    _close(float((gu * v).sum()), _fd(lambda e: _loss(adj, u0 + e * v, w), eps))
    # system viscosity
    nu0 = pd._sim_visc.clone()

    def with_nu(e):
        pd._sim_visc.copy_(nu0 * (1 + e))
        return _loss(adj, u0, w)
    _close(float(gnu[0] * nu0[0]), _fd(with_nu, 1e-4))
    pd._sim_visc.copy_(nu0)
    # block parameters: viscosity, source, boundary velocity
    for b in blocks:
        params = []
        if b.viscosity is not None:
            params.append((b.viscosity, b.viscosityGrad))
        if b.velocitySource is not None:
            params.append((b.velocitySource, b.velocitySourceGrad))
        for f, bnd in enumerate(b.boundaries):
            if hasattr(bnd, "velocityGrad") and bnd.velocityGrad is not None and bnd.velocityGrad.numel() > 0:
                params.append((bnd.velocity, bnd.velocityGrad, f >> 1))
        for val, grad, *axis in params:
            dvec = torch.randn(val.shape, generator=g, dtype=torch.float64).cuda()
            if axis:
                # tangential boundary velocity only: a normal component would change the net inflow and
                # make the pressure system inconsistent
                dvec[:, axis[0]] = 0
            base = val.clone()
            scale = float(base.abs().max().clamp(min=1e-2))

            def with_param(e):
                val.copy_(base + e * dvec)
                return _loss(adj, u0, w)
            fd = _fd(with_param, 1e-4 * scale)
            val.copy_(base)
            _close(float((grad * dvec).sum()), fd)


def test_checkpointed_rollout_matches_stepwise_tape():
    """Windows of 3 steps over 7 steps with losses at steps 3, 5 and 7: same gradient as taping every
    step, and the domain keeps the forward end state."""
    from pict_b200.adjoint import rollout
    pd, st, adj = _setup("twoblock2d_rotated")
    g = torch.Generator(device="cpu").manual_seed(3)
    u0 = adj.velocity().clone()
    ws = [torch.randn(u0.numel(), generator=g, dtype=torch.float64).cuda() for _ in range(3)]
    grads = []
    for K in (1, 3):
        u0r = u0.clone().requires_grad_(True)
        outs = rollout(adj, u0r, 7, [3, 5, 7], checkpoint_every=K)
        sum((w * o).sum() for w, o in zip(ws, outs)).backward()
        grads.append(u0r.grad.clone())
        end = adj.velocity().clone()
        assert torch.equal(end, outs[-1].detach())
    assert torch.allclose(grads[0], grads[1], rtol=1e-10, atol=1e-14)


def test_rollout_last_window_taped_or_recomputed():
    """The forward pass tapes its last checkpoint window, which the backward pass then reverses without
    recomputing it.  When another rollout reuses the tapes before the backward pass, that window is
    recomputed from its checkpoint instead: same gradients either way, and the domain ends in the state
    at the end of its own forward pass."""
    from pict_b200.adjoint import rollout
    pd, st, adj = _setup("twoblock2d_rotated")
    g = torch.Generator(device="cpu").manual_seed(7)
    u0 = adj.velocity().clone()
    w = torch.randn(u0.numel(), generator=g, dtype=torch.float64).cuda()
    u0a = u0.clone().requires_grad_(True)
    (w * rollout(adj, u0a, 5, [5], checkpoint_every=2)[0]).sum().backward()
    u0b = u0.clone().requires_grad_(True)
    out_b = rollout(adj, u0b, 5, [5], checkpoint_every=2)[0]
    rollout(adj, (0.5 * u0).requires_grad_(True), 3, [3], checkpoint_every=2)  # reuses the tapes
    (w * out_b).sum().backward()
    assert torch.allclose(u0b.grad, u0a.grad, rtol=1e-8, atol=1e-12 * float(u0a.grad.abs().max()))
    assert torch.equal(adj.velocity(), out_b.detach())


def test_graphed_rollout_equals_eager():
    """With use_graph the backward pass replays per-slot CUDA graphs of the taped step and of the adjoint
    step: its gradients equal the eager pass's, also on a second pass through the same graphs, with a last
    checkpoint window shorter than the others and losses at two steps."""
    from pict_b200.adjoint import rollout
    pd, st, adj = _setup("twoblock2d_rotated")
    adj.check_solves = False
    st.capture(steps=1)
    g = torch.Generator(device="cpu").manual_seed(5)
    u0 = adj.velocity().clone()
    nu0 = pd._sim_visc.clone()
    ws = [torch.randn(u0.numel(), generator=g, dtype=torch.float64).cuda() for _ in range(2)]
    res = []
    for graphed in (False, True, True):
        adj.use_graph = graphed
        u0r = u0.clone().requires_grad_(True)
        nur = nu0.clone().requires_grad_(True)
        outs = rollout(adj, u0r, 7, [4, 7], checkpoint_every=3, nu=nur)
        sum((w * o).sum() for w, o in zip(ws, outs)).backward()
        res.append((u0r.grad.clone(), nur.grad.clone()))
        pd._sim_visc.copy_(nu0)
    for gu, gn in res[1:]:
        assert torch.allclose(gu, res[0][0], rtol=1e-8, atol=1e-12 * float(res[0][0].abs().max()))
        assert torch.allclose(gn, res[0][1], rtol=1e-8)
    assert len(adj._taped_graphs) == 3 and len(adj._back_graphs) == 3


def test_multigrid_adjoint_pressure_solves_equal_cg():
    """The transposed pressure solves preconditioned by the stepper's multigrid hierarchy give the gradients
    of the persistent CG solves (FP64, both to 1e-11 relative to their right-hand side), on a batch of two
    cavities through the refined step; the multigrid solves report convergence."""
    from pict_b200 import PISOtorch as P
    from pict_b200.adjoint import PISOAdjoint, rollout
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    from setups import lid_cavity
    sides = (24, 32)
    b = BatchDomain([build_product(lid_cavity(s, viscosity=1e-2), torch.float64) for s in sides],
                    time_steps=[0.5 / s for s in sides])
    st = PISOStepper(b, time_step=0.5 / sides[0], advection_tol=1e-12, pressure_tol=1e-12, pressure_refine=1,
                     refine_tol=1e-10, warm_start_pressure=True, pressure_first_solve=False, refine_solver="auto")
    assert st._mg is not None
    w = torch.linspace(-1, 1, 2 * b.getTotalSize(), dtype=torch.float64, device="cuda")
    grads = []
    for solver in ("cg", "mg"):
        for blk in b.getBlocks():
            blk.velocity.zero_()
            blk.pressure.zero_()
        adj = PISOAdjoint(st, relative_tolerance=True, adjoint_pressure_tol=1e-11, adjoint_advection_tol=1e-11,
                          adjoint_pressure_solver=solver)
        assert adj.p_mg == (solver == "mg")
        u0 = adj.velocity().clone().requires_grad_(True)
        nu = b._sim_visc.clone().requires_grad_(True)
        out = rollout(adj, u0, 3, [3], nu=nu)
        (w * out[0]).sum().backward()
        infos = P.decode_infos(adj.info)[2 * len(sides):]
        assert all(i.converged for i in infos), infos
        grads.append((u0.grad.clone(), nu.grad.clone()))
    (gu_cg, gn_cg), (gu_mg, gn_mg) = grads
    assert float((gu_mg - gu_cg).abs().max() / gu_cg.abs().max()) < 1e-8
    assert float((gn_mg - gn_cg).abs().max() / gn_cg.abs().max()) < 1e-8


def test_fp32_multigrid_adjoint_pressure_reaches_1e6_relative_on_large_cavities():
    """On 200^2 and 230^2 cavities a transposed pressure solve on FP32 vectors levels off between 1e-6 and
    6e-6 relative to its right-hand side; warm-started and refined in FP64, the multigrid adjoint pressure
    solves of the timed precision report convergence to 1e-6 relative, and the gradient is finite."""
    from pict_b200 import PISOtorch as P
    from pict_b200.adjoint import PISOAdjoint, rollout
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    from setups import lid_cavity
    sides = (200, 230)
    b = BatchDomain([build_product(lid_cavity(s, viscosity=1.0 / 2000), torch.float32) for s in sides],
                    time_steps=[0.5 / s for s in sides])
    st = PISOStepper(b, time_step=0.5 / sides[0], advection_tol=5e-7, pressure_tol=1e-6, pressure_refine=1,
                     refine_tol=5e-10, warm_start_pressure="increment", pressure_first_solve=False,
                     refine_solver="auto", warm_start_advection="increment")
    assert st._mg is not None
    for _ in range(5):
        st.step()
    adj = PISOAdjoint(st, relative_tolerance=True, adjoint_pressure_tol=1e-6)
    n_s = torch.diff(b._sim_cells.long()).cuda()
    w = torch.repeat_interleave(1.0 / n_s.float(), n_s).repeat(2)
    nu = b._sim_visc.clone().requires_grad_(True)
    out = rollout(adj, adj.velocity().clone(), 4, [4], checkpoint_every=2, nu=nu)
    (0.5 * (w * out[0] * out[0]).sum()).backward()
    infos = P.decode_infos(adj.info)[2 * len(sides):]
    assert all(i.converged and i.finalResidual <= 1e-6 for i in infos), infos
    assert bool(torch.isfinite(nu.grad).all())


def test_fp32_gradient_close_to_fp64():
    from pict_b200.adjoint import rollout
    res = []
    for dt_ in (torch.float64, torch.float32):
        pd, st, adj = _setup("cavity2d", dt_, tol=1e-12 if dt_ == torch.float64 else 1e-7)
        u0 = adj.velocity().clone()
        w = torch.linspace(-1, 1, u0.numel(), dtype=dt_, device="cuda")
        u0r = u0.clone().requires_grad_(True)
        nu = pd._sim_visc.clone().requires_grad_(True)
        out = rollout(adj, u0r, T, [T], nu=nu)
        (w * out[0]).sum().backward()
        res.append((u0r.grad.double(), nu.grad.double()))
    gu64, gn64 = res[0]
    gu32, gn32 = res[1]
    assert float((gu32 - gu64).abs().max() / gu64.abs().max()) < 1e-4
    assert float((gn32 - gn64).abs().max() / gn64.abs().max()) < 1e-3


def test_mixed_precision_viscosity_gradient_relative_adjoint():
    """The timed precision (FP32 fields, FP64 reductions, FP64 pressure refinement) with adjoint solves to
    1e-6 relative to their right-hand side: the viscosity gradient of the mean kinetic energy of two
    cavities (a loss whose gradient is ~1e-3 per cell) within 1e-4 of central differences of the FP64
    step, where adjoint solves to the same absolute tolerance are off by ~1e-2."""
    from pict_b200.adjoint import PISOAdjoint, rollout
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    from setups import lid_cavity
    sides, dts, steps = (32, 40), (0.5 / 32, 0.5 / 40), 3

    def batch(dtype):
        return BatchDomain([build_product(lid_cavity(s, viscosity=1.0 / 1500), dtype) for s in sides], time_steps=list(dts))
    b32 = batch(torch.float32)
    st32 = PISOStepper(b32, time_step=dts[0], advection_tol=1e-6, pressure_tol=1e-6, pressure_refine=1,
                       refine_tol=1e-9, warm_start_pressure=True, pressure_first_solve=False, refine_solver="auto")
    n_s = torch.diff(b32._sim_cells.long()).cuda()
    grads = []
    for relative in (True, False):
        for b in b32.getBlocks():
            b.velocity.zero_()
            b.pressure.zero_()
        adj = PISOAdjoint(st32, relative_tolerance=relative)
        w = torch.repeat_interleave(1.0 / n_s.float(), n_s).repeat(2)
        nu = b32._sim_visc.clone().requires_grad_(True)
        out = rollout(adj, adj.velocity().clone(), steps, [steps], nu=nu)
        (0.5 * (w * out[0] * out[0]).sum()).backward()
        grads.append(nu.grad.double().cpu())
    b64 = batch(torch.float64)
    st64 = PISOStepper(b64, time_step=dts[0], advection_tol=1e-12, pressure_tol=1e-12)
    adj64 = PISOAdjoint(st64)
    u0 = adj64.velocity().clone()
    nu0 = b64._sim_visc.clone()
    w64 = torch.repeat_interleave(1.0 / n_s.double(), n_s).repeat(2)
    for s in range(2):
        def loss(e):
            nu_ = nu0.clone()
            nu_[s] *= 1 + e
            b64._sim_visc.copy_(nu_)
            adj64.set_velocity(u0)
            for _ in range(steps):
                st64.step()
            st64.check()
            u = adj64.velocity()
            return float(0.5 * (w64 * u * u).sum())
        fd = (loss(1e-4) - loss(-1e-4)) / 2e-4
        rel = [abs(float(g[s]) * float(nu0[s]) - fd) / abs(fd) for g in grads]
        print("sim %d: FD %.6e, relative error of the FP32 adjoint: relative solves %.2e, absolute solves %.2e"
              % (s, fd, rel[0], rel[1]))
        assert rel[0] < 1e-4
