"""Batched simulations (GPU): many independent domains advanced in one launch per stage give the same
results as advancing each domain alone, and the Krylov results do not depend on the launch shape."""
import numpy as np
import pytest
import torch

from setups import build_product, case, lid_cavity

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().double().cpu().numpy()


def test_batch_equals_individual_steps():
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    specs = [lid_cavity(n, viscosity=v) for n, v in [(20, 1e-2), (33, 2e-3), (48, 1e-3), (17, 5e-3)]]
    specs.append(case("twoblock2d"))
    dts = [0.01, 0.008, 0.005, 0.02, 0.01]
    solo = [build_product(s, torch.float32) for s in specs]
    batched = [build_product(s, torch.float32) for s in specs]
    for d, dt in zip(solo, dts):
        st = PISOStepper(d, time_step=dt, advection_tol=1e-6, pressure_tol=1e-6)
        for _ in range(3):
            st.step()
        st.check()
    b = BatchDomain(batched, time_steps=dts)
    sb = PISOStepper(b, time_step=dts[0], advection_tol=1e-6, pressure_tol=1e-6)
    for _ in range(3):
        sb.step()
    sb.check()
    for d1, d2 in zip(solo, batched):
        for b1, b2 in zip(d1.getBlocks(), d2.getBlocks()):
            assert np.array_equal(_np(b1.velocity), _np(b2.velocity))
            assert np.array_equal(_np(b1.pressure), _np(b2.pressure))


@pytest.mark.parametrize("use_bicg,variant", [(False, 0), (False, 1), (True, 0)])
def test_solver_independent_of_grid_size(use_bicg, variant):
    from pict_b200 import PISOtorch as P
    spec = lid_cavity(96, viscosity=1e-3)
    d = build_product(spec, torch.float32)
    ts = torch.tensor([0.01], dtype=torch.float32)
    P.SetupAdvectionMatrix(d, ts, 0)
    P.SetupAdvectionVelocity(d, ts, 0)
    P.CopyVelocityResultFromBlocks(d)
    P.SetupPressureCorrection(d, ts)
    coef = d.C.coef if use_bicg else d.P.coef
    rhs = d.velocityRHS if use_bicg else d.pressureRHSdiv
    nrhs = 2 if use_bicg else 1
    outs = []
    for grid in [0, 1, 2, 3]:
        x = torch.zeros_like(rhs)
        prm = P._solve_params(nrhs, 2000, 1e-7, 1, use_bicg, False, x_zero=True, group_size=grid, variant=variant)
        infos = P.decode_infos(P.solve_stencil(d, coef, rhs, x, prm))
        assert all(i.converged for i in infos)
        outs.append((_np(x), [i.usedIterations for i in infos]))
    for x, its in outs[1:]:
        assert np.array_equal(x, outs[0][0]) and its == outs[0][1]


def test_many_uneven_systems_single_reduction_cg():
    """Many systems converging at different iterations in one persistent launch (exit decision must be
    identical in every CTA; a disagreement would surface as a barrier timeout)."""
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    rng = np.random.default_rng(5)
    sides = rng.integers(12, 80, size=48)
    doms = [build_product(lid_cavity(int(s), viscosity=float(1e-3 + 1e-2 * rng.random())), torch.float32) for s in sides]
    b = BatchDomain(doms, time_steps=[0.5 / s for s in sides])
    for variant in (0, 1):
        st = PISOStepper(b, time_step=0.01, advection_tol=1e-6, pressure_tol=1e-6, cg_variant=variant)
        for _ in range(3):
            st.step()
        adv, ps = st.check()
        assert all(i.status == 0 for i in adv) and all(i.status == 0 for p in ps for i in p)


def test_packed_batch_state_gives_the_same_steps():
    """BatchDomain.pack_state moves the blocks' fields into two contiguous tensors (views): the batched
    steps are unchanged, the member domains see the state through their blocks, and one copy of the
    arenas moves the whole state."""
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    specs = [lid_cavity(n, viscosity=v) for n, v in [(20, 1e-2), (33, 2e-3)]] + [case("twoblock2d")]
    dts = [0.01, 0.008, 0.01]
    plain = [build_product(s, torch.float32) for s in specs]
    packed = [build_product(s, torch.float32) for s in specs]
    b1 = BatchDomain(plain, time_steps=dts)
    b2 = BatchDomain(packed, time_steps=dts)
    va, pa = b2.pack_state()
    assert va.numel() == sum(b.velocity.numel() for b in b2.getBlocks())
    s1 = PISOStepper(b1, time_step=dts[0], advection_tol=1e-6, pressure_tol=1e-6)
    s2 = PISOStepper(b2, time_step=dts[0], advection_tol=1e-6, pressure_tol=1e-6)
    for _ in range(3):
        s1.step()
        s2.step()
    s1.check()
    s2.check()
    for d1, d2 in zip(plain, packed):
        for x1, x2 in zip(d1.getBlocks(), d2.getBlocks()):
            assert np.array_equal(_np(x1.velocity), _np(x2.velocity))
            assert np.array_equal(_np(x1.pressure), _np(x2.pressure))
    host = va.cpu()
    va.zero_()
    assert all(float(b.velocity.abs().max()) == 0.0 for b in b2.getBlocks())
    va.copy_(host.cuda())
    assert np.array_equal(_np(packed[0].getBlocks()[0].velocity), _np(plain[0].getBlocks()[0].velocity))
