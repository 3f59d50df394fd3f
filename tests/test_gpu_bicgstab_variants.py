"""The two-barrier BiCGStab kernels (variants 1 and 2 of pict_krylov_set_bicgstab_variant) against the
default four-barrier kernel (GPU):
the same iteration counts (within one) and solutions (to the solver tolerance) on single and batched
domains, 2D and 3D, plain and transposed, FP32 and FP64, and against the oracle's BiCGStab
(extensions/bicgstab_solver_kernel.cu:240-360)."""
import numpy as np
import pytest
import torch

import piso_oracle as po
from setups import build_oracle, build_product, case

pytestmark = pytest.mark.gpu
DT = 0.05


def _solve(pd, b, tol, transpose, variant, conv=None):
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    lib = _lib.load()
    lib.pict_krylov_set_bicgstab_variant(variant)
    try:
        x = torch.zeros_like(b)
        infos = P.SolveLinear(pd.C, b, x, torch.IntTensor([500]), torch.tensor([tol], dtype=b.dtype),
                              conv if conv is not None else P.ConvergenceCriterion.NORM2_NORMALIZED, True, False, 0,
                              transpose, False, False, BiCGwithPreconditioner=False)
        torch.cuda.synchronize()
    finally:
        lib.pict_krylov_set_bicgstab_variant(0)
    return x, infos


@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("name", ["cavity2d", "twoblock2d_rotated", "periodic2d", "channel3d", "distorted2d"])
def test_two_barrier_bicgstab_matches_four_barrier(name, dtype, transpose):
    from pict_b200 import PISOtorch as P
    pd = build_product(case(name), dtype)
    P.SetupAdvectionMatrix(pd, torch.tensor([DT], dtype=dtype), 0)
    g = torch.Generator().manual_seed(3)
    b = torch.randn(pd.getSpatialDims() * pd.getTotalSize(), generator=g, dtype=torch.float64).to(dtype).cuda()
    tol = 1e-12 if dtype == torch.float64 else 1e-6
    x0, i0 = _solve(pd, b, tol, transpose, 0)
    scale = float(x0.abs().max())
    for v in (1, 2):
        x1, i1 = _solve(pd, b, tol, transpose, v)
        for a, c in zip(i0, i1):
            assert c.converged and c.isFiniteResidual
            assert abs(a.usedIterations - c.usedIterations) <= 1
        bound = 1e-9 if dtype == torch.float64 else 2e-5
        assert float((x1 - x0).abs().max()) <= bound * scale


@pytest.mark.parametrize("name", ["cavity2d", "channel3d"])
def test_two_barrier_bicgstab_against_oracle(name):
    from pict_b200 import PISOtorch as P
    pd = build_product(case(name), torch.float64)
    P.SetupAdvectionMatrix(pd, torch.tensor([DT], dtype=torch.float64), 0)
    od = build_oracle(case(name))
    coef, _ = po.advection_matrix(od, DT)
    A = po.stencil_to_scipy(od, coef)
    n, D = pd.getTotalSize(), pd.getSpatialDims()
    g = torch.Generator().manual_seed(4)
    b = torch.randn(D * n, generator=g, dtype=torch.float64).cuda()
    x, infos = _solve(pd, b, 1e-11, False, 1)
    bn = b.cpu().numpy().reshape(D, n)
    xs = x.cpu().numpy().reshape(D, n)
    for c in range(D):
        xo, io = po.bicgstab(A, bn[c], tol=1e-11, maxit=500)
        assert abs(io.usedIterations - infos[c].usedIterations) <= 1
        assert np.abs(xs[c] - xo).max() <= 1e-8 * np.abs(xo).max()


def test_two_barrier_bicgstab_batched_systems_stop_independently():
    """A batch of cavities of different sizes stepped with either kernel: the same advection iteration
    counts per system (within one) and the same velocities to the solver tolerance."""
    import bench
    from pict_b200 import _lib
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    lib = _lib.load()
    out = []
    for v in (0, 1):
        lib.pict_krylov_set_bicgstab_variant(v)
        try:
            doms = [bench.make_cavity_domain(n, 1e-3, torch.float32) for n in (24, 40, 64, 96)]
            batch = BatchDomain(doms, time_steps=[0.01] * 4)
            st = PISOStepper(batch, time_step=0.01, advection_tol=1e-6, pressure_tol=1e-6)
            for _ in range(3):
                st.step()
            st.check()
            adv, _ = st.infos()
            out.append(([i.usedIterations for i in adv], [d.getBlock(0).velocity.clone() for d in doms]))
        finally:
            lib.pict_krylov_set_bicgstab_variant(0)
    for a, c in zip(out[0][0], out[1][0]):
        assert abs(a - c) <= 1
    for u0, u1 in zip(out[0][1], out[1][1]):
        assert float((u0 - u1).abs().max()) <= 1e-4 * float(u0.abs().max())


def test_advection_increment_guess_same_step_fewer_iterations():
    """Starting the advection solves from the velocity plus the previous step's advection increment gives the
    same fields (to the solver tolerance) in fewer BiCGStab iterations on viscous-dominated cavities."""
    import bench
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    out = []
    for guess in (True, "increment"):
        doms = [bench.make_cavity_domain(n, 1.0 / re, torch.float32) for n, re in ((128, 100.0), (96, 150.0))]
        b = BatchDomain(doms, time_steps=[0.5 / 128, 0.5 / 96])
        st = PISOStepper(b, time_step=0.5 / 128, advection_tol=1e-6, pressure_tol=1e-6, warm_start_advection=guess)
        its = []
        for _ in range(8):
            st.step()
            adv, _ = st.infos()
            its.append(sum(i.usedIterations for i in adv))
        st.check()
        out.append((its, [d.getBlock(0).velocity.clone() for d in doms]))
    assert sum(out[1][0][2:]) < sum(out[0][0][2:]), out[0][0] + out[1][0]
    for u0, u1 in zip(out[0][1], out[1][1]):
        assert float((u0 - u1).abs().max()) <= 1e-4 * float(u0.abs().max())


def test_pressure_increment_warm_start_same_step():
    """The refinement of the second corrector started from the first corrector's pressure plus the previous
    step's corrector increment gives the same fields (to the refinement tolerance) in no more iterations."""
    import bench
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    out = []
    for ws in (True, "increment"):
        doms = [bench.make_cavity_domain(n, 1.0 / re, torch.float32) for n, re in ((128, 150.0), (96, 2000.0))]
        b = BatchDomain(doms, time_steps=[0.5 / 128, 0.5 / 96])
        st = PISOStepper(b, time_step=0.5 / 128, advection_tol=1e-6, pressure_tol=1e-6, pressure_refine=1,
                         refine_tol=5e-10, warm_start_pressure=ws, refine_solver="mg", pressure_first_solve=False)
        its = []
        for _ in range(8):
            st.step()
            its.append(sum(i.usedIterations for i in st.refine_infos()[1][0]))
        st.check()
        out.append((its, [torch.cat([d.getBlock(0).velocity.reshape(-1), d.getBlock(0).pressure.reshape(-1)])
                          for d in doms]))
    assert sum(out[1][0][2:]) < sum(out[0][0][2:]), out[0][0] + out[1][0]
    for a, c in zip(out[0][1], out[1][1]):
        assert float((a - c).abs().max()) <= 1e-4 * float(a.abs().max())
