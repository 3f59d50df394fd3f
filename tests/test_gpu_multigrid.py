"""Multigrid-preconditioned CG (GPU): Galerkin coarse operators against R A R^T assembled with SciPy,
convergence of the batched preconditioned CG, and the mixed-precision step with multigrid correction
solves against the FP64 oracle."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import piso_oracle as po
from setups import build_oracle, build_product, case, lid_cavity

pytestmark = pytest.mark.gpu


def _stencil_matrix(coef, blocks, dims):
    """SciPy matrix of a level stencil (structured neighbours, periodic wrap)."""
    K = 2 * dims + 1
    N = coef.size // K
    coef = coef.reshape(K, N)
    rows, cols, vals = [], [], []
    for row in blocks:
        off, sx, sy, sz, px, py, pz = row[:7]
        n = (sx, sy, sz)
        per = (px, py, pz)
        for l in range(sx * sy * sz):
            q = [l % sx, (l // sx) % sy, l // (sx * sy)]
            i = off + l
            rows.append(i); cols.append(i); vals.append(coef[0, i])
            for f in range(2 * dims):
                a = f >> 1
                qq = list(q)
                qq[a] += 1 if f & 1 else -1
                if qq[a] < 0 or qq[a] >= n[a]:
                    if not per[a]:
                        continue
                    qq[a] %= n[a]
                j = off + qq[0] + sx * (qq[1] + sy * qq[2])
                rows.append(i); cols.append(j); vals.append(coef[f + 1, i])
    return sp.csr_matrix((vals, (rows, cols)), shape=(N, N))


def _aggregation(fine_blocks, coarse_blocks):
    rows, cols = [], []
    for fb, cb in zip(fine_blocks, coarse_blocks):
        off, sx, sy, sz = fb[:4]
        coff, csx, csy = cb[0], cb[1], cb[2]
        hx, hy, hz = cb[8], cb[9], cb[10]
        for l in range(sx * sy * sz):
            x, y, z = l % sx, (l // sx) % sy, l // (sx * sy)
            rows.append(coff + (x >> hx) + csx * ((y >> hy) + csy * (z >> hz)))
            cols.append(off + l)
    nf = sum(b[1] * b[2] * b[3] for b in fine_blocks)
    nc = sum(b[1] * b[2] * b[3] for b in coarse_blocks)
    return sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(nc, nf))


def _prepared_batch(dtype, sides=(13, 20, 9)):
    from pict_b200 import PISOtorch as P
    from pict_b200.batch import BatchDomain
    doms = [build_product(lid_cavity(n, viscosity=1e-3), dtype) for n in sides]
    b = BatchDomain(doms, time_steps=[0.5 / n for n in sides])
    from pict_b200.engine import PISOStepper
    st = PISOStepper(b, time_step=0.01, advection_tol=1e-8, pressure_tol=1e-8)
    st.step()
    torch.cuda.synchronize()
    return b, st


def test_galerkin_matches_scipy():
    from pict_b200.multigrid import hierarchy_for
    b, st = _prepared_batch(torch.float64)
    mg = hierarchy_for(b)
    assert mg.num_levels >= 3
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    mg.setup(b.P.coef, s)
    torch.cuda.synchronize()
    tables = [t[0].cpu().numpy().reshape(-1, 12) for t in mg.levels_py]
    A = _stencil_matrix(b.P.coef.cpu().numpy().reshape(-1), tables[0], 2)
    for l in range(1, mg.num_levels):
        R = _aggregation(tables[l - 1], tables[l])
        Ac_ref = (R @ A @ R.T).toarray()
        Ac = _stencil_matrix(mg.levels_py[l][2].cpu().numpy(), tables[l], 2).toarray()
        assert np.abs(Ac - Ac_ref).max() <= 1e-12 * np.abs(Ac_ref).max()
        A = sp.csr_matrix(Ac_ref)


def test_pcg_mg_reduces_residual_like_cg():
    from pict_b200 import PISOtorch as P
    from pict_b200.multigrid import hierarchy_for
    b, st = _prepared_batch(torch.float32, sides=(64, 48, 100, 37))
    mg = hierarchy_for(b)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    mg.setup(b.P.coef, s)
    g = torch.Generator(device="cpu").manual_seed(4)
    rhs = torch.randn(b.getTotalSize(), generator=g).cuda()
    # mean-free per system
    sc = b._sim_cells.cpu().numpy()
    for k in range(len(sc) - 1):
        rhs[sc[k]:sc[k + 1]] -= rhs[sc[k]:sc[k + 1]].mean()
    x = torch.zeros_like(rhs)
    info = torch.zeros(b.num_sims * 24, dtype=torch.uint8, device="cuda")
    ws = torch.empty(mg.workspace_bytes(b._desc), dtype=torch.uint8, device="cuda")
    mg.solve(b._desc, rhs, x, 12, 1e-30, info, ws, s)
    infos = P.decode_infos(info)
    # true residual of the result, in FP64
    from pict_b200 import _lib
    r_true = torch.zeros_like(rhs)
    x64 = torch.zeros(rhs.numel(), dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().pict_refine_residual(ctypes.byref(b._desc), b.P.coef.data_ptr(), rhs.data_ptr(), x.data_ptr(),
                                                ctypes.c_void_p(x64.data_ptr()), r_true.data_ptr(), 0, None, s), "residual")
    # plain CG with the same budget of 12 iterations, for comparison
    x_cg = torch.zeros_like(rhs)
    prm = P._solve_params(1, 12, 1e-30, 1, False, False, x_zero=True)
    cg_infos = P.decode_infos(P.solve_stencil(b, b.P.coef, rhs, x_cg, prm))
    torch.cuda.synchronize()
    for k in range(len(sc) - 1):
        n = sc[k + 1] - sc[k]
        r0 = float(rhs[sc[k]:sc[k + 1]].double().norm()) / np.sqrt(n)
        assert infos[k].finalResidual < 1e-4 * r0, (k, infos[k], r0)
        rt = float(r_true[sc[k]:sc[k + 1]].double().norm()) / np.sqrt(n)
        assert rt < 1e-3 * r0, (k, rt, r0)
        assert infos[k].finalResidual < 0.01 * cg_infos[k].finalResidual


def test_refined_step_with_multigrid_within_1e5_of_fp64_oracle():
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    specs = [lid_cavity(32, viscosity=1.0 / 1500.0), lid_cavity(33, viscosity=1.0 / 800.0)]
    doms = [build_product(s_, torch.float32) for s_ in specs]
    b = BatchDomain(doms, time_steps=[0.5 / 32, 0.5 / 33])
    st = PISOStepper(b, time_step=0.01, advection_tol=1e-6, pressure_tol=1e-6, pressure_refine=1, refine_tol=1e-9,
                     warm_start_pressure=True, refine_solver="mg", mg_iterations=10)
    assert st._mg is not None
    for _ in range(10):
        st.step()
        st.check()
    for s_, n, d in zip(specs, (32, 33), doms):
        od = build_oracle(s_)
        for _ in range(10):
            po.piso_step(od, 0.5 / n, adv_tol=1e-12, p_tol=1e-12)
        u = d.getBlock(0).velocity.double().cpu().numpy().reshape(2, -1)
        p = d.getBlock(0).pressure.double().cpu().numpy().reshape(-1)
        ur, pr = od.velocity_global(), od.pressure_global()
        assert np.abs(u - ur).max() / np.abs(ur).max() < 1e-5
        assert np.abs(p - pr).max() / np.abs(pr).max() < 1e-5


def test_semicoarsening_on_stretched_grid():
    """A strongly stretched 2D block: the stretched axis is halved first, the Galerkin operators still
    equal R A R^T, and the preconditioned CG converges."""
    from pict_b200 import PISOtorch as P
    from pict_b200.multigrid import hierarchy_for
    from pict_b200.engine import PISOStepper
    from setups import tensor_grid, stretched
    xs = np.linspace(0, 4.0, 65)
    ys = stretched(48, length=1.0, beta=3.0)
    spec = dict(dims=2, viscosity=1e-2, blocks=[dict(coords=tensor_grid(xs, ys))],
                ops=[("periodic", 0, "x"), ("close", 0, "-y"), ("close", 0, "+y")])
    pd = build_product(spec, torch.float64)
    st = PISOStepper(pd, time_step=0.01, advection_tol=1e-10, pressure_tol=1e-10)
    st.step()
    mg = hierarchy_for(pd)
    assert mg.shifts[1][0, 1] == 1 and mg.shifts[1][0, 0] == 0   # y (stretched) only
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    mg.setup(pd.P.coef, s)
    torch.cuda.synchronize()
    tables = [t[0].cpu().numpy().reshape(-1, 12) for t in mg.levels_py]
    A = _stencil_matrix(pd.P.coef.cpu().numpy().reshape(-1), tables[0], 2)
    for l in range(1, mg.num_levels):
        R = _aggregation(tables[l - 1], tables[l])
        Ac_ref = (R @ A @ R.T).toarray()
        Ac = _stencil_matrix(mg.levels_py[l][2].cpu().numpy(), tables[l], 2).toarray()
        assert np.abs(Ac - Ac_ref).max() <= 1e-12 * np.abs(Ac_ref).max()
        A = sp.csr_matrix(Ac_ref)
    g = torch.Generator(device="cpu").manual_seed(8)
    rhs = torch.randn(pd.getTotalSize(), generator=g, dtype=torch.float64).cuda()
    rhs -= rhs.mean()
    x = torch.zeros_like(rhs)
    info = torch.zeros(24, dtype=torch.uint8, device="cuda")
    ws = torch.empty(mg.workspace_bytes(pd._desc), dtype=torch.uint8, device="cuda")
    mg.solve(pd._desc, rhs, x, 16, 1e-30, info, ws, s)
    inf = P.decode_infos(info)[0]
    r0 = float(rhs.norm()) / np.sqrt(rhs.numel())
    # point smoothing with a per-block coarsening choice is only partly robust to the wall stretching
    assert inf.isFiniteResidual and inf.finalResidual < 0.1 * r0, (inf, r0)


def _mg_solve(b, mg, rhs, iterations=12):
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    x = torch.zeros_like(rhs)
    info = torch.zeros(b.num_sims * 24, dtype=torch.uint8, device="cuda")
    ws = torch.empty(mg.workspace_bytes(b._desc), dtype=torch.uint8, device="cuda")
    mg.solve(b._desc, rhs, x, iterations, 1e-30, info, ws, s)
    torch.cuda.synchronize()
    return x, info


@pytest.mark.parametrize("dtype,tile", [(torch.float32, 1024), (torch.float32, 2048), (torch.float64, 1024)])
@pytest.mark.parametrize("layout", ["cavities", "periodic"])
def test_bulk_staged_spmv_equals_gather_kernel(dtype, tile, layout):
    """The PCG SpMV with its operands staged by bulk copies (persistent grid, two stage buffers) gives the
    gather kernel's result: same cells, arithmetic and per-warp partials, on uneven batched cavities (rows
    of 37..100 cells, tiles starting mid-row) and on periodic boxes (wraps in x inside the stage, in y from
    global memory)."""
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    from pict_b200.batch import BatchDomain
    from pict_b200.multigrid import hierarchy_for
    from setups import forcing_box
    lib = _lib.load()
    if layout == "cavities":
        doms = [build_product(lid_cavity(n, viscosity=1e-3), dtype) for n in (64, 48, 100, 37)]
    else:
        doms = [build_product(forcing_box(n), dtype) for n in (48, 96)]
    b = BatchDomain(doms, time_steps=[0.01] * len(doms))
    b.set_tile_cells(tile)
    from pict_b200.engine import PISOStepper
    st = PISOStepper(b, time_step=0.01, advection_tol=1e-8, pressure_tol=1e-8)
    st.step()
    torch.cuda.synchronize()
    mg = hierarchy_for(b)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    mg.setup(b.P.coef, s)
    g = torch.Generator(device="cpu").manual_seed(5)
    rhs = torch.randn(b.getTotalSize(), generator=g, dtype=dtype).cuda()
    sc = b._sim_cells.cpu().numpy()
    for k in range(len(sc) - 1):
        rhs[sc[k]:sc[k + 1]] -= rhs[sc[k]:sc[k + 1]].mean()
    try:
        lib.pict_mg_set_bulk_staging(0)
        x_gather, info_g = _mg_solve(b, mg, rhs)
        lib.pict_mg_set_bulk_staging(1)
        x_bulk, info_b = _mg_solve(b, mg, rhs)
    finally:
        lib.pict_mg_set_bulk_staging(1)
    ig, ib = P.decode_infos(info_g), P.decode_infos(info_b)
    assert all(i.status == 0 for i in ib)
    diff = float((x_bulk - x_gather).abs().max() / x_gather.abs().max())
    print("%s %s tile %d: bulk vs gather max rel diff %.3e, bitwise %s" % (layout, dtype, tile, diff,
                                                                        bool(torch.equal(x_bulk, x_gather))))
    assert diff < (1e-5 if dtype == torch.float32 else 1e-12)
    for a, c in zip(ig, ib):
        assert abs(a.finalResidual - c.finalResidual) <= 1e-3 * abs(a.finalResidual) + 1e-30


@pytest.mark.parametrize("sides", [(64, 48, 100, 37), (256, 181, 90)])
def test_two_sweep_smoothing_needs_fewer_iterations(sides):
    """Two damped-Jacobi sweeps per smoothing step (the default where the tiles' stages allow it) keep the
    preconditioner symmetric and reach a 1e-6 residual reduction in fewer PCG iterations than one sweep."""
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    from pict_b200.multigrid import hierarchy_for
    lib = _lib.load()
    b, st = _prepared_batch(torch.float32, sides=sides)
    mg = hierarchy_for(b)
    assert mg.levels[0].sweeps == 2
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    mg.setup(b.P.coef, s)
    g = torch.Generator(device="cpu").manual_seed(5)
    rhs = torch.randn(b.getTotalSize(), generator=g).cuda()
    sc = b._sim_cells.cpu().numpy()
    for k in range(len(sc) - 1):
        rhs[sc[k]:sc[k + 1]] -= rhs[sc[k]:sc[k + 1]].mean()
    r0 = [float(rhs[sc[k]:sc[k + 1]].double().norm()) / np.sqrt(sc[k + 1] - sc[k]) for k in range(len(sc) - 1)]
    tol = 1e-6 * min(r0)
    used = {}
    try:
        for nu in (1, 2):
            lib.pict_mg_set_smoothing_sweeps(nu)
            x = torch.zeros_like(rhs)
            info = torch.zeros(b.num_sims * 24, dtype=torch.uint8, device="cuda")
            ws = torch.empty(mg.workspace_bytes(b._desc), dtype=torch.uint8, device="cuda")
            mg.solve(b._desc, rhs, x, 40, tol, info, ws, s)
            infos = P.decode_infos(info)
            torch.cuda.synchronize()
            assert all(i.converged and i.isFiniteResidual for i in infos), infos
            used[nu] = [i.usedIterations for i in infos]
    finally:
        lib.pict_mg_set_smoothing_sweeps(2)
    assert all(a <= c for a, c in zip(used[2], used[1])), used
    assert max(used[2]) < max(used[1]), used


def test_graph_loop_equals_fixed_iterations():
    """A captured mixed-precision step whose multigrid PCG loop is a conditional WHILE node (stopping once every
    system has converged) gives the same fields and reports as the captured fixed iteration sequence."""
    import bench
    from pict_b200 import _lib
    from pict_b200.batch import BatchDomain
    from pict_b200.engine import PISOStepper
    lib = _lib.load()
    out = []
    try:
        for loop in (0, 1):
            lib.pict_mg_set_graph_loop(loop)
            doms = [bench.make_cavity_domain(n, 1e-3, torch.float32) for n in (96, 64, 40, 33)]
            b = BatchDomain(doms, time_steps=[0.5 / n for n in (96, 64, 40, 33)])
            st = PISOStepper(b, time_step=0.01, advection_tol=1e-6, pressure_tol=1e-6, pressure_refine=1,
                             refine_tol=5e-10, warm_start_pressure=True, refine_solver="mg",
                             pressure_first_solve=False)
            assert st._mg is not None
            for _ in range(2):
                st.step()
            st.capture(steps=3)
            for _ in range(2):
                st.replay()
            torch.cuda.synchronize()
            st.check()
            rep = [[(i.usedIterations, i.finalResidual) for i in r] for row in st.refine_infos() for r in row]
            out.append(([torch.cat([d.getBlock(0).velocity.reshape(-1), d.getBlock(0).pressure.reshape(-1)])
                         for d in doms], rep))
    finally:
        lib.pict_mg_set_graph_loop(1)
    for a, c in zip(out[0][0], out[1][0]):
        assert torch.equal(a, c)
    assert out[0][1] == out[1][1]
