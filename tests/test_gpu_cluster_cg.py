"""Cluster CG (GPU): the single-reduction CG with one thread-block cluster per system (inner products
through distributed shared memory, one cluster barrier per iteration) against the same recurrence on
the persistent grid (grid-wide barriers), on batched uneven cavities, the multi-block cylinder street,
periodic boxes and a 3D channel, FP32 and FP64, with mean removal and the blocks' pressure written.
Both stop at the same RMS residual; their inner products are summed in different orders, so iteration
counts may differ by one and solutions by the tolerance."""
import ctypes

import numpy as np
import pytest
import torch

from setups import build_product, case, forcing_box, lid_cavity

pytestmark = pytest.mark.gpu


def _domain(layout, dtype):
    from pict_b200.batch import BatchDomain
    if layout == "cavities":
        doms = [build_product(lid_cavity(n, viscosity=1e-3), dtype) for n in (96, 64, 48, 33, 20)]
        return BatchDomain(doms, time_steps=[0.01] * len(doms))
    if layout == "street":
        from pict_b200.cylinder_street import build_street, street_prep_fn, street_spec
        from pict_b200.PISOtorch_simulation import Simulation
        dom, info = build_street(street_spec(16, 16, 0.5), dtype=dtype)
        Simulation(domain=dom, time_step=0.005, prep_fn=street_prep_fn(info), advection_tol=1e-6, pressure_tol=1e-6,
                   non_orthogonal=False).make_divergence_free()
        return dom
    if layout == "periodic":
        doms = [build_product(forcing_box(n), dtype) for n in (64, 40)]
        return BatchDomain(doms, time_steps=[0.01] * len(doms))
    return build_product(case("channel3d"), dtype)


def _solve(dom, mode, rhs, tol, sub_mean):
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    lib = _lib.load()
    x = torch.zeros_like(rhs)
    prm = P._solve_params(1, 5000, tol, 1, False, False, x_zero=True, variant=1, subtract_mean=sub_mean,
                          write_block_pressure=sub_mean)
    try:
        lib.pict_krylov_set_cluster_mode(mode)
        infos = P.decode_infos(P.solve_stencil(dom, dom.P.coef, rhs, x, prm))
    finally:
        lib.pict_krylov_set_cluster_mode(1)
    torch.cuda.synchronize()
    bp = torch.cat([b.pressure.reshape(-1) for b in dom.getBlocks()]).clone()
    return x, infos, bp


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("layout", ["cavities", "street", "periodic", "channel3d"])
def test_cluster_cg_matches_grid_cg(layout, dtype):
    from pict_b200.engine import PISOStepper
    dom = _domain(layout, dtype)
    st = PISOStepper(dom, time_step=0.005 if layout == "street" else 0.01, advection_tol=1e-6, pressure_tol=1e-6)
    st.step()  # leaves the last corrector's pressure system in P and pressureRHSdiv
    torch.cuda.synchronize()
    rhs = dom.pressureRHSdiv.clone()
    # an RMS tolerance relative to the right-hand side (the street's unprojected start has a large one)
    rms = float(rhs.double().norm()) / np.sqrt(rhs.numel())
    tol = (1e-5 if dtype == torch.float32 else 1e-11) * rms
    xg, ig, bg = _solve(dom, 0, rhs, tol, True)
    xc, ic, bc = _solve(dom, 2, rhs, tol, True)
    assert all(i.converged for i in ig) and all(i.converged for i in ic), (ig, ic)
    its_g = [i.usedIterations for i in ig]
    its_c = [i.usedIterations for i in ic]
    assert all(abs(a - b) <= 1 for a, b in zip(its_g, its_c)), (its_g, its_c)
    scale = float(xg.abs().max())
    err = float((xc - xg).abs().max()) / scale
    print("%s %s: grid iterations %s, cluster %s, max rel diff %.2e" % (layout, dtype, its_g, its_c, err))
    assert err < (1e-3 if dtype == torch.float32 else 1e-8)
    assert float((bc - xc).abs().max()) == 0.0  # blocks' pressure = the mean-free solution
    # mean-free per system
    sc = dom._sim_cells.cpu().numpy()
    for k in range(len(sc) - 1):
        assert abs(float(xc[sc[k]:sc[k + 1]].double().mean())) < 1e-6 * scale
