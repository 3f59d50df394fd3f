"""Maximum velocity and the adaptive time step (GPU), against the reference's CUDA build.

Domain.getMaxVelocity / getMaxVelocityMagnitude (extensions/domain_structs.cpp:1564-1600, 2387-2410) with
and without boundaries, physical and computational, on every test setup and the reduced cylinder street
(with a varying outflow face); get_max_time_step (PISOtorch_simulation.py:55-64); and
Simulation(substeps="ADAPTIVE") (PISOtorch_simulation.py:1329-1372) on a cavity whose lid moves at 4,
whose substep counts and fields equal the reference's.  Fixtures: tests/golden/make_ref_maxvel_fixtures.py.
"""
import os

import numpy as np
import pytest
import torch

from setups import ALL_CASES, build_product, case, lid_cavity

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
COMBOS = [(wb, comp) for wb in (False, True) for comp in (False, True)]


def _fx():
    d = np.load(os.path.join(HERE, "golden", "ref_maxvel.npz"))
    return {k: d[k] for k in d.files}


def _domain(name):
    if name == "street16":
        from pict_b200.cylinder_street import build_street, street_spec
        dom, _ = build_street(street_spec(16, 16, 0.5), dtype=torch.float64)
        return dom
    return build_product(case(name), torch.float64)


@pytest.mark.parametrize("name", list(ALL_CASES) + ["street16"])
def test_max_velocity_matches_reference(name):
    fx = _fx()
    dom = _domain(name)
    for bi, b in enumerate(dom.getBlocks()):
        b.setVelocity(torch.tensor(fx["%s_b%d_velocity" % (name, bi)], device="cuda").contiguous())
    if name == "street16":
        bnd = dom.getBlock(dom.getNumBlocks() - 1).getBoundary("+x")
        bnd.setVelocity(torch.tensor(fx["%s_outflow" % name], device="cuda").contiguous())
    ref = fx["%s_values" % name]
    k = 0
    for wb, comp in COMBOS:
        for fn in (dom.getMaxVelocity, dom.getMaxVelocityMagnitude):
            if not np.isnan(ref[k]):
                v = float(fn(wb, comp).cpu())
                assert abs(v - ref[k]) <= 1e-13 * abs(ref[k]), (name, wb, comp, fn.__name__, v, ref[k])
            k += 1


def test_max_time_step():
    from pict_b200.PISOtorch_simulation import get_max_time_step
    dom = build_product(lid_cavity(16, viscosity=1e-2, lid=4.0), torch.float64)
    vmax = float(dom.getMaxVelocity(True, True).cpu())  # the lid, in cells per unit time
    ts, ss = get_max_time_step(dom, 1.0, CFL_cond=0.8)
    assert ss == int(np.ceil(1.0 / (0.8 / vmax))) and abs(ts * ss - 1.0) < 1e-14
    ts, ss = get_max_time_step(dom, 0.1 * 0.8 / vmax, CFL_cond=0.8)
    assert ss == 1


def test_adaptive_step_matches_reference():
    from pict_b200.PISOtorch_simulation import Simulation
    fx = _fx()
    dom = build_product(lid_cavity(24, viscosity=1e-2, lid=4.0), torch.float64)
    sim = Simulation(domain=dom, time_step=float(fx["adaptive_target"]), substeps="ADAPTIVE",
                     adaptive_CFL=float(fx["adaptive_cfl"]), advection_tol=1e-12, pressure_tol=1e-12,
                     non_orthogonal=False)
    counts = []
    for _ in range(len(fx["adaptive_counts"])):
        before = sim.total_step
        assert sim.run(1)
        counts.append(sim.total_step - before)
    assert counts == list(fx["adaptive_counts"]), (counts, fx["adaptive_counts"])
    assert abs(sim.total_time - float(fx["adaptive_ts"].sum())) < 1e-12
    u = np.concatenate([b.velocity.double().cpu().numpy().reshape(2, -1) for b in dom.getBlocks()], axis=1)
    p = np.concatenate([b.pressure.double().cpu().numpy().reshape(-1) for b in dom.getBlocks()])
    assert np.abs(u - fx["adaptive_velocity"]).max() / np.abs(fx["adaptive_velocity"]).max() < 1e-9
    assert np.abs(p - fx["adaptive_pressure"]).max() / np.abs(fx["adaptive_pressure"]).max() < 1e-8
