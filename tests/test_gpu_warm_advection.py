"""Advection solves started from the current velocity (PISOStepper(warm_start_advection=True), the reference
driver's advect_use_prev_result) reach the same step as solves from zero, to the solver tolerance."""
import pytest
import torch

from setups import build_product, case, lid_cavity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cavity2d_refined", "twoblock2d_rotated", "ring4_2d", "channel3d"])
def test_warm_advection_same_step(name):
    from pict_b200.engine import PISOStepper
    fields = []
    for warm in (False, True):
        dom = build_product(case(name), torch.float64)
        st = PISOStepper(dom, time_step=0.02, advection_tol=1e-12, pressure_tol=1e-12, warm_start_advection=warm)
        for _ in range(3):
            st.step()
        torch.cuda.synchronize()
        fields.append([(b.velocity.clone(), b.pressure.clone()) for b in dom.getBlocks()])
    for (u0, p0), (u1, p1) in zip(*fields):
        assert (u0 - u1).abs().max().item() <= 1e-9 * max(u0.abs().max().item(), 1.0)
        assert (p0 - p1).abs().max().item() <= 1e-8 * max(p0.abs().max().item(), 1.0)


def test_warm_advection_fewer_iterations():
    """On a developed cavity flow the warm-started BiCGStab needs fewer iterations than from zero."""
    from pict_b200.engine import PISOStepper
    import numpy as np
    from pict_b200 import PISOtorch as P
    its = []
    for warm in (False, True):
        dom = build_product(lid_cavity(48, viscosity=1e-3), torch.float32)
        st = PISOStepper(dom, time_step=0.01, advection_tol=1e-6, pressure_tol=1e-6, warm_start_advection=warm)
        for _ in range(20):
            st.step()
        torch.cuda.synchronize()
        its.append(max(i.usedIterations for i in P.decode_infos(st.info_adv)))
    assert its[1] <= its[0], its
