"""The 3D periodic channel (Re_tau 180, tanh-stretched walls) in the timed mixed precision (GPU).

At half resolution (96 x 48 x 48, 221k cells, the largest the FP64 oracle steps in seconds): per-field
error after 5 steps against the oracle (1e-10 solves), and every step's FP64 pressure refinement down to
the configuration's 1e-10 RMS divergence.  At full size (192 x 96 x 96, 1.77M cells): the configuration's
500 steps with the refinement reaching 1e-10 in every corrector of every step and the flow staying finite
and bounded.
"""
import numpy as np
import pytest
import torch

import bench
import piso_oracle as po

pytestmark = pytest.mark.gpu

MIXED = dict(pressure_refine=1, refine_tol=1e-10, warm_start_pressure=True, pressure_first_solve=False,
             refine_solver="auto")


def _refine_max(st):
    return max(max(float(i.finalResidual) for i in r) for row in st.refine_infos() for r in row)


def test_channel_half_resolution_mixed_vs_fp64_oracle():
    nx, ny, nz, steps = 96, 48, 48, 5
    dom = bench.make_channel_domain(nx, ny, nz, torch.float32)
    dt = bench.channel_dt(nx)
    from pict_b200.engine import PISOStepper
    st = PISOStepper(dom, time_step=dt, advection_tol=1e-6, pressure_tol=1e-6, **MIXED)
    res = []
    for _ in range(steps):
        st.step()
        st.check()
        res.append(_refine_max(st))
    _, d = bench._oracle_channel(nx, ny, nz)
    for _ in range(steps):
        po.piso_step(d, dt, adv_tol=1e-10, p_tol=1e-10)
    u = dom.getBlock(0).velocity.double().cpu().numpy().reshape(3, -1)
    p = dom.getBlock(0).pressure.double().cpu().numpy().reshape(-1)
    ur, pr = d.velocity_global(), d.pressure_global()
    eu = [float(np.abs(u[c] - ur[c]).max() / np.abs(ur).max()) for c in range(3)]
    ep = float(np.abs(p - pr).max() / np.abs(pr).max())
    print("channel %dx%dx%d, %d steps, mixed vs FP64 oracle: velocity components %s, pressure %.2e; refinement "
          "residual per step %s" % (nx, ny, nz, steps, ["%.2e" % e for e in eu], ep, ["%.1e" % r for r in res]))
    assert max(res) <= 1e-10
    assert max(eu) < 1e-5 and ep < 1e-4


def test_channel_full_size_500_steps():
    from pict_b200.engine import PISOStepper
    dom = bench.make_channel_domain(192, 96, 96, torch.float32)
    st = PISOStepper(dom, time_step=bench.channel_dt(192), advection_tol=1e-6, pressure_tol=1e-6, **MIXED)
    u0 = float(dom.getBlock(0).velocity.abs().max())
    worst = 0.0
    for _ in range(500):
        st.step()
        st.check()
        worst = max(worst, _refine_max(st))
    umax = float(dom.getBlock(0).velocity.abs().max())
    print("channel 192x96x96, 500 steps: largest refinement residual %.2e, max |u| %.3f (start %.3f)" % (worst, umax, u0))
    assert worst <= 1e-10
    assert np.isfinite(umax) and umax < 1.5 * u0
