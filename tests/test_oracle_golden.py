"""Pin the FP64 oracle against golden fixtures produced by the reference's own CUDA build.

The fixtures in tests/golden/ were generated on a B200 by tests/golden/make_ref_fixtures.py, which
builds every setup of tests/setups.py through the reference's compiled ``PISOtorch`` module and
records its operator outputs (advection matrix and RHS, pressure matrix / RHS / divergence, FD
velocity correction, in FP64), four full PISO steps with 1e-13 solves, and 100 steps of the 64x64
lid-driven cavity.  CPU only.
"""
import os

import numpy as np
import pytest

import piso_oracle as po
from setups import ALL_CASES, build_oracle, case, lid_cavity

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DT = 0.05


def _load(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip("fixture %s missing" % name)
    return np.load(p)


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", ALL_CASES)
def test_oracle_operators_match_reference(name):
    fx = _load("ref_ops_%s.npz" % name)
    od = build_oracle(case(name))
    D = od.dims
    C, A = po.advection_matrix(od, DT)
    v, i, r = po.stencil_to_csr(od, C)
    assert np.array_equal(r, fx["C_row"]) and np.array_equal(i, fx["C_index"])
    assert _rel(v, fx["C_value"]) < 1e-12
    assert _rel(A, fx["A"]) < 1e-12
    assert _rel(po.advection_rhs(od, DT).reshape(-1), fx["velocityRHS"]) < 1e-12
    ustar = fx["ustar"]
    P = po.pressure_matrix(od, A)
    v, i, r = po.stencil_to_csr(od, P)
    assert np.array_equal(r, fx["P_row"]) and np.array_equal(i, fx["P_index"])
    assert _rel(v, fx["P_value"]) < 1e-12
    h = po.pressure_rhs(od, DT, C, A, ustar)
    assert _rel(h.reshape(-1), fx["pressureRHS"]) < 1e-12
    assert _rel(po.divergence(od, h), fx["pressureRHSdiv"]) < 1e-11
    u = po.correct_velocity(od, fx["corr_p"], A, fx["corr_h"])
    assert _rel(u.reshape(-1), fx["corr_velocityResult"]) < 1e-12


@pytest.mark.parametrize("name", ALL_CASES)
def test_oracle_steps_match_reference(name):
    fx = _load("ref_ops_%s.npz" % name)
    od = build_oracle(case(name))
    for _ in range(int(fx["steps_n"])):
        po.piso_step(od, float(fx["steps_dt"]), adv_tol=1e-13, p_tol=1e-13)
    assert _rel(od.velocity_global(), fx["steps_velocity"]) < 1e-8
    assert _rel(od.pressure_global(), fx["steps_pressure"]) < 1e-7


def test_oracle_lid_cavity_100_steps_fp64():
    fx = _load("ref_lid64_f64.npz")
    od = build_oracle(lid_cavity(int(fx["n"]), viscosity=float(fx["viscosity"])))
    for _ in range(int(fx["steps"])):
        po.piso_step(od, float(fx["dt"]), adv_tol=float(fx["tol"]), p_tol=float(fx["tol"]))
    # both sides stop their solves at 1e-10 RMS residual; same algorithm, different summation order
    assert _rel(od.velocity_global(), fx["velocity"]) < 1e-6
    assert _rel(od.pressure_global(), fx["pressure"]) < 1e-5
