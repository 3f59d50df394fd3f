"""Pin the oracle's non-orthogonal terms against the reference's own CUDA build (CPU only).

The fixtures tests/golden/ref_nonortho_*.npz were generated on a B200 by
tests/golden/make_ref_nonortho_fixtures.py from the reference's compiled ``PISOtorch`` module: for
skewed and distorted 2D/3D grids (walls, periodic axes, an inflow face, two connected blocks with and
without an axis permutation) the advection matrix and velocity RHS, the pressure matrix and pressure
RHS divergence for the flag sets 25 (the driver's default: center + direct matrix terms, diagonal RHS
terms), 27 (plus direct RHS terms) and 19 (direct RHS instead of diagonal RHS), and 4 FP64 steps of the
non-orthogonal driver branch from rest.
"""
import os
import sys

import numpy as np
import pytest

import piso_oracle as po
from setups import NONORTHO_CASES, NONORTHO_FLAG_SETS, build_oracle, case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from make_ref_nonortho_fixtures import DT, rest_spec  # noqa: E402

# setups whose 4 reference steps need pressure iterations (the source-driven channels converge with
# zero iterations and a pressure of round-off size)
STEP_CASES = ["distorted2d", "skewed_twoblock2d", "skewed_cavity3d", "skewed_channel2d"]


def _load(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip("fixture %s missing" % name)
    return np.load(p)


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("flags", NONORTHO_FLAG_SETS)
@pytest.mark.parametrize("name", NONORTHO_CASES)
def test_oracle_nonortho_operators_match_reference(name, flags):
    fx = _load("ref_nonortho_%s.npz" % name)
    k = "f%d_" % flags
    od = build_oracle(case(name))
    C, A = po.advection_matrix(od, DT, flags)
    v, i, r = po.stencil_to_csr(od, C)
    assert np.array_equal(r, fx[k + "C_row"]) and np.array_equal(i, fx[k + "C_index"])
    assert _rel(v, fx[k + "C_value"]) < 1e-12
    assert _rel(A, fx[k + "A"]) < 1e-12
    assert _rel(po.advection_rhs(od, DT, flags, fx[k + "ures"]).reshape(-1), fx[k + "velocityRHS"]) < 1e-12
    P = po.pressure_matrix(od, A, flags)
    v, i, r = po.stencil_to_csr(od, P)
    assert np.array_equal(r, fx[k + "P_row"]) and np.array_equal(i, fx[k + "P_index"])
    assert _rel(v, fx[k + "P_value"]) < 1e-12
    h = po.pressure_rhs(od, DT, C, A, fx[k + "ustar"])
    assert _rel(h.reshape(-1), fx[k + "pressureRHS"]) < 1e-12
    div = po.pressure_rhs_nonortho(od, flags, po.divergence(od, h), A, fx[k + "pres"])
    assert _rel(div, fx[k + "pressureRHSdiv"]) < 1e-11


@pytest.mark.parametrize("name", STEP_CASES)
def test_oracle_nonortho_steps_match_reference(name):
    fx = _load("ref_nonortho_%s.npz" % name)
    assert fx["steps_infos"][:, 2].all()  # every reference solve converged
    od = build_oracle(rest_spec(name))
    p_its = []
    for _ in range(int(fx["steps_n"])):
        res = po.piso_step(od, float(fx["steps_dt"]), adv_tol=1e-12, p_tol=float(fx["steps_p_tol"]),
                           non_ortho_flags=int(fx["steps_flags"]))
        p_its += [i[2].usedIterations for i in res.infos if i[0] == "p"]
    ref_its = [int(x) for x, kind in zip(fx["steps_infos"][:, 1], fx["steps_info_kind"]) if kind == 1]
    assert p_its == ref_its
    u, ur = od.velocity_global(), fx["steps_velocity"]
    assert _rel(u, ur) < 1e-10
    # pressure relative to its own scale, or to round-off where no pressure iteration was needed
    pr = fx["steps_pressure"]
    scale = max(np.abs(pr).max(), 1e-12 * np.abs(ur).max())
    assert np.abs(od.pressure_global() - pr).max() <= 1e-9 * scale + 1e-15


def test_oracle_nonortho_terms_vanish_on_orthogonal_grids():
    """On orthogonal grids the off-diagonal metric is zero, so every flag set reproduces the orthogonal operators."""
    for name in ["cavity2d_refined", "twoblock2d_rotated", "channel3d"]:
        od = build_oracle(case(name))
        C0, A0 = po.advection_matrix(od, DT)
        for flags in NONORTHO_FLAG_SETS:
            C1, _ = po.advection_matrix(od, DT, flags)
            assert np.abs(C1 - C0).max() == 0.0
            assert np.abs(po.advection_rhs(od, DT, flags) - po.advection_rhs(od, DT)).max() == 0.0
            assert np.abs(po.pressure_matrix(od, A0, flags) - po.pressure_matrix(od, A0)).max() == 0.0
