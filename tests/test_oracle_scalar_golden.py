"""Pin the oracle's passive scalar operators against the reference's own CUDA build (CPU only).

Fixtures: tests/golden/ref_scalar_*.npz from tests/golden/make_ref_scalar_fixtures.py: the scalar
advection matrix of every channel and the scalar RHS for nonOrthoFlags 0, 25 and 27, and one scalar
advection sub-step of the driver, on 1-2 channel setups with Dirichlet and Neumann faces.
"""
import os
import sys

import numpy as np
import pytest

import piso_oracle as po
from setups import SCALAR_CASES, build_oracle, scalar_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from make_ref_scalar_fixtures import DT, FLAG_SETS  # noqa: E402


def _load(name):
    p = os.path.join(GOLDEN, "ref_scalar_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    return np.load(p)


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", SCALAR_CASES)
def test_oracle_scalar_operators_match_reference(name):
    fx = _load(name)
    od = build_oracle(scalar_case(name))
    C, N = od.scalar_channels, od.N
    for flags in FLAG_SETS:
        k = "f%d_" % flags
        for ch in range(C):
            coef, A = po.scalar_matrix(od, DT, ch, flags)
            v, i, r = po.stencil_to_csr(od, coef)
            assert np.array_equal(i, fx[k + "C_index"]) and np.array_equal(r, fx[k + "C_row"])
            assert _rel(v, fx[k + "C%d_value" % ch]) < 1e-12, (flags, ch)
            assert _rel(A, fx[k + "A%d" % ch]) < 1e-12
        rhs = po.scalar_rhs(od, DT, flags, fx[k + "sres"].reshape(C, N))
        assert _rel(rhs.reshape(-1), fx[k + "scalarRHS"]) < 1e-12, flags


@pytest.mark.parametrize("name", SCALAR_CASES)
def test_oracle_scalar_substep_matches_reference(name):
    """One scalar advection sub-step from the setup's state: every channel solved exactly."""
    fx = _load(name)
    od = build_oracle(scalar_case(name))
    C, N = od.scalar_channels, od.N
    rhs = po.scalar_rhs(od, DT)
    out = np.zeros((C, N))
    for ch in range(C):
        coef, _ = po.scalar_matrix(od, DT, ch)
        out[ch], _ = po.solve(po.stencil_to_scipy(od, coef), rhs[ch], True, 1e-12, method="direct")
    assert _rel(out, fx["step_scalar"]) < 1e-9
