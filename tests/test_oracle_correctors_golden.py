"""Pin the oracle's velocity correctors (versions 1, 4, 5, 6) against the reference's own CUDA build (CPU only).

Fixtures: tests/golden/ref_corrector_*.npz from tests/golden/make_ref_corrector_fixtures.py (seeded block
pressures, A and H/A; the reference's CorrectVelocity output for each version).
"""
import os
import sys

import numpy as np
import pytest

import piso_oracle as po
from setups import build_oracle, case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from make_ref_corrector_fixtures import CORRECTOR_CASES, DT  # noqa: E402


@pytest.mark.parametrize("name", CORRECTOR_CASES)
def test_oracle_correctors_match_reference(name):
    p = os.path.join(GOLDEN, "ref_corrector_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    fx = np.load(p)
    od = build_oracle(case(name))
    D, N = od.dims, od.N
    pb, A, h = fx["p"], fx["A"], fx["h"].reshape(D, N)
    cands = {"u_v1": po.correct_velocity(od, pb, A, h),
             "u_v4": po.correct_velocity_v4(od, pb, A, h, DT),
             "u_v5": po.correct_velocity_fvm(od, pb, A, h, DT, 5),
             "u_v5_tsn": po.correct_velocity_fvm(od, pb, A, h, DT, 5, True),
             "u_v6": po.correct_velocity_fvm(od, pb, A, h, DT, 6)}
    for k in fx.files:
        if k.startswith("u_"):
            ref = fx[k].reshape(D, N)
            err = np.abs(cands[k] - ref).max() / max(np.abs(ref).max(), 1e-30)
            assert err < 1e-12, (k, err)
