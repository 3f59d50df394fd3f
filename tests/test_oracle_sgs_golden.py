"""Pin the oracle's Smagorinsky viscosity against the reference's own CUDA build (CPU only); fixtures from
tests/golden/make_ref_sgs_fixtures.py."""
import os
import sys

import numpy as np
import pytest

import piso_oracle as po
from setups import build_oracle, case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from make_ref_sgs_fixtures import COEFFICIENT, SGS_CASES  # noqa: E402


@pytest.mark.parametrize("name", SGS_CASES)
def test_oracle_sgs_matches_reference(name):
    p = os.path.join(GOLDEN, "ref_sgs_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    fx = np.load(p)
    nu = po.sgs_smagorinsky(build_oracle(case(name)), COEFFICIENT)
    err = np.abs(nu - fx["nu_sgs"]).max() / np.abs(fx["nu_sgs"]).max()
    assert err < 1e-12, err
