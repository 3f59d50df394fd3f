"""Smagorinsky sub-grid-scale viscosity (SGSviscosityIncompressibleSmagorinsky) of the CUDA path against the
reference's own CUDA build (GPU); fixtures from tests/golden/make_ref_sgs_fixtures.py (FP64)."""
import os
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_ref_sgs_fixtures as G  # noqa: E402


@pytest.mark.parametrize("name", G.SGS_CASES)
def test_sgs_viscosity_matches_reference(name):
    from pict_b200 import PISOtorch as P
    p = os.path.join(GOLDEN, "ref_sgs_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    fx = np.load(p)
    out = G.sgs_fixture(P, name)
    assert np.array_equal(out["shapes"], fx["shapes"])
    err = np.abs(out["nu_sgs"] - fx["nu_sgs"]).max() / np.abs(fx["nu_sgs"]).max()
    assert err < 1e-12, err


def test_sgs_viscosity_feeds_the_block_viscosity():
    """The returned tensors have the block viscosity shape and can be set as block viscosities."""
    from pict_b200 import PISOtorch as P
    from setups import build_product, case
    pd = build_product(case("distorted2d"), torch.float32)
    nus = P.SGSviscosityIncompressibleSmagorinsky(pd, torch.tensor([0.03], dtype=torch.float32))
    for b, nu in zip(pd.getBlocks(), nus):
        b.setViscosity(nu + 1e-3)
    pd.UpdateDomainData()
    P.SetupAdvectionMatrix(pd, torch.tensor([0.05], dtype=torch.float32), 0)
    assert torch.isfinite(pd.A).all()
