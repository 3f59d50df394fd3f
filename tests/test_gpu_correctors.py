"""Velocity correctors (CorrectVelocity versions 1, 4, 5, 6) of the CUDA path against the reference's own CUDA
build (GPU).

Fixtures: tests/golden/ref_corrector_*.npz, generated on a B200 by tests/golden/make_ref_corrector_fixtures.py
from the reference's compiled module (seeded block pressures, A and H/A on 13 setups: stretched, distorted
and skewed grids, periodic axes, inflow faces, two blocks with straight and rotated connections, 2D and
3D).  The same function runs here with this library's module; FP64 results must agree to round-off.
"""
import os
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_ref_corrector_fixtures as G  # noqa: E402


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", G.CORRECTOR_CASES)
def test_correctors_match_reference(name):
    from pict_b200 import PISOtorch as P
    p = os.path.join(GOLDEN, "ref_corrector_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    fx = np.load(p)
    out = G.corrector_fixture(P, name)
    assert int(out["fvm_ready"]) == int(fx["fvm_ready"])
    keys = [k for k in fx.files if k.startswith("u_")]
    assert len(keys) >= 2
    for k in keys:
        assert _rel(out[k], fx[k]) < 1e-12, (k, _rel(out[k], fx[k]))


def test_fvm_corrector_equals_fd_on_orthogonal_uniform_grids():
    """On a uniform orthogonal grid the finite-volume gradient (version 5) is the finite-difference one
    away from prescribed faces, where the half-cell extrapolation differs."""
    from pict_b200 import PISOtorch as P
    from setups import build_product, case
    pd = build_product(case("fullperiodic2d"), torch.float64)
    g = torch.Generator(device="cpu").manual_seed(2)
    for b in pd.getBlocks():
        b.setPressure(torch.randn(b.pressure.shape, generator=g, dtype=torch.float64).cuda())
    N, D = pd.getTotalSize(), pd.getSpatialDims()
    pd.setA(1 + torch.rand(N, generator=g, dtype=torch.float64).cuda())
    pd.setPressureRHS(torch.randn(D * N, generator=g, dtype=torch.float64).cuda())
    pd.UpdateDomainData()
    ts = torch.tensor([0.05], dtype=torch.float64)
    P.CorrectVelocity(pd, ts, version=1)
    u1 = pd.velocityResult.clone()
    P.CorrectVelocity(pd, ts, version=5)
    assert torch.allclose(pd.velocityResult, u1, rtol=1e-12, atol=1e-12)


def test_corrector_version_checks():
    from pict_b200 import PISOtorch as P
    from setups import build_product, case
    pd = build_product(case("distorted2d"), torch.float64)
    ts = torch.tensor([0.05], dtype=torch.float64)
    # numbers other than 4, 5, 6 take the reference's default branch, the finite-difference corrector
    g = torch.Generator(device="cpu").manual_seed(3)
    for b in pd.getBlocks():
        b.setPressure(torch.randn(b.pressure.shape, generator=g, dtype=torch.float64).cuda())
    N, D = pd.getTotalSize(), pd.getSpatialDims()
    pd.setA(1 + torch.rand(N, generator=g, dtype=torch.float64).cuda())
    pd.setPressureRHS(torch.randn(D * N, generator=g, dtype=torch.float64).cuda())
    pd.UpdateDomainData()
    P.CorrectVelocity(pd, ts, version=1)
    u1 = pd.velocityResult.clone()
    for v in (2, 3, 7):
        P.CorrectVelocity(pd, ts, version=v)
        assert torch.isfinite(u1).all() and torch.equal(pd.velocityResult, u1)
    b = pd.getBlock(0)
    b.setTransform(b.transform, None)  # drop the face transforms
    pd.UpdateDomainData()
    with pytest.raises(RuntimeError):
        P.CorrectVelocity(pd, ts, version=6)
