"""Passive scalar transport of the CUDA path against the reference's own CUDA build (GPU).

Fixtures: tests/golden/ref_scalar_*.npz, generated on a B200 by tests/golden/make_ref_scalar_fixtures.py
from the reference's compiled module: the scalar advection matrix of every channel and the scalar RHS
for nonOrthoFlags 0, 25 and 27, and one scalar advection sub-step of the driver.  The same function runs
here with this library's module (operators to FP64 round-off); Simulation's scalar advection, in the
step and in static advection, must give the same sub-step.
"""
import os
import sys

import numpy as np
import pytest
import torch

from setups import SCALAR_CASES, build_product, scalar_case

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_ref_scalar_fixtures as G  # noqa: E402


def _load(name):
    p = os.path.join(GOLDEN, "ref_scalar_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    return np.load(p)


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", SCALAR_CASES)
def test_scalar_operators_match_reference(name):
    from pict_b200 import PISOtorch as P
    fx = _load(name)
    out = G.scalar_fixture(P, name)
    assert int(out["step_split"]) == int(fx["step_split"])
    for key in fx.files:
        if key.endswith("_index") or key.endswith("_row"):
            assert np.array_equal(out[key], fx[key]), key
        elif key == "step_scalar":
            assert _rel(out[key], fx[key]) < 1e-9, key
        elif key not in ("step_split",) and not key.endswith("sres"):
            assert _rel(out[key], fx[key]) < 1e-12, (key, _rel(out[key], fx[key]))


@pytest.mark.parametrize("static", [False, True])
@pytest.mark.parametrize("name", ["scalar_cavity2d", "scalar_twoblock2d_rotated", "scalar_skewed_cavity3d"])
def test_simulation_advects_the_scalar_like_the_reference_driver(name, static):
    """Simulation with advect_passive_scalar: the scalar after one step (taken first in the step, with the
    velocity at its start) and after one static advection step equals the reference's sub-step."""
    from pict_b200.PISOtorch_simulation import Simulation
    fx = _load(name)
    pd = build_product(scalar_case(name), torch.float64)
    sim = Simulation(pd, time_step=G.DT, corrector_steps=2, advection_tol=1e-12, pressure_tol=1e-10,
                     non_orthogonal=False, advect_passive_scalar=True)
    if static:
        assert sim.advect_static(1)
    else:
        assert sim._PISO_split_step(1)
    torch.cuda.synchronize()
    C = pd.getPassiveScalarChannels()
    s = np.concatenate([b.passiveScalar.double().cpu().numpy().reshape(C, -1) for b in pd.getBlocks()], axis=1)
    assert _rel(s, fx["step_scalar"]) < 1e-9


def test_scalar_fp32_operators():
    """FP32 operators against the reference's FP64 ones: single-precision round-off."""
    from pict_b200 import PISOtorch as P
    fx = _load("scalar_distorted2d")
    pd = build_product(scalar_case("scalar_distorted2d"), torch.float32)
    ts = torch.tensor([G.DT], dtype=torch.float32)
    P.SetupAdvectionMatrix(pd, ts, 25, forPassiveScalar=True, passiveScalarChannel=0)
    assert _rel(pd.C.value.double().cpu().numpy(), fx["f25_C0_value"]) < 2e-5
    pd.setScalarResult(torch.tensor(fx["f25_sres"], dtype=torch.float32, device="cuda"))
    pd.UpdateDomainData()
    P.SetupAdvectionScalar(pd, ts, 25)
    assert _rel(pd.scalarRHS.double().cpu().numpy(), fx["f25_scalarRHS"]) < 2e-5
