"""The CUDA path against the reference's own CUDA build (GPU): golden fixtures of tests/golden/
(generated by tests/golden/make_ref_fixtures.py on a B200 from the reference's compiled module).

Operators are compared in FP64 to round-off; whole runs of the 64x64 lid-driven cavity (Re 1000,
dt 0.01, 100 steps, 2 correctors) are compared in FP64 (solves to 1e-10 on both sides) and in FP32
(solves to 1e-6 RMS residual on both sides), with the measured differences bounded below.
"""
import os

import numpy as np
import pytest
import torch

from setups import ALL_CASES, build_product, case, lid_cavity

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DT = 0.05


def _load(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip("fixture %s missing" % name)
    return np.load(p)


def _np(t):
    return t.detach().double().cpu().numpy()


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-30)


def _fields(pd):
    D = pd.getSpatialDims()
    u = np.concatenate([_np(b.velocity).reshape(D, -1) for b in pd.getBlocks()], axis=1)
    p = np.concatenate([_np(b.pressure).reshape(-1) for b in pd.getBlocks()])
    return u, p


@pytest.mark.parametrize("name", ALL_CASES)
def test_operators_match_reference_cuda(name):
    from pict_b200 import PISOtorch as P
    fx = _load("ref_ops_%s.npz" % name)
    pd = build_product(case(name), torch.float64)
    ts = torch.tensor([DT], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupAdvectionVelocity(pd, ts, 0, False)
    assert np.array_equal(pd.C.row.cpu().numpy(), fx["C_row"])
    assert np.array_equal(pd.C.index.cpu().numpy(), fx["C_index"])
    assert _rel(_np(pd.C.value), fx["C_value"]) < 1e-12
    assert _rel(_np(pd.A), fx["A"]) < 1e-12
    assert _rel(_np(pd.velocityRHS), fx["velocityRHS"]) < 1e-12
    pd.setVelocityResult(torch.tensor(fx["ustar"].reshape(-1), device="cuda"))
    pd.UpdateDomainData()
    P.SetupPressureCorrection(pd, ts)
    assert _rel(_np(pd.P.value), fx["P_value"]) < 1e-12
    assert _rel(_np(pd.pressureRHS), fx["pressureRHS"]) < 1e-12
    assert _rel(_np(pd.pressureRHSdiv), fx["pressureRHSdiv"]) < 1e-11


@pytest.mark.parametrize("variant", [0, 1])
def test_lid_cavity_100_steps_fp64_vs_reference(variant):
    from pict_b200.engine import PISOStepper
    fx = _load("ref_lid64_f64.npz")
    pd = build_product(lid_cavity(int(fx["n"]), viscosity=float(fx["viscosity"])), torch.float64)
    st = PISOStepper(pd, time_step=float(fx["dt"]), advection_tol=float(fx["tol"]), pressure_tol=float(fx["tol"]),
                     cg_variant=variant)
    for _ in range(int(fx["steps"])):
        st.step()
    st.check()
    u, p = _fields(pd)
    assert _rel(u, fx["velocity"]) < 1e-6
    assert _rel(p, fx["pressure"]) < 1e-5


@pytest.mark.parametrize("variant", [0, 1])
def test_lid_cavity_100_steps_fp32_vs_reference(variant):
    from pict_b200.engine import PISOStepper
    fx = _load("ref_lid64_f32.npz")
    pd = build_product(lid_cavity(int(fx["n"]), viscosity=float(fx["viscosity"])), torch.float32)
    st = PISOStepper(pd, time_step=float(fx["dt"]), advection_tol=float(fx["tol"]), pressure_tol=float(fx["tol"]),
                     cg_variant=variant)
    for _ in range(int(fx["steps"])):
        st.step()
    st.check()
    u, p = _fields(pd)
    eu, ep = _rel(u, fx["velocity"]), _rel(p, fx["pressure"])
    print("fp32 vs reference CUDA after 100 steps: velocity %.3e pressure %.3e" % (eu, ep))
    # relative velocity / pressure error bound of the FP32 step against the reference's FP32 CUDA build
    # after 100 steps; both sides stop at 1e-6 RMS residual with different summation orders
    assert eu < 1e-5 and ep < 1e-5
