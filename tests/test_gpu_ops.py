"""Per-operator parity of the CUDA path against the FP64 oracle (GPU).

Each operator of the PISO step is run through the public ``PISOtorch`` API of
``pict_b200`` on the same seeded inputs as the oracle restatement
(oracle/piso_oracle.py) and compared field by field: in FP64 to round-off
(rtol/atol 1e-11), in FP32 to single-precision accuracy (rtol 2e-5 relative to
the field's max magnitude).
"""
import numpy as np
import pytest
import torch

import piso_oracle as po
from setups import ALL_CASES, build_oracle, build_product, case

pytestmark = pytest.mark.gpu

DT = 0.05


def _np(t):
    return t.detach().double().cpu().numpy()


def _close(a, b, rtol, what):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    err = np.abs(a - b).max() / scale
    assert err <= rtol, "%s: max rel err %.3e > %.1e" % (what, err, rtol)


def _ts(dom, dt=DT):
    return torch.tensor([dt], dtype=dom.getDtype())


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("name", ALL_CASES)
def test_advection_matrix_and_rhs(name, dtype):
    from pict_b200 import PISOtorch as P
    spec = case(name)
    od = build_oracle(spec)
    pd = build_product(spec, dtype)
    Cref, Aref = po.advection_matrix(od, DT)
    rref = po.advection_rhs(od, DT)
    P.SetupAdvectionMatrix(pd, _ts(pd), 0)
    P.SetupAdvectionVelocity(pd, _ts(pd), 0, False)
    tol = 1e-11 if dtype == torch.float64 else 2e-5
    _close(_np(pd.C.coef), Cref, tol, "C")
    _close(_np(pd.A), Aref, tol, "A")
    _close(_np(pd.velocityRHS).reshape(spec["dims"], -1), rref, tol, "velocityRHS")


@pytest.mark.parametrize("name", ALL_CASES)
def test_csr_export_matches_reference_layout(name):
    from pict_b200 import PISOtorch as P
    spec = case(name)
    od = build_oracle(spec)
    pd = build_product(spec, torch.float64)
    Cref, _ = po.advection_matrix(od, DT)
    P.SetupAdvectionMatrix(pd, _ts(pd), 0)
    v, i, r = po.stencil_to_csr(od, Cref)
    assert np.array_equal(pd.C.row.cpu().numpy(), r)
    assert np.array_equal(pd.C.index.cpu().numpy(), i)
    _close(_np(pd.C.value), v, 1e-11, "C.value")
    # the CSR size equals the reference's Block::ComputeCSRSize sum (extensions/domain_structs.cpp:2151-2161)
    assert pd.C.getSize() == sum(b.ComputeCSRSize() for b in pd.getBlocks())
    # round trip CSR -> stencil
    coef = pd.C.coef.clone()
    pd.C.setValue(pd.C.value.clone())
    _close(_np(pd.C.coef), _np(coef), 0.0, "csr round trip")


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("name", ALL_CASES)
def test_pressure_setup(name, dtype):
    from pict_b200 import PISOtorch as P
    spec = case(name)
    od = build_oracle(spec)
    pd = build_product(spec, dtype)
    Cref, Aref = po.advection_matrix(od, DT)
    rng = np.random.default_rng(7)
    ustar = rng.standard_normal((spec["dims"], od.N)) * 0.3
    Pref = po.pressure_matrix(od, Aref)
    href = po.pressure_rhs(od, DT, Cref, Aref, ustar)
    dref = po.divergence(od, href)
    P.SetupAdvectionMatrix(pd, _ts(pd), 0)
    pd.setVelocityResult(torch.tensor(ustar.reshape(-1), dtype=dtype, device="cuda"))
    pd.UpdateDomainData()
    P.SetupPressureCorrection(pd, _ts(pd), 0, False, False)
    tol = 1e-11 if dtype == torch.float64 else 3e-5
    _close(_np(pd.P.coef), Pref, tol, "P")
    _close(_np(pd.pressureRHS).reshape(spec["dims"], -1), href, tol, "pressureRHS")
    _close(_np(pd.pressureRHSdiv), dref, tol * 10, "pressureRHSdiv")
    # the split entry points give the same result
    pdiv = pd.pressureRHSdiv.clone()
    P.SetupPressureMatrix(pd, _ts(pd), 0, False)
    P.SetupPressureRHS(pd, _ts(pd), 0, False, False)
    _close(_np(pd.pressureRHSdiv), _np(pdiv), 0.0, "split == fused")


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("name", ALL_CASES)
def test_velocity_correction(name, dtype):
    from pict_b200 import PISOtorch as P
    spec = case(name)
    od = build_oracle(spec)
    pd = build_product(spec, dtype)
    rng = np.random.default_rng(11)
    p = rng.standard_normal(od.N)
    h = rng.standard_normal((spec["dims"], od.N))
    Cref, Aref = po.advection_matrix(od, DT)
    uref = po.correct_velocity(od, p, Aref, h)
    P.SetupAdvectionMatrix(pd, _ts(pd), 0)
    pd.setPressureResult(torch.tensor(p, dtype=dtype, device="cuda"))
    pd.setPressureRHS(torch.tensor(h.reshape(-1), dtype=dtype, device="cuda"))
    pd.UpdateDomainData()
    P.CopyPressureResultToBlocks(pd)
    P.CorrectVelocity(pd, _ts(pd), version=1)
    tol = 1e-11 if dtype == torch.float64 else 3e-5
    _close(_np(pd.velocityResult).reshape(spec["dims"], -1), uref, tol, "velocityResult")
    P.CopyVelocityResultToBlocks(pd)
    u_blocks = np.concatenate([_np(b.velocity).reshape(spec["dims"], -1) for b in pd.getBlocks()], axis=1)
    _close(u_blocks, uref, tol, "block velocity")


@pytest.mark.parametrize("name", ["cavity2d", "twoblock2d_rotated", "channel3d"])
def test_velocity_divergence(name):
    from pict_b200 import PISOtorch as P
    spec = case(name)
    od = build_oracle(spec)
    pd = build_product(spec, torch.float64)
    ref = po.divergence(od, od.velocity_global())
    _close(_np(P.ComputeVelocityDivergence(pd)), ref, 1e-11, "velocity divergence")


@pytest.mark.parametrize("name", ["cavity2d_refined", "distorted2d", "channel3d"])
def test_transforms_from_coordinates(name):
    from pict_b200 import PISOtorch as P
    spec = case(name)
    coords = spec["blocks"][0]["coords"]
    t = torch.tensor(coords, dtype=torch.float64, device="cuda").contiguous()
    _close(_np(P.CoordsToTransforms(t)), po.coords_to_transforms(coords), 1e-12, "transforms")
    _close(_np(P.CoordsToFaceTransforms(t)), po.coords_to_face_transforms(coords), 1e-12, "face transforms")
