"""Non-orthogonal terms (nonOrthoFlags) of the CUDA path against the reference's own CUDA build (GPU).

Fixtures: tests/golden/ref_nonortho_*.npz, generated on a B200 from the reference's compiled module by
tests/golden/make_ref_nonortho_fixtures.py (skewed and distorted 2D/3D grids with walls, periodic axes,
an inflow face and two connected blocks, flag sets 25, 27 and 19).  Operators are compared in FP64 to
round-off and in FP32 to single-precision round-off; four FP64 steps of the non-orthogonal driver
branch (pressure solves to 1e-5, where the reference's CG stops too) are compared field by field and
by CG iteration counts, through the operator API and through Simulation.
"""
import os
import sys

import numpy as np
import pytest
import torch

from setups import NONORTHO_CASES, NONORTHO_FLAG_SETS, build_oracle, build_product, case

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from make_ref_nonortho_fixtures import DT, piso_step_nonortho, rest_spec  # noqa: E402

STEP_CASES = ["distorted2d", "skewed_twoblock2d", "skewed_cavity3d", "skewed_channel2d"]


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


def _operators(pd, fx, flags, dtype):
    from pict_b200 import PISOtorch as P
    k = "f%d_" % flags
    ts = torch.tensor([DT], dtype=dtype)
    P.SetupAdvectionMatrix(pd, ts, flags)
    pd.setVelocityResult(torch.tensor(fx[k + "ures"].reshape(-1), dtype=dtype, device="cuda"))
    pd.UpdateDomainData()
    P.SetupAdvectionVelocity(pd, ts, flags, False)
    out = dict(C_row=pd.C.row.cpu().numpy(), C_index=pd.C.index.cpu().numpy(), C_value=_np(pd.C.value), A=_np(pd.A),
               velocityRHS=_np(pd.velocityRHS))
    pd.setVelocityResult(torch.tensor(fx[k + "ustar"].reshape(-1), dtype=dtype, device="cuda"))
    pd.setPressureResult(torch.tensor(fx[k + "pres"], dtype=dtype, device="cuda"))
    pd.UpdateDomainData()
    P.SetupPressureMatrix(pd, ts, flags, False)
    P.SetupPressureRHS(pd, ts, flags, False, timeStepNorm=False)
    out.update(P_row=pd.P.row.cpu().numpy(), P_index=pd.P.index.cpu().numpy(), P_value=_np(pd.P.value),
               pressureRHS=_np(pd.pressureRHS), pressureRHSdiv=_np(pd.pressureRHSdiv))
    return out


@pytest.mark.parametrize("flags", NONORTHO_FLAG_SETS)
@pytest.mark.parametrize("name", NONORTHO_CASES)
def test_nonortho_operators_match_reference_fp64(name, flags):
    fx = _load("ref_nonortho_%s.npz" % name)
    k = "f%d_" % flags
    out = _operators(build_product(case(name), torch.float64), fx, flags, torch.float64)
    for m in ("C", "P"):
        assert np.array_equal(out[m + "_row"], fx[k + m + "_row"])
        assert np.array_equal(out[m + "_index"], fx[k + m + "_index"])
        assert _rel(out[m + "_value"], fx[k + m + "_value"]) < 1e-12
    assert _rel(out["A"], fx[k + "A"]) < 1e-12
    assert _rel(out["velocityRHS"], fx[k + "velocityRHS"]) < 1e-12
    assert _rel(out["pressureRHS"], fx[k + "pressureRHS"]) < 1e-12
    assert _rel(out["pressureRHSdiv"], fx[k + "pressureRHSdiv"]) < 1e-11


@pytest.mark.parametrize("name", NONORTHO_CASES)
def test_nonortho_operators_fp32(name):
    """FP32 operators against the reference's FP64 operators: single-precision round-off."""
    fx = _load("ref_nonortho_%s.npz" % name)
    k = "f25_"
    out = _operators(build_product(case(name), torch.float32), fx, 25, torch.float32)
    for m in ("C_value", "A", "velocityRHS", "P_value", "pressureRHS"):
        assert _rel(out[m], fx[k + m]) < 2e-5, m
    assert _rel(out["pressureRHSdiv"], fx[k + "pressureRHSdiv"]) < 1e-4


@pytest.mark.parametrize("name", STEP_CASES)
def test_nonortho_steps_match_reference(name):
    from pict_b200 import PISOtorch as P
    fx = _load("ref_nonortho_%s.npz" % name)
    assert fx["steps_infos"][:, 2].all()
    pd = build_product(rest_spec(name), torch.float64)
    infos = []
    for _ in range(int(fx["steps_n"])):
        infos += piso_step_nonortho(P, pd, float(fx["steps_dt"]), int(fx["steps_flags"]))
    torch.cuda.synchronize()
    its = [int(i[2]) for i in infos if i[0] == "p"]
    ref_its = [int(x) for x, kind in zip(fx["steps_infos"][:, 1], fx["steps_info_kind"]) if kind == 1]
    assert its == ref_its
    u, p = _fields(pd)
    ur, pr = fx["steps_velocity"], fx["steps_pressure"]
    assert _rel(u, ur) < 1e-9
    scale = max(np.abs(pr).max(), 1e-12 * np.abs(ur).max())
    assert np.abs(p - pr).max() <= 1e-8 * scale + 1e-15


def test_simulation_non_orthogonal_branch_matches_reference():
    """Simulation(non_orthogonal=True) on a distorted grid takes the reference's non-orthogonal branch."""
    from pict_b200.PISOtorch_simulation import Simulation
    fx = _load("ref_nonortho_distorted2d.npz")
    pd = build_product(rest_spec("distorted2d"), torch.float64)
    sim = Simulation(pd, time_step=float(fx["steps_dt"]), corrector_steps=2, non_orthogonal=True,
                     advection_tol=1e-12, pressure_tol=float(fx["steps_p_tol"]), velocity_corrector="FD")
    assert sim._non_ortho_flags() == 25
    assert sim._PISO_split_step(int(fx["steps_n"]))
    torch.cuda.synchronize()
    u, p = _fields(pd)
    assert _rel(u, fx["steps_velocity"]) < 1e-9
    assert _rel(p, fx["steps_pressure"]) < 1e-8


def test_simulation_orthogonal_metrics_take_the_orthogonal_step():
    """On orthogonal metrics the non-orthogonal terms vanish: the flags resolve to 0 and the fused step runs."""
    from pict_b200.PISOtorch_simulation import Simulation
    pd = build_product(case("cavity2d_refined"), torch.float64)
    sim = Simulation(pd, time_step=0.02, non_orthogonal=True)
    assert sim._non_ortho_flags() == 0


def test_nonortho_operator_path_equals_oracle_on_a_fresh_setup():
    """Independent of the fixtures: a distorted two-block grid with a rotated connection, operators vs oracle."""
    import piso_oracle as po
    spec = case("skewed_twoblock2d_rotated", seed=3)
    od = build_oracle(spec)
    pd = build_product(spec, torch.float64)
    from pict_b200 import PISOtorch as P
    ts = torch.tensor([0.03], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 25)
    P.CopyVelocityResultFromBlocks(pd)
    P.SetupAdvectionVelocity(pd, ts, 25, False)
    C, A = po.advection_matrix(od, 0.03, 25)
    assert _rel(_np(pd.A), A) < 1e-12
    assert _rel(_np(pd.velocityRHS), po.advection_rhs(od, 0.03, 25, od.velocity_global()).reshape(-1)) < 1e-12
