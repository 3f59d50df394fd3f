"""pict_solve_static (GPU): the solve entry point whose workspace is the library's fixed device scratch.

Called through the C-ABI and compared with pict_solve (caller-provided workspace) on the same
inputs, twice in a row, for the CG pressure solve and the BiCGStab velocity solve of a 48x48
lid-driven cavity, and for a BiCGStab velocity solve on the largest cavity whose workspace still
fits the scratch; a solve whose workspace exceeds the scratch (that cavity plus one row and column,
or a single-reduction CG on a 640x640 cavity) is rejected before any launch.
The file name sorts last so that the test also runs after every other GPU test of the session.
"""
import ctypes

import numpy as np
import pytest
import torch

from setups import build_product, lid_cavity

pytestmark = pytest.mark.gpu
DT = 0.02


def _solve_both(pd, coef, rhs, params):
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    lib = _lib.load()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ninfo = params.nrhs * pd._desc.num_sims * _lib.SOLVE_INFO_BYTES
    x_ref = torch.zeros_like(rhs)
    info_ref = P.solve_stencil(pd, coef, rhs, x_ref, params)
    outs = []
    for _ in range(2):  # two calls in a row share the scratch
        x = torch.zeros_like(rhs)
        info = torch.zeros(ninfo, dtype=torch.uint8, device=rhs.device)
        _lib.check(lib.pict_solve_static(ctypes.byref(pd._desc), coef.data_ptr(), rhs.data_ptr(), x.data_ptr(),
                                         ctypes.byref(params), info.data_ptr(), st), "pict_solve_static")
        outs.append((x, info))
    torch.cuda.synchronize()
    return x_ref, P.decode_infos(info_ref), [(x, P.decode_infos(i)) for x, i in outs]


def _rel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def _prepared_cavity(n=48):
    """One PISO step's systems of the cavity: advection matrix and RHS, then (after the advection
    solve) the pressure matrix and divergence of the first corrector."""
    from pict_b200 import PISOtorch as P
    pd = build_product(lid_cavity(n, viscosity=1e-3), torch.float32)
    ts = torch.tensor([DT], dtype=torch.float32)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupAdvectionVelocity(pd, ts, 0, False)
    params = P._solve_params(2, 1000, 1e-6, 1, True, False, x_zero=True)
    pd.velocityResult.zero_()
    P.solve_stencil(pd, pd.C.coef, pd.velocityRHS, pd.velocityResult, params)
    P.SetupPressureCorrection(pd, ts)
    torch.cuda.synchronize()
    return pd, ts


def test_static_scratch_cg_matches_workspace_solve():
    from pict_b200 import PISOtorch as P
    pd, ts = _prepared_cavity()
    params = P._solve_params(1, 2000, 1e-6, 1, False, False, x_zero=True, variant=1)
    x_ref, info_ref, outs = _solve_both(pd, pd.P.coef, pd.pressureRHSdiv, params)
    assert info_ref[0].converged and info_ref[0].usedIterations > 5
    for x, info in outs:
        assert info[0].converged and info[0].usedIterations == info_ref[0].usedIterations
        assert _rel(x, x_ref) < 1e-6


def test_static_scratch_bicgstab_matches_workspace_solve():
    from pict_b200 import PISOtorch as P
    pd, ts = _prepared_cavity()
    params = P._solve_params(2, 1000, 1e-6, 1, True, False, x_zero=True)
    x_ref, info_ref, outs = _solve_both(pd, pd.C.coef, pd.velocityRHS, params)
    assert all(i.converged for i in info_ref)
    for x, info in outs:
        assert [i.usedIterations for i in info] == [i.usedIterations for i in info_ref]
        assert _rel(x, x_ref) < 1e-6


def test_static_scratch_rejects_large_workspace():
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    lib = _lib.load()
    cap = lib.pict_solve_static_scratch_bytes()
    pd = build_product(lid_cavity(640, viscosity=1e-3), torch.float32)
    params = P._solve_params(1, 10, 1e-6, 1, False, False, x_zero=True, variant=1)
    assert lib.pict_solve_workspace_bytes(ctypes.byref(pd._desc), ctypes.byref(params)) > cap
    x = torch.zeros_like(pd.pressureRHSdiv)
    info = torch.zeros(_lib.SOLVE_INFO_BYTES, dtype=torch.uint8, device=x.device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    status = lib.pict_solve_static(ctypes.byref(pd._desc), pd.P.coef.data_ptr(), pd.pressureRHSdiv.data_ptr(),
                                   x.data_ptr(), ctypes.byref(params), info.data_ptr(), st)
    assert status != 0
    assert b"static scratch" in lib.pict_last_error()


def _static_status(pd, coef, rhs, params):
    from pict_b200 import _lib
    lib = _lib.load()
    x = torch.zeros_like(rhs)
    info = torch.zeros(params.nrhs * pd._desc.num_sims * _lib.SOLVE_INFO_BYTES, dtype=torch.uint8, device=x.device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.pict_solve_static(ctypes.byref(pd._desc), coef.data_ptr(), rhs.data_ptr(), x.data_ptr(),
                                 ctypes.byref(params), info.data_ptr(), st)


def test_static_scratch_bicgstab_at_the_limit():
    """The byte count that pict_solve_static checks is the layout the solve uses: the largest cavity
    whose 2-component BiCGStab workspace fits the scratch solves like pict_solve; one more row and
    column is rejected."""
    from pict_b200 import PISOtorch as P
    from pict_b200 import _lib
    lib = _lib.load()
    cap = lib.pict_solve_static_scratch_bytes()
    params = P._solve_params(2, 1000, 1e-6, 1, True, False, x_zero=True)

    def need(n):
        pd = build_product(lid_cavity(n, viscosity=1e-3), torch.float32)
        return lib.pict_solve_workspace_bytes(ctypes.byref(pd._desc), ctypes.byref(params))

    n = int((cap / (7 * 2 * 4)) ** 0.5)  # 7 vectors of 2 FP32 components per cell
    while need(n) > cap:
        n -= 1
    while need(n + 1) <= cap:
        n += 1
    assert need(n) <= cap < need(n + 1)
    pd = build_product(lid_cavity(n, viscosity=1e-3), torch.float32)
    ts = torch.tensor([DT], dtype=torch.float32)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupAdvectionVelocity(pd, ts, 0, False)
    torch.cuda.synchronize()
    x_ref, info_ref, outs = _solve_both(pd, pd.C.coef, pd.velocityRHS, params)
    assert all(i.converged for i in info_ref)
    for x, info in outs:
        assert [i.usedIterations for i in info] == [i.usedIterations for i in info_ref]
        assert _rel(x, x_ref) < 1e-6
    big = build_product(lid_cavity(n + 1, viscosity=1e-3), torch.float32)
    P.SetupAdvectionMatrix(big, ts, 0)
    P.SetupAdvectionVelocity(big, ts, 0, False)
    torch.cuda.synchronize()
    assert _static_status(big, big.C.coef, big.velocityRHS, params) != 0
    assert b"static scratch" in lib.pict_last_error()
