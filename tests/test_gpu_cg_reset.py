"""CG with residualResetSteps (the restart of extensions/cg_solver_kernel.cu:266-286) against the oracle's CG with
the same restarts (GPU, FP64): the same iteration counts and solutions."""
import numpy as np
import pytest
import torch

import piso_oracle as po
from setups import build_oracle, build_product, case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("reset", [1, 3, 7, 0])
@pytest.mark.parametrize("name", ["cavity2d_refined", "skewed_twoblock2d", "channel3d"])
def test_cg_residual_reset_matches_oracle(name, reset):
    from pict_b200 import PISOtorch as P
    pd = build_product(case(name), torch.float64)
    od = build_oracle(case(name))
    ts = torch.tensor([0.05], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupPressureMatrix(pd, ts, 0, False)
    coef = pd.P.coef.double().cpu().numpy()
    A = po.stencil_to_scipy(od, coef)
    g = np.random.default_rng(4)
    b = g.standard_normal(od.N)
    b -= b.mean()
    tol = 1e-9
    x_ref, inf_ref = po.cg(A, b, tol=tol, maxit=400, reset=reset)
    x = torch.zeros(od.N, dtype=torch.float64, device="cuda")
    infos = P.SolveLinear(pd.P, torch.tensor(b, device="cuda"), x, 400, tol, P.ConvergenceCriterion.NORM2_NORMALIZED,
                          False, False, reset, False, False, False)
    assert infos[0].converged == inf_ref.converged
    assert infos[0].usedIterations == inf_ref.usedIterations, (infos[0].usedIterations, inf_ref.usedIterations)
    err = np.abs(x.cpu().numpy() - x_ref).max() / np.abs(x_ref).max()
    assert err < 1e-8, err


@pytest.mark.parametrize("maxit", [4, 9])
@pytest.mark.parametrize("name", ["cavity2d_refined", "skewed_twoblock2d"])
def test_cg_return_best_result_matches_oracle(name, maxit):
    """returnBestResult: a CG stopped unconverged returns its best iterate with that iteration and criterion."""
    from pict_b200 import PISOtorch as P
    pd = build_product(case(name), torch.float64)
    od = build_oracle(case(name))
    ts = torch.tensor([0.05], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupPressureMatrix(pd, ts, 0, False)
    A = po.stencil_to_scipy(od, pd.P.coef.double().cpu().numpy())
    b = np.random.default_rng(5).standard_normal(od.N)
    b -= b.mean()
    x_ref, inf_ref = po.cg(A, b, tol=1e-14, maxit=maxit, return_best=True)
    x = torch.zeros(od.N, dtype=torch.float64, device="cuda")
    infos = P.SolveLinear(pd.P, torch.tensor(b, device="cuda"), x, maxit, 1e-14,
                          P.ConvergenceCriterion.NORM2_NORMALIZED, False, False, 0, False, False, True)
    assert not infos[0].converged and not inf_ref.converged
    assert infos[0].usedIterations == inf_ref.usedIterations
    assert abs(infos[0].finalResidual - inf_ref.finalResidual) <= 1e-10 * inf_ref.finalResidual
    assert np.abs(x.cpu().numpy() - x_ref).max() <= 1e-10 * np.abs(x_ref).max()
