"""SolveLinear's CG with every convergence criterion and with matrixRankDeficient against the reference's own CUDA
build (fixtures from tests/golden/make_ref_solver_criteria_fixtures.py), through this library's module."""
import os
import sys

import numpy as np
import pytest
import torch

from test_oracle_criteria_golden import CASES, GOLDEN, check_solve

sys.path.insert(0, GOLDEN)
from make_ref_solver_criteria_fixtures import CRITERIA, criteria_fixture  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", CASES)
def test_cg_criteria_match_reference(name):
    from pict_b200 import PISOtorch as P
    with np.load(os.path.join(GOLDEN, "ref_criteria_%s.npz" % name)) as z:
        f = {k: z[k] for k in z.files}
    ours = criteria_fixture(P, name, csr=False)
    np.testing.assert_array_equal(ours["b0"], f["b0"])
    for conv, _ in CRITERIA:
        for key in ("%s_rd0" % conv, "%s_rd1" % conv, "%s_rd1_early" % conv):
            check_solve(ours["x_" + key], ours["info_" + key], f, key)


@pytest.mark.parametrize("rd", [False, True])
@pytest.mark.parametrize("name", ["periodic2d", "twoblock2d_rotated", "channel3d"])
def test_cg_abs_max_matches_oracle(name, rd):
    """ABS_MAX (max |r|; the reference's own result is not usable, see the fixture script) against the oracle."""
    import scipy.sparse as sp
    import piso_oracle as po
    from pict_b200 import PISOtorch as P
    from setups import build_product, case
    with np.load(os.path.join(GOLDEN, "ref_criteria_%s.npz" % name)) as z:
        f = {k: z[k] for k in z.files}
    n = f["b0"].size
    A = sp.csr_matrix((f["value"], f["index"], f["row"]), shape=(n, n))
    b = f["b1"] if rd else f["b0"]
    maxit = 40 if rd else 300  # rank-deficient solves compared while still reproducible (unconverged)
    x_ref, inf_ref = po.cg(A, b, tol=1e-9, maxit=maxit, conv="ABS_MAX", rank_deficient=rd)
    dom = build_product(case(name), torch.float64)
    ts = torch.tensor([0.05], dtype=torch.float64)
    P.SetupAdvectionMatrix(dom, ts, 0)
    P.SetupPressureMatrix(dom, ts, 0, False)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    infos = P.SolveLinear(dom.P, torch.tensor(b, device="cuda"), x, maxit, 1e-9, P.ConvergenceCriterion.ABS_MAX,
                          False, rd)
    assert infos[0].converged == inf_ref.converged
    assert abs(infos[0].usedIterations - inf_ref.usedIterations) <= (0 if rd else 1)
    if infos[0].usedIterations == inf_ref.usedIterations:
        assert abs(infos[0].finalResidual - inf_ref.finalResidual) <= 0.1 * inf_ref.finalResidual
    assert np.abs(x.cpu().numpy() - x_ref).max() <= 1e-6 * np.abs(x_ref).max()


@pytest.mark.parametrize("name", CASES)
def test_bicgstab_criteria_match_reference(name):
    from pict_b200 import PISOtorch as P
    from test_oracle_criteria_golden import BICG_CRITERIA, check_bicg
    with np.load(os.path.join(GOLDEN, "ref_criteria_%s.npz" % name)) as z:
        f = {k: z[k] for k in z.files}
    ours = criteria_fixture(P, name, csr=False)
    for conv, _ in BICG_CRITERIA:
        check_bicg(ours["x_bicg_" + conv], ours["info_bicg_" + conv], f, conv)


@pytest.mark.parametrize("name", ["cavity2d_refined", "channel3d"])
def test_bicgstab_abs_max_matches_oracle(name):
    """BiCGStab with ABS_MAX (max |r|) against the oracle, every component."""
    import scipy.sparse as sp
    import piso_oracle as po
    from pict_b200 import PISOtorch as P
    from setups import build_product, case
    with np.load(os.path.join(GOLDEN, "ref_criteria_%s.npz" % name)) as z:
        f = {k: z[k] for k in z.files}
    n = f["b0"].size
    C = sp.csr_matrix((f["value_C"], f["index_C"], f["row_C"]), shape=(n, n))
    rb = f["b_bicg"]
    D = rb.size // n
    dom = build_product(case(name), torch.float64)
    P.SetupAdvectionMatrix(dom, torch.tensor([0.05], dtype=torch.float64), 0)
    x = torch.zeros(D * n, dtype=torch.float64, device="cuda")
    infos = P.SolveLinear(dom.C, torch.tensor(rb, device="cuda"), x, 300, 1e-10, P.ConvergenceCriterion.ABS_MAX, True,
                          BiCGwithPreconditioner=False)
    for c in range(D):
        xr, ir = po.bicgstab(C, rb[c * n:(c + 1) * n], tol=1e-10, maxit=300, conv="ABS_MAX")
        assert infos[c].converged and ir.converged
        assert abs(infos[c].usedIterations - ir.usedIterations) <= 1
        xs = x[c * n:(c + 1) * n].cpu().numpy()
        assert np.abs(xs - xr).max() <= 1e-6 * np.abs(xr).max()
