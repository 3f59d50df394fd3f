"""The raw gradient operators of pict_b200.PISOtorch (SetupAdvectionMatrixGrad, SetupAdvectionVelocityGrad,
SetupPressureCorrectionGrad, CorrectVelocityGrad, Copy*Grad*) driven exactly as the reference's autograd
wrappers drive its own (GPU).

tests/golden/make_ref_grad_fixtures.py ran two FP64 PISO steps and their reverse pass with the
reference's compiled module on a B200; here the same script runs with this library's module in place
of the reference's and must reproduce the stored gradients.  The gradient of a static per-block
velocity source is left out: there the reference's kernels are about 1% away from central finite
differences (tests/test_gpu_reference_grads.py compares this build's value with finite differences).
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_ref_grad_fixtures as G  # noqa: E402


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64).reshape(-1), np.asarray(b, dtype=np.float64).reshape(-1)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("variant", list(G.VARIANTS))
@pytest.mark.parametrize("name", G.GRAD_CASES)
def test_raw_grad_operators_reproduce_reference_gradients(name, variant):
    """variant "tsnorm": timeStepNorm in the pressure and corrector operators and their gradients;
    "pgrad": applyPressureGradient in SetupAdvectionVelocity(Grad)."""
    from pict_b200 import PISOtorch as P
    from setups import case
    p = os.path.join(GOLDEN, G.fixture_name(variant, name))
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    fx = np.load(p)
    out = G.grad_fixture(P, name, **G.VARIANTS[variant])
    static_src = {"grad_source_%d" % k for k, b in enumerate(case(name)["blocks"])
                  if b.get("source") is not None and np.asarray(b["source"]).ndim == 2}
    errs = {}
    for key in fx.files:
        if not key.startswith("grad_") or key in static_src:
            continue
        assert key in out, key
        if np.abs(fx[key]).max() == 0 and np.abs(out[key]).max() == 0:
            continue
        errs[key] = _rel(out[key], fx[key])
    print(name, {k: "%.1e" % v for k, v in errs.items()})
    assert max(errs.values()) < 1e-9, errs


def test_raw_grad_operators_accumulate_and_assign_like_the_reference():
    """Gradient fields are added to (parameter gradients) or assigned (CorrectVelocityGrad's AGrad and
    pressureRHSGrad), so calling an operator twice without Create*Grad doubles the added ones only."""
    import torch
    from pict_b200 import PISOtorch as P
    from setups import build_product, case
    pd = build_product(case("cavity2d"), torch.float64)
    ts = torch.tensor([0.05], dtype=torch.float64)
    P.SetupAdvectionMatrix(pd, ts, 0)
    P.SetupAdvectionVelocity(pd, ts, 0, False)
    g = torch.Generator(device="cpu").manual_seed(5)
    pd.setVelocityRHSGrad(torch.randn(pd.velocityRHS.numel(), generator=g, dtype=torch.float64).cuda())
    pd.CreateVelocityGradOnBlocks()
    pd.CreateViscosityGrad()
    pd.UpdateDomainData()
    P.SetupAdvectionVelocityGrad(pd, ts, 0, False)
    once = pd.getBlock(0).velocityGrad.clone()
    P.SetupAdvectionVelocityGrad(pd, ts, 0, False)
    assert torch.allclose(pd.getBlock(0).velocityGrad, 2 * once, rtol=1e-12, atol=1e-14)
    pd.setVelocityResultGrad(torch.randn(pd.velocityResult.numel(), generator=g, dtype=torch.float64).cuda())
    pd.UpdateDomainData()
    P.CorrectVelocityGrad(pd, ts, False)
    h1, a1 = pd.pressureRHSGrad.clone(), pd.AGrad.clone()
    P.CorrectVelocityGrad(pd, ts, False)
    assert torch.equal(pd.pressureRHSGrad, h1) and torch.equal(pd.AGrad, a1)
