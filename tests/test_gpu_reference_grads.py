"""Adjoint against the reference's own gradient kernels (GPU): fixtures of tests/golden/ produced by
tests/golden/make_ref_grad_fixtures.py, which runs the reference's compiled operators, solvers and
*Grad operators in the order of its autograd wrappers (PISOtorch_diff.py).

Two FP64 PISO steps (solves to 1e-12) of small setups, loss sum(w * u^T); compared: gradients with
respect to the initial velocity, domain viscosity, block viscosity, velocity source and boundary
velocities.  The one quantity on which the reference's kernels disagree with central finite
differences of the forward step (the gradient of a static, per-block velocity source, off by about 1%)
is compared with finite differences instead.
"""
import os

import numpy as np
import pytest
import torch

from setups import build_product, case

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _blocks_to_global(vec, blocks, D):
    out, o = [], 0
    for b in blocks:
        n = b.velocity[0, 0].numel()
        out.append(vec[o:o + D * n].reshape(D, n))
        o += D * n
    return np.concatenate(out, axis=1).reshape(-1)


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64).reshape(-1), np.asarray(b, dtype=np.float64).reshape(-1)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def _fd_static_source(adj, b, u0, w, steps, eps=1e-6):
    src = b.velocitySource
    base = src.clone()
    g = np.zeros(src.numel())
    for c in range(src.numel()):
        vals = []
        for sgn in (1, -1):
            src.copy_(base)
            src.view(-1)[c] += sgn * eps
            adj.set_velocity(u0)
            for _ in range(steps):
                adj.st.step()
            adj.st.check()
            vals.append(float((w * adj.velocity()).sum()))
        g[c] = (vals[0] - vals[1]) / (2 * eps)
    src.copy_(base)
    return g


@pytest.mark.parametrize("name", ["cavity2d", "periodic2d", "inflow2d", "twoblock2d_rotated"])
def test_adjoint_matches_reference_grad_kernels(name):
    from pict_b200.engine import PISOStepper
    from pict_b200.adjoint import PISOAdjoint, rollout
    p = os.path.join(GOLDEN, "ref_grads_%s.npz" % name)
    if not os.path.exists(p):
        pytest.skip("fixture missing")
    fx = np.load(p)
    pd = build_product(case(name), torch.float64)
    pd.CreateVelocityGradOnBoundaries()
    for b in pd.getBlocks():
        b.CreateViscosityGrad()
        b.CreateVelocitySourceGrad()
    pd.UpdateDomainData()
    D = pd.getSpatialDims()
    blocks = pd.getBlocks()
    st = PISOStepper(pd, time_step=float(fx["dt"]), advection_tol=float(fx["tol"]), pressure_tol=float(fx["tol"]))
    adj = PISOAdjoint(st)
    u0 = adj.velocity().clone()
    assert _rel(u0.cpu().numpy(), _blocks_to_global(fx["u0"], blocks, D)) < 1e-12
    w = torch.tensor(_blocks_to_global(fx["w"], blocks, D), dtype=torch.float64, device="cuda")
    u0r = u0.clone().requires_grad_(True)
    nu = pd._sim_visc.clone().requires_grad_(True)
    out = rollout(adj, u0r, int(fx["T"]), [int(fx["T"])], nu=nu)
    (w * out[0]).sum().backward()
    errs = {"velocity": _rel(u0r.grad.cpu().numpy(), _blocks_to_global(fx["grad_velocity"], blocks, D))}
    if np.abs(fx["grad_viscosity"]).max() > 0:
        errs["viscosity"] = _rel(nu.grad.cpu().numpy(), fx["grad_viscosity"])
    for k, b in enumerate(blocks):
        if "grad_block_viscosity_%d" % k in fx:
            errs["block_viscosity_%d" % k] = _rel(b.viscosityGrad.cpu().numpy(), fx["grad_block_viscosity_%d" % k])
        if "grad_source_%d" % k in fx:
            if b.velocitySource.dim() == 2:
                # static [1, D] source: the reference's accumulated gradient differs from central finite
                # differences of the (identical) forward step by ~1%; compare both with FD instead
                fd = _fd_static_source(adj, b, u0, w, int(fx["T"]))
                mine = b.velocitySourceGrad.cpu().numpy().reshape(-1)
                print("static source: this build vs FD %.1e, reference vs FD %.1e"
                      % (_rel(mine, fd), _rel(fx["grad_source_%d" % k], fd)))
                errs["source_%d_vs_fd" % k] = _rel(mine, fd)
            else:
                errs["source_%d" % k] = _rel(b.velocitySourceGrad.cpu().numpy(), fx["grad_source_%d" % k])
        for f, bnd in enumerate(b.boundaries):
            key = "grad_boundary_velocity_%d_%d" % (k, f)
            if key in fx:
                errs[key] = _rel(bnd.velocityGrad.cpu().numpy(), fx[key])
    print(name, {k: "%.1e" % v for k, v in errs.items()})
    assert max(errs.values()) < 1e-6, errs
