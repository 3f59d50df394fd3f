"""Gradient fixtures from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``),
runs T orthogonal PISO steps of small setups in FP64 with the reference's operators and solvers, and
then the reverse pass of those steps with the reference's gradient operators (SetupAdvectionMatrixGrad,
SetupAdvectionVelocityGrad, SetupPressureCorrectionGrad, CorrectVelocityGrad, Copy*Grad*) and its
solver (transposed SolveLinear + SparseOuterProduct), in the order the reference's autograd wrappers
apply them (PISOtorch_diff.py: linear_solve_GPU :295-375, SetupAdvectionMatrix :377-441,
SetupAdvectionVelocity :531-613, CopyVelocityResultToBlocks :697-729, CopyPressureResultToBlocks
:765-800, SetupPressureCorrection :802-895, CorrectVelocity :1160-1236; driver order
PISOtorch_simulation.py:1170-1312 with the pressure mean removal as a torch op).

Variants: "plain" (the driver's defaults), "tsnorm" (pressure normalised by the time step: timeStepNorm in
SetupPressureCorrection(Grad) and CorrectVelocity(Grad)) and "pgrad" (applyPressureGradient in
SetupAdvectionVelocity(Grad), which subtracts dt grad p of the blocks' pressure from the velocity RHS).

Loss: sum(w * u^T) over the blocks' velocity after T steps, w seeded.  Saved per setup: the gradient
with respect to the initial block velocities, the domain viscosity, block viscosity, block velocity
source and the boundary velocities of fixed faces.  ``tests/test_gpu_reference_grads.py`` compares the
adjoint of this build against these fixtures.

Usage (GPU machine):  python tests/golden/make_ref_grad_fixtures.py --out <dir> [--variants plain,tsnorm,pgrad]
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))

import torch  # noqa: E402

DT = 0.05
T = 2
TOL = 1e-12
GRAD_CASES = ["cavity2d", "periodic2d", "inflow2d", "twoblock2d_rotated"]
VARIANTS = {"plain": dict(ts_norm=False, pgrad=False), "tsnorm": dict(ts_norm=True, pgrad=False),
            "pgrad": dict(ts_norm=False, pgrad=True)}


def fixture_name(variant, name):
    return "ref_grads_%s.npz" % name if variant == "plain" else "ref_grads_%s_%s.npz" % (variant, name)


def solve(R, A, rhs, use_bicg, transpose=False, tol=TOL, maxit=5000):
    x = torch.zeros_like(rhs)
    if bool(rhs.eq(0).all()):
        return x
    infos = R.SolveLinear(A, rhs, x, torch.IntTensor([maxit]), torch.tensor([tol], dtype=rhs.dtype),
                          R.ConvergenceCriterion.NORM2_NORMALIZED, use_bicg, False, 0, transpose, False, False,
                          BiCGwithPreconditioner=False)
    for i in infos:
        assert i.converged and i.isFiniteResidual, i
    return x


def fixed_faces(dom):
    out = []
    for bi, b in enumerate(dom.getBlocks()):
        for f in range(2 * dom.getSpatialDims()):
            bnd = b.getBoundary(f)
            if isinstance(bnd, type(None)):
                continue
            if type(bnd).__name__ in ("FixedBoundary",):
                out.append((bi, f, bnd))
    return out


def forward_step(R, dom, ts, ts_norm=False, pgrad=False):
    blocks = dom.getBlocks()
    st = {"vel": [b.velocity for b in blocks]}
    dom.CreateA()
    dom.C.CreateValue()
    dom.UpdateDomainData()
    R.SetupAdvectionMatrix(dom, ts, 0)
    dom.CreateVelocityRHS()
    dom.UpdateDomainData()
    R.SetupAdvectionVelocity(dom, ts, 0, pgrad)
    st["A"], st["Cval"] = dom.A, dom.C.value
    x = solve(R, dom.C, dom.velocityRHS, True)
    dom.setVelocityResult(x)
    dom.UpdateDomainData()
    st["ustar"] = x
    cors = []
    for _ in range(2):
        c = {"U": dom.velocityResult}
        dom.CreatePressureRHS()
        dom.CreatePressureRHSdiv()
        dom.P.CreateValue()
        dom.UpdateDomainData()
        R.SetupPressureCorrection(dom, ts, 0, False, timeStepNorm=ts_norm)
        c["h"], c["Pval"] = dom.pressureRHS, dom.P.value
        p0 = solve(R, dom.P, dom.pressureRHSdiv, False)
        p = p0 - torch.mean(p0)
        dom.setPressureResult(p)
        dom.CreatePressureOnBlocks()
        dom.UpdateDomainData()
        R.CopyPressureResultToBlocks(dom)
        c["p0"], c["pb"] = p0, [b.pressure for b in blocks]
        dom.CreateVelocityResult()
        dom.UpdateDomainData()
        R.CorrectVelocity(dom, ts, version=1, timeStepNorm=ts_norm)
        cors.append(c)
    st["cors"] = cors
    dom.CreateVelocityOnBlocks()
    dom.UpdateDomainData()
    R.CopyVelocityResultToBlocks(dom)
    return st


class Acc:
    """Accumulated parameter gradients (the reference's Create*Grad zero them before every operator)."""

    def __init__(self, dom):
        blocks = dom.getBlocks()
        self.nu = torch.zeros_like(dom.viscosity)
        self.block_nu = [None if b.viscosity is None else torch.zeros_like(b.viscosity) for b in blocks]
        self.src = [None if b.velocitySource is None else torch.zeros_like(b.velocitySource) for b in blocks]
        self.vb = {(bi, f): torch.zeros_like(bnd.velocity) for bi, f, bnd in fixed_faces(dom)}

    def add(self, dom):
        if dom.viscosityGrad is not None:
            self.nu += dom.viscosityGrad.to(self.nu.device)
        for k, b in enumerate(dom.getBlocks()):
            if self.block_nu[k] is not None and b.viscosityGrad is not None and b.viscosityGrad.numel() > 0:
                self.block_nu[k] += b.viscosityGrad
            if self.src[k] is not None and b.velocitySourceGrad is not None and b.velocitySourceGrad.numel() > 0:
                self.src[k] += b.velocitySourceGrad
        for (bi, f), g in self.vb.items():
            vg = dom.getBlock(bi).getBoundary(f).velocityGrad
            if vg is not None and vg.numel() > 0:
                g += vg


def restore(dom, st, U=None, h=None):
    for b, v in zip(dom.getBlocks(), st["vel"]):
        b.setVelocity(v)
    dom.setA(st["A"])
    dom.C.setValue(st["Cval"])
    if U is not None:
        dom.setVelocityResult(U)
    if h is not None:
        dom.setPressureRHS(h)


def block_velocity_grads(dom):
    return [b.velocityGrad.clone() for b in dom.getBlocks()]


def backward_step(R, dom, ts, st, ubar_blocks, acc, ts_norm=False, pgrad=False):
    blocks = dom.getBlocks()
    # CopyVelocityResultToBlocks
    for b, g in zip(blocks, ubar_blocks):
        b.setVelocityGrad(g)
    dom.CreateVelocityResultGrad()
    dom.UpdateDomainData()
    R.CopyVelocityResultGradFromBlocks(dom)
    ubar = dom.velocityResultGrad.clone()
    Abar = torch.zeros_like(st["A"])
    Cbar = torch.zeros_like(st["Cval"])
    un = [torch.zeros_like(b.velocity) for b in blocks]
    for k in reversed(range(2)):
        c = st["cors"][k]
        # CorrectVelocity
        restore(dom, st, h=c["h"])
        for b, pb in zip(blocks, c["pb"]):
            b.setPressure(pb)
        dom.setVelocityResultGrad(ubar)
        dom.CreateAGrad()
        dom.CreatePressureGradOnBlocks()
        dom.CreatePressureRHSGrad()
        dom.UpdateDomainData()
        R.CorrectVelocityGrad(dom, ts, ts_norm)
        Abar += dom.AGrad
        pbar_b = [b.pressureGrad.clone() for b in blocks]
        hbar = dom.pressureRHSGrad.clone()
        # CopyPressureResultToBlocks
        for b, g in zip(blocks, pbar_b):
            b.setPressureGrad(g)
        dom.CreatePressureResultGrad()
        dom.UpdateDomainData()
        R.CopyPressureResultGradFromBlocks(dom)
        pbar = dom.pressureResultGrad.clone()
        pbar = pbar - torch.mean(pbar)          # p = p0 - mean(p0)
        # pressure solve: b_grad = P^-T p_grad, P_grad = -b_grad p0^T
        dom.P.setValue(c["Pval"])
        dom.UpdateDomainData()
        bbar = solve(R, dom.P, pbar, False, transpose=True)
        Pg = dom.P.WithZeroValue()
        R.SparseOuterProduct(bbar, c["p0"], Pg)
        Pbar = -Pg.value
        # SetupPressureCorrection
        restore(dom, st, U=c["U"], h=c["h"])
        dom.PGrad.setValue(Pbar)
        dom.setPressureRHSGrad(hbar)
        dom.setPressureRHSdivGrad(bbar)
        dom.CreateAGrad()
        dom.CGrad.CreateValue()
        dom.CreateViscosityGrad()
        dom.CreateVelocityResultGrad()
        dom.CreateVelocityGradOnBlocks()
        dom.CreateVelocitySourceGradOnBlocks()
        dom.CreateVelocityGradOnBoundaries()
        dom.UpdateDomainData()
        R.SetupPressureCorrectionGrad(dom, ts, 0, False, ts_norm)
        Abar += dom.AGrad
        Cbar += dom.CGrad.value
        for g, bg in zip(un, block_velocity_grads(dom)):
            g += bg
        acc.add(dom)
        ubar = dom.velocityResultGrad.clone()
    # advection solve: rhs_grad = C^-T u*_grad, C_grad -= rhs_grad u*^T
    restore(dom, st)
    dom.UpdateDomainData()
    rbar = solve(R, dom.C, ubar, True, transpose=True)
    Cg = dom.C.WithZeroValue()
    D = dom.getSpatialDims()
    n = dom.getTotalSize()
    for comp in range(D):
        Cc = dom.C.WithZeroValue()
        R.SparseOuterProduct(rbar[comp * n:(comp + 1) * n].contiguous(), st["ustar"][comp * n:(comp + 1) * n].contiguous(), Cc)
        Cbar -= Cc.value
    # SetupAdvectionVelocity
    dom.setVelocityRHSGrad(rbar)
    dom.CreateViscosityGrad()
    dom.CreateVelocityGradOnBlocks()
    dom.CreateVelocityGradOnBoundaries()
    dom.CreateVelocitySourceGradOnBlocks()
    dom.UpdateDomainData()
    R.SetupAdvectionVelocityGrad(dom, ts, 0, pgrad)
    for g, bg in zip(un, block_velocity_grads(dom)):
        g += bg
    acc.add(dom)
    # SetupAdvectionMatrix
    dom.setAGrad(Abar)
    dom.CGrad.setValue(Cbar)
    dom.CreateViscosityGrad()
    dom.CreateVelocityGradOnBlocks()
    dom.CreateVelocityGradOnBoundaries()
    dom.UpdateDomainData()
    R.SetupAdvectionMatrixGrad(dom, ts, 0)
    for g, bg in zip(un, block_velocity_grads(dom)):
        g += bg
    acc.add(dom)
    return un


def grad_fixture(R, name, ts_norm=False, pgrad=False):
    from setups import build_product, case
    dom = build_product(case(name), torch.float64, module=R)
    ts = torch.tensor([DT], dtype=torch.float64)
    blocks = dom.getBlocks()
    u0 = [b.velocity.clone() for b in blocks]
    tapes = [forward_step(R, dom, ts, ts_norm, pgrad) for _ in range(T)]
    g = torch.Generator(device="cpu").manual_seed(17)
    w = [torch.randn(b.velocity.shape, generator=g, dtype=torch.float64).cuda() for b in dom.getBlocks()]
    acc = Acc(dom)
    ubar = [x.clone() for x in w]
    for st in reversed(tapes):
        ubar = backward_step(R, dom, ts, st, ubar, acc, ts_norm, pgrad)
    out = {"T": T, "dt": DT, "tol": TOL,
           "u0": np.concatenate([x.cpu().numpy().reshape(-1) for x in u0]),
           "w": np.concatenate([x.cpu().numpy().reshape(-1) for x in w]),
           "grad_velocity": np.concatenate([x.cpu().numpy().reshape(-1) for x in ubar]),
           "grad_viscosity": acc.nu.cpu().numpy()}
    for k, t in enumerate(acc.block_nu):
        if t is not None:
            out["grad_block_viscosity_%d" % k] = t.cpu().numpy()
    for k, t in enumerate(acc.src):
        if t is not None:
            out["grad_source_%d" % k] = t.cpu().numpy()
    for (bi, f), t in acc.vb.items():
        out["grad_boundary_velocity_%d_%d" % (bi, f)] = t.cpu().numpy()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    ap.add_argument("--variants", default="plain,tsnorm,pgrad", help="comma-separated subset of %s" % list(VARIANTS))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    for variant in args.variants.split(","):
        for name in GRAD_CASES:
            fx = grad_fixture(R, name, **VARIANTS[variant])
            np.savez_compressed(os.path.join(args.out, fixture_name(variant, name)), **fx)
            print("gradient fixture", variant, name,
                  {k: float(np.abs(v).max()) for k, v in fx.items() if isinstance(v, np.ndarray)}, flush=True)


if __name__ == "__main__":
    main()
