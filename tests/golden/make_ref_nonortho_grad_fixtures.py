"""Gradient fixtures of the non-orthogonal terms from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``).  For
every setup of ``tests/setups.py:NONORTHO_CASES`` (with a per-cell block viscosity added, so that the
viscosity gradient is checked cell by cell) and every flag set of ``NONORTHO_FLAG_SETS``, this runs the
forward operators once in FP64 and then each raw gradient operator once with seeded gradient inputs:

* SetupAdvectionMatrixGrad    (CGrad, AGrad)          -> velocity / viscosity / boundary velocity gradients
* SetupAdvectionVelocityGrad  (velocityRHSGrad)       -> velocityResultGrad and the parameter gradients
* SetupPressureMatrixGrad     (PGrad)                 -> AGrad
* SetupPressureRHSdivGrad     (pressureRHSdivGrad)    -> pressureRHSGrad, pressureResultGrad, AGrad
* SetupPressureRHSGrad        (pressureRHSGrad, pressureRHSdivGrad) -> AGrad, CGrad, velocityResultGrad,
  pressureResultGrad and the parameter gradients

(extensions/PISO_multiblock_cuda_kernel.cu: PISO_build_matrix_GRAD :3869-4077, kPISO_build_advection_RHS_GRAD
:4388-4478, PISO_build_pressure_matrix_GRAD :4967-5117, k_pressureRHSaddNonOrthoComponents_GRAD :5478-5496, with
the non-orthogonal scatters scatterNonOrthoLaplaceComponents_GRAD :1992-2098 and
scatterNonOrthoLaplaceRHS_v2_GRAD :3212-3392).  ``grad_ops_fixture`` takes the module as an argument, so
``tests/test_gpu_nonortho_grad.py`` runs the same function with this library's module and compares.

Usage (GPU machine):  python tests/golden/make_ref_nonortho_grad_fixtures.py --out <dir>
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


def _np(t):
    return t.detach().double().cpu().numpy().copy()


def _cuda(a):
    return torch.tensor(np.ascontiguousarray(a).reshape(-1), dtype=torch.float64, device="cuda")


def viscous_spec(name, spec=None):
    """The setup (or `spec`) with a per-cell block viscosity 1e-2 * (1 + U[0, 0.5))."""
    from setups import case
    spec = case(name) if spec is None else spec
    rng = np.random.default_rng(11)
    for b in spec["blocks"]:
        shape = np.asarray(b["velocity"]).shape
        b["viscosity"] = 1e-2 * (1.0 + 0.5 * rng.random((1, 1) + tuple(shape[2:])))
    return spec


def fixed_faces(dom):
    out = []
    for bi, b in enumerate(dom.getBlocks()):
        for f in range(2 * dom.getSpatialDims()):
            bnd = b.getBoundary(f)
            if bnd is not None and type(bnd).__name__ == "FixedBoundary":
                out.append((bi, f, bnd))
    return out


def fresh_parameter_grads(dom):
    dom.CreateViscosityGrad()
    dom.CreateVelocityGradOnBlocks()
    dom.CreateVelocityGradOnBoundaries()
    dom.CreateVelocitySourceGradOnBlocks()


def collect_parameter_grads(dom, pre, out):
    out[pre + "viscosity"] = _np(dom.viscosityGrad)
    for k, b in enumerate(dom.getBlocks()):
        out[pre + "velocity_%d" % k] = _np(b.velocityGrad)
        if b.viscosityGrad is not None and b.viscosityGrad.numel() > 0:
            out[pre + "block_viscosity_%d" % k] = _np(b.viscosityGrad)
        if b.velocitySourceGrad is not None and b.velocitySourceGrad.numel() > 0:
            out[pre + "source_%d" % k] = _np(b.velocitySourceGrad)
    for bi, f, bnd in fixed_faces(dom):
        if bnd.velocityGrad is not None and bnd.velocityGrad.numel() > 0:
            out[pre + "boundary_velocity_%d_%d" % (bi, f)] = _np(bnd.velocityGrad)


def grad_ops_fixture(R, name, flag_sets=None):
    from setups import NONORTHO_FLAG_SETS, build_product
    spec = viscous_spec(name)
    D = spec["dims"]
    out = {}
    for flags in (flag_sets or NONORTHO_FLAG_SETS):
        dom = build_product(spec, torch.float64, module=R)
        N = dom.getTotalSize()
        ts = torch.tensor([DT], dtype=torch.float64)
        rng = np.random.default_rng(23 + flags)
        k = "f%d_" % flags
        # forward state
        R.SetupAdvectionMatrix(dom, ts, flags)
        ures = rng.standard_normal((D, N)) * 0.3
        dom.setVelocityResult(_cuda(ures))
        dom.UpdateDomainData()
        R.SetupAdvectionVelocity(dom, ts, flags, False)
        # advection matrix
        dom.CGrad.setValue(_cuda(rng.standard_normal(dom.C.value.numel())))
        dom.setAGrad(_cuda(rng.standard_normal(N)))
        fresh_parameter_grads(dom)
        dom.UpdateDomainData()
        R.SetupAdvectionMatrixGrad(dom, ts, flags)
        torch.cuda.synchronize()
        collect_parameter_grads(dom, k + "advM_", out)
        # advection RHS
        dom.setVelocityRHSGrad(_cuda(rng.standard_normal(D * N)))
        dom.CreateVelocityResultGrad()
        fresh_parameter_grads(dom)
        dom.UpdateDomainData()
        R.SetupAdvectionVelocityGrad(dom, ts, flags, False)
        torch.cuda.synchronize()
        collect_parameter_grads(dom, k + "advV_", out)
        out[k + "advV_velocityResult"] = _np(dom.velocityResultGrad)
        # pressure operators at a given velocity and pressure result
        dom.setVelocityResult(_cuda(rng.standard_normal((D, N)) * 0.3))
        dom.setPressureResult(_cuda(rng.standard_normal(N)))
        dom.UpdateDomainData()
        R.SetupPressureMatrix(dom, ts, flags, False)
        R.SetupPressureRHS(dom, ts, flags, False, timeStepNorm=False)
        dom.PGrad.setValue(_cuda(rng.standard_normal(dom.P.value.numel())))
        dom.CreateAGrad()
        dom.UpdateDomainData()
        R.SetupPressureMatrixGrad(dom, ts, flags, False)
        torch.cuda.synchronize()
        out[k + "pM_A"] = _np(dom.AGrad)
        # pressure RHS divergence
        dom.setPressureRHSdivGrad(_cuda(rng.standard_normal(N)))
        dom.CreatePressureRHSGrad()
        dom.CreatePressureResultGrad()
        dom.CreateAGrad()
        fresh_parameter_grads(dom)
        dom.UpdateDomainData()
        R.SetupPressureRHSdivGrad(dom, ts, flags, False, timeStepNorm=False)
        torch.cuda.synchronize()
        out[k + "pD_pressureRHS"] = _np(dom.pressureRHSGrad)
        out[k + "pD_pressureResult"] = _np(dom.pressureResultGrad)
        out[k + "pD_A"] = _np(dom.AGrad)
        collect_parameter_grads(dom, k + "pD_", out)
        # full pressure RHS
        dom.setPressureRHSGrad(_cuda(rng.standard_normal(D * N)))
        dom.setPressureRHSdivGrad(_cuda(rng.standard_normal(N)))
        dom.CreatePressureResultGrad()
        dom.CreateAGrad()
        dom.CGrad.CreateValue()
        dom.CreateVelocityResultGrad()
        fresh_parameter_grads(dom)
        dom.UpdateDomainData()
        R.SetupPressureRHSGrad(dom, ts, flags, False, timeStepNorm=False)
        torch.cuda.synchronize()
        out[k + "pR_A"] = _np(dom.AGrad)
        out[k + "pR_C"] = _np(dom.CGrad.value)
        out[k + "pR_velocityResult"] = _np(dom.velocityResultGrad)
        out[k + "pR_pressureResult"] = _np(dom.pressureResultGrad)
        out[k + "pR_pressureRHS"] = _np(dom.pressureRHSGrad)
        collect_parameter_grads(dom, k + "pR_", out)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    from setups import NONORTHO_CASES
    for name in NONORTHO_CASES:
        fx = grad_ops_fixture(R, name)
        np.savez_compressed(os.path.join(args.out, "ref_nonortho_grad_%s.npz" % name), **fx)
        print("non-orthogonal gradient fixture", name, len(fx), "arrays", flush=True)


if __name__ == "__main__":
    main()
