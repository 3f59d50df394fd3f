"""Passive scalar gradient fixtures from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``).  For
every setup of ``tests/setups.py:SCALAR_CASES`` and nonOrthoFlags 0, 25 and 27 this runs, in FP64 with
seeded gradient inputs, the reference's raw gradient operators of the passive scalar:

* SetupAdvectionMatrixGrad with forPassiveScalar for every channel (CGrad, AGrad) -> block velocity
  gradients and the scalar viscosity gradient (extensions/PISO_multiblock_cuda_kernel.cu:3869-4077);
* SetupAdvectionScalarGrad (scalarRHSGrad) -> block and boundary scalar gradients, boundary velocity
  gradients, scalar viscosity gradient and scalarResultGrad (extensions/PISO_multiblock_cuda_kernel.cu:4185-4278);
* CopyScalarResultGradFromBlocks / CopyScalarResultGradToBlocks.

``scalar_grad_fixture`` takes the module as an argument, so ``tests/test_gpu_scalar_grad.py`` runs it with
this library's module and compares.

Usage (GPU machine):  python tests/golden/make_ref_scalar_grad_fixtures.py --out <dir>
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
FLAG_SETS = [0, 25, 27]


def _np(t):
    return t.detach().double().cpu().numpy().copy()


def _cuda(a):
    return torch.tensor(np.ascontiguousarray(a).reshape(-1), dtype=torch.float64, device="cuda")


def fresh(dom):
    dom.CreateViscosityGrad()
    dom.CreateVelocityGradOnBlocks()
    dom.CreateVelocityGradOnBoundaries()
    dom.CreatePassiveScalarGradOnBlocks()
    dom.CreatePassiveScalarGradOnBoundaries()


def collect(dom, pre, out):
    out[pre + "viscosity"] = _np(dom.viscosityGrad)
    if dom.hasPassiveScalarViscosityGrad():
        out[pre + "scalar_viscosity"] = _np(dom.passiveScalarViscosityGrad)
    for k, b in enumerate(dom.getBlocks()):
        out[pre + "velocity_%d" % k] = _np(b.velocityGrad)
        out[pre + "scalar_%d" % k] = _np(b.passiveScalarGrad)
        for f in range(2 * dom.getSpatialDims()):
            bnd = b.getBoundary(f)
            if type(bnd).__name__ != "FixedBoundary":
                continue
            if bnd.velocityGrad is not None and bnd.velocityGrad.numel() > 0:
                out[pre + "bvel_%d_%d" % (k, f)] = _np(bnd.velocityGrad)
            if bnd.passiveScalarGrad is not None and bnd.passiveScalarGrad.numel() > 0:
                out[pre + "bscalar_%d_%d" % (k, f)] = _np(bnd.passiveScalarGrad)


def scalar_grad_fixture(R, name):
    from setups import build_product, scalar_case
    spec = scalar_case(name)
    out = {}
    for flags in FLAG_SETS:
        dom = build_product(spec, torch.float64, module=R)
        C, N = dom.getPassiveScalarChannels(), dom.getTotalSize()
        ts = torch.tensor([DT], dtype=torch.float64)
        rng = np.random.default_rng(61 + flags)
        k = "f%d_" % flags
        for ch in range(C):
            R.SetupAdvectionMatrix(dom, ts, flags, forPassiveScalar=True, passiveScalarChannel=ch)
            dom.CGrad.setValue(_cuda(rng.standard_normal(dom.C.value.numel())))
            dom.setAGrad(_cuda(rng.standard_normal(N)))
            fresh(dom)
            dom.UpdateDomainData()
            R.SetupAdvectionMatrixGrad(dom, ts, flags, forPassiveScalar=True, passiveScalarChannel=ch)
            torch.cuda.synchronize()
            collect(dom, k + "M%d_" % ch, out)
        dom.setScalarResult(_cuda(rng.random(C * N)))
        dom.UpdateDomainData()
        R.SetupAdvectionScalar(dom, ts, flags)
        dom.setScalarRHSGrad(_cuda(rng.standard_normal(C * N)))
        dom.CreateScalarResultGrad()
        fresh(dom)
        dom.UpdateDomainData()
        R.SetupAdvectionScalarGrad(dom, ts, flags)
        torch.cuda.synchronize()
        collect(dom, k + "R_", out)
        out[k + "R_scalarResult"] = _np(dom.scalarResultGrad)
    for b in dom.getBlocks():
        b.setPassiveScalarGrad(torch.tensor(rng.standard_normal(tuple(b.passiveScalar.shape)), dtype=torch.float64,
                                            device="cuda"))
    dom.UpdateDomainData()
    R.CopyScalarResultGradFromBlocks(dom)
    torch.cuda.synchronize()
    out["copy_from_blocks"] = _np(dom.scalarResultGrad)
    dom.setScalarResultGrad(_cuda(rng.standard_normal(C * N)))
    dom.UpdateDomainData()
    R.CopyScalarResultGradToBlocks(dom)
    torch.cuda.synchronize()
    out["copy_to_blocks"] = np.concatenate([_np(b.passiveScalarGrad).reshape(C, -1) for b in dom.getBlocks()], axis=1)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    from setups import SCALAR_CASES
    for name in SCALAR_CASES:
        fx = scalar_grad_fixture(R, name)
        np.savez_compressed(os.path.join(args.out, "ref_scalar_grad_%s.npz" % name), **fx)
        print("scalar gradient fixture", name, len(fx), flush=True)


if __name__ == "__main__":
    main()
