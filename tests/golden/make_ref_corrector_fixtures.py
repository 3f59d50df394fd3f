"""Velocity-corrector fixtures from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``).  For
every setup of ``CORRECTOR_CASES`` this sets seeded block pressures, A and H/A (pressureRHS) in FP64 and
records the velocity result of CorrectVelocity for the versions 1 (finite differences), 4 (face fluxes
with orthogonal metrics), 5 and 6 (finite-volume pressure gradient with interpolated cell fluxes /
staggered face transforms), 5 also with timeStepNorm (extensions/PISO_multiblock_cuda_kernel.cu:6163-6201).

The finite-volume versions read the transforms of fixed boundaries (5) and the blocks' face transforms
(6) without checking for them, so they are only run where every transformed block has both.
``corrector_fixture`` takes the module as an argument, so ``tests/test_gpu_correctors.py`` runs the
same function with this library's module and compares.

Usage (GPU machine):  python tests/golden/make_ref_corrector_fixtures.py --out <dir>
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
CORRECTOR_CASES = ["cavity2d_refined", "distorted2d", "periodic2d", "fullperiodic2d", "inflow2d", "twoblock2d_rotated",
                   "channel3d", "twoblock3d", "skewed_channel2d", "skewed_twoblock2d", "skewed_twoblock2d_rotated",
                   "skewed_cavity3d", "skewed_channel3d"]
RUNS = [(1, False), (4, False), (5, False), (5, True), (6, False)]


def _np(t):
    return t.detach().double().cpu().numpy().copy()


def fvm_ready(dom):
    """Every transformed block has face transforms and transformed fixed boundaries."""
    for b in dom.getBlocks():
        if not b.hasTransform():
            continue
        if not b.hasFaceTransform():
            return False
        for f in range(2 * dom.getSpatialDims()):
            bnd = b.getBoundary(f)
            if type(bnd).__name__ == "FixedBoundary" and not bnd.hasTransform():
                return False
    return True


def corrector_fixture(R, name):
    from setups import build_product, case
    dom = build_product(case(name), torch.float64, module=R)
    D, N = dom.getSpatialDims(), dom.getTotalSize()
    rng = np.random.default_rng(31)
    for b in dom.getBlocks():
        b.setPressure(torch.tensor(rng.standard_normal(tuple(b.pressure.shape)), dtype=torch.float64, device="cuda"))
    A = 1.0 + rng.random(N)
    h = rng.standard_normal(D * N) * 0.5
    dom.setA(torch.tensor(A, dtype=torch.float64, device="cuda"))
    dom.setPressureRHS(torch.tensor(h, dtype=torch.float64, device="cuda"))
    dom.CreateVelocityResult()
    dom.UpdateDomainData()
    ts = torch.tensor([DT], dtype=torch.float64)
    out = {"A": A, "h": h, "p": np.concatenate([_np(b.pressure).reshape(-1) for b in dom.getBlocks()]),
           "fvm_ready": int(fvm_ready(dom))}
    for version, tsn in RUNS:
        if version in (5, 6) and not out["fvm_ready"]:
            continue
        R.CorrectVelocity(dom, ts, version=version, timeStepNorm=tsn)
        torch.cuda.synchronize()
        out["u_v%d%s" % (version, "_tsn" if tsn else "")] = _np(dom.velocityResult)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    for name in CORRECTOR_CASES:
        fx = corrector_fixture(R, name)
        np.savez_compressed(os.path.join(args.out, "ref_corrector_%s.npz" % name), **fx)
        print("corrector fixture", name, sorted(k for k in fx if k.startswith("u_")), flush=True)


if __name__ == "__main__":
    main()
