"""Smagorinsky sub-grid-scale viscosity fixtures from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``) and
records SGSviscosityIncompressibleSmagorinsky (extensions/PISO_multiblock_cuda_kernel.cu:6896-7019) in FP64
for ``SGS_CASES`` (stretched, distorted and skewed grids, a varying inflow face, periodic axes, two
blocks with a rotated connection, 3D), with the setups' seeded block velocities.  ``sgs_fixture`` takes
the module as an argument, so ``tests/test_gpu_sgs.py`` runs it with this library's module.

Usage (GPU machine):  python tests/golden/make_ref_sgs_fixtures.py --out <dir>
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

SGS_CASES = ["cavity2d_refined", "distorted2d", "inflow2d", "periodic2d", "twoblock2d_rotated", "channel3d",
             "skewed_twoblock2d_rotated", "skewed_cavity3d"]
COEFFICIENT = 0.17 ** 2


def sgs_fixture(R, name):
    from setups import build_product, case
    dom = build_product(case(name), torch.float64, module=R)
    res = R.SGSviscosityIncompressibleSmagorinsky(dom, torch.tensor([COEFFICIENT], dtype=torch.float64))
    torch.cuda.synchronize()
    return {"nu_sgs": np.concatenate([r.detach().cpu().numpy().reshape(-1) for r in res]),
            "shapes": np.array([list(r.shape) + [1] * (5 - r.dim()) for r in res])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    for name in SGS_CASES:
        np.savez_compressed(os.path.join(args.out, "ref_sgs_%s.npz" % name), **sgs_fixture(R, name))
        print("sgs fixture", name, flush=True)


if __name__ == "__main__":
    main()
