"""Passive scalar fixtures from the reference's own CUDA build (run on a GPU machine).

Imports the reference extension built from its sources by ``oracle/build_ref.py`` (``oracle/_ref``).  For
every setup of ``tests/setups.py:SCALAR_CASES`` (1-2 channels, scalar viscosities, Dirichlet and Neumann
faces per channel, static and varying boundary scalars, orthogonal and skewed grids, two blocks, 2D
and 3D) this records in FP64, through the reference's own ``PISOtorch`` API:

* for nonOrthoFlags 0, 25 and 27: the scalar advection matrix of every channel
  (SetupAdvectionMatrix with forPassiveScalar, extensions/PISO_multiblock_cuda_kernel.cu:3601-3865) and the
  scalar RHS of a given scalar result (SetupAdvectionScalar, extensions/PISO_multiblock_cuda_kernel.cu:4079-4183);
* one scalar advection sub-step of the driver (PISOtorch_simulation.py:1085-1167, orthogonal branch)
  from the setup's state, solved with BiCGStab to 1e-12: the blocks' scalar afterwards.

``scalar_fixture`` takes the module as an argument, so ``tests/test_gpu_scalar.py`` runs the same
function with this library's module and compares.

Usage (GPU machine):  python tests/golden/make_ref_scalar_fixtures.py --out <dir>
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
TOL = 1e-12


def _np(t):
    return t.detach().double().cpu().numpy().copy()


def solve(R, A, rhs, tol=TOL, maxit=5000):
    x = torch.zeros_like(rhs)
    if bool(rhs.eq(0).all()):
        return x
    infos = R.SolveLinear(A, rhs, x, torch.IntTensor([maxit]), torch.tensor([tol], dtype=rhs.dtype),
                          R.ConvergenceCriterion.NORM2_NORMALIZED, True, False, 0, False, False, False,
                          BiCGwithPreconditioner=False)
    for i in infos:
        assert i.converged and i.isFiniteResidual, i
    return x


def scalar_substep(R, dom, dt):
    """The scalar part of Simulation._PISO_split_step, orthogonal branch (PISOtorch_simulation.py:1085-1129):
    one matrix and C right-hand sides unless the scalar viscosity or the boundary types differ per
    channel, then one matrix per channel."""
    ts = torch.tensor([dt], dtype=torch.float64)
    C, n = dom.getPassiveScalarChannels(), dom.getTotalSize()
    split = not (dom.isPassiveScalarViscosityStatic() and dom.isAllFixedBoundariesPassiveScalarTypeStatic())
    dom.UpdateDomainData()
    mats = []
    if split:
        for ch in range(C):
            R.SetupAdvectionMatrix(dom, ts, 0, forPassiveScalar=True, passiveScalarChannel=ch)
            mats.append(dom.C.clone())
    else:
        R.SetupAdvectionMatrix(dom, ts, 0, forPassiveScalar=True, passiveScalarChannel=0)
    R.SetupAdvectionScalar(dom, ts, 0)
    if split:
        rhs = torch.split(dom.scalarRHS, n)
        res = torch.cat([solve(R, mats[ch], rhs[ch].contiguous()) for ch in range(C)])
    else:
        res = solve(R, dom.C, dom.scalarRHS)
    dom.setScalarResult(res)
    dom.UpdateDomainData()
    R.CopyScalarResultToBlocks(dom)
    torch.cuda.synchronize()
    return int(split)


def block_scalars(dom):
    C = dom.getPassiveScalarChannels()
    return np.concatenate([_np(b.passiveScalar).reshape(C, -1) for b in dom.getBlocks()], axis=1)


def scalar_fixture(R, name):
    from setups import build_product, scalar_case
    spec = scalar_case(name)
    out = {}
    for flags in FLAG_SETS:
        dom = build_product(spec, torch.float64, module=R)
        C, N = dom.getPassiveScalarChannels(), dom.getTotalSize()
        ts = torch.tensor([DT], dtype=torch.float64)
        k = "f%d_" % flags
        for ch in range(C):
            R.SetupAdvectionMatrix(dom, ts, flags, forPassiveScalar=True, passiveScalarChannel=ch)
            torch.cuda.synchronize()
            out[k + "C%d_value" % ch] = _np(dom.C.value)
            out[k + "A%d" % ch] = _np(dom.A)
        out[k + "C_index"] = dom.C.index.cpu().numpy()
        out[k + "C_row"] = dom.C.row.cpu().numpy()
        sres = np.random.default_rng(41 + flags).random(C * N)
        dom.setScalarResult(torch.tensor(sres, dtype=torch.float64, device="cuda"))
        dom.UpdateDomainData()
        R.SetupAdvectionScalar(dom, ts, flags)
        torch.cuda.synchronize()
        out[k + "sres"] = sres
        out[k + "scalarRHS"] = _np(dom.scalarRHS)
    dom = build_product(spec, torch.float64, module=R)
    out["step_split"] = scalar_substep(R, dom, DT)
    out["step_scalar"] = block_scalars(dom)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import PISOtorch as R
    from setups import SCALAR_CASES
    for name in SCALAR_CASES:
        fx = scalar_fixture(R, name)
        np.savez_compressed(os.path.join(args.out, "ref_scalar_%s.npz" % name), **fx)
        print("scalar fixture", name, "split", int(fx["step_split"]), flush=True)


if __name__ == "__main__":
    main()
