"""Advective outflow fixtures from the reference's own functions (run in a checkout of the reference
sources; no GPU needed).

update_advective_boundaries, balance_boundary_fluxes, get_advective_velocity and the flux helpers of the
reference driver (PISOtorch_simulation.py:80-312) are plain PyTorch over the boundary interface.  This
script reads them from the reference's PISOtorch_simulation.py (and the tolerance default
_get_solver_tolerance from its PISOtorch_diff.py), executes their definitions in a namespace whose
``PISOtorch`` is the CPU stand-in of tests/outflow_standins.py, runs them on FP64 cases, and writes
inputs and resulting boundary tensors to ``ref_outflow_<case>.npz``.  tests/test_outflow_golden.py runs
this package's restatement (pict_b200.PISOtorch_simulation) and the oracle's (oracle/piso_oracle.py
advective_outflow) on the same inputs.

Cases: the reduced cylinder street (outflow face with a boundary transform, static characteristic
velocity); a skewed 2D block with two outflow faces, per-face characteristic velocities (one static
and oblique, one varying) and two passive scalar channels; a 3D block without transforms; and a 3D
block whose fluxes already balance (no rescale).

Usage:  python tests/golden/make_ref_outflow_fixtures.py --reference <reference checkout> --out <dir>
"""
import argparse
import ast
import contextlib
import logging
import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import torch  # noqa: E402

import outflow_standins as S  # noqa: E402
import piso_oracle as po  # noqa: E402

SIM_FUNCS = ["get_fixed_boundary_flux", "get_fixed_boundary_fluxes", "get_advective_velocity",
             "balance_boundary_fluxes", "update_advective_boundaries"]


def _defs(path, names):
    """Source of the named top-level function definitions of a Python file."""
    src = open(path).read()
    tree = ast.parse(src)
    out = []
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in names:
            out.append(ast.get_source_segment(src, node))
    missing = set(names) - {n.split("(")[0].replace("def ", "").strip() for n in out}
    assert not missing, missing
    return "\n\n".join(out)


def reference_namespace(ref):
    diff_ns = {"torch": torch}
    exec(_defs(os.path.join(ref, "PISOtorch_diff.py"), ["_get_solver_tolerance"]), diff_ns)
    diff = type(sys)("PISOtorch_diff")
    diff._get_solver_tolerance = diff_ns["_get_solver_tolerance"]
    ns = {"torch": torch, "warnings": warnings, "PISOtorch": S.stub_module(), "PISOtorch_diff": diff,
          "SAMPLE": lambda name: contextlib.nullcontext(), "_LOG": logging.getLogger("ref")}
    exec(_defs(os.path.join(ref, "PISOtorch_simulation.py"), SIM_FUNCS), ns)
    return ns


# ------------------------------------------------------------------ cases (arrays only)

def _fixed_faces_from_oracle(od, arrs, rng, perturb):
    for i, b in enumerate(od.blocks):
        v = np.array(b.velocity)
        v = v + perturb * rng.standard_normal(v.shape)
        arrs["b%d_velocity" % i] = v
        for f, bnd in enumerate(b.boundaries):
            if bnd.kind != "fixed":
                continue
            arrs["f%d_%d_velocity" % (i, f)] = np.array(bnd.velocity)
            if bnd.transform is not None:
                arrs["f%d_%d_transform" % (i, f)] = np.array(bnd.transform)


def case_street16():
    from pict_b200.cylinder_street import street_spec
    from setups import build_oracle
    spec = street_spec(16, 16, 0.5)
    od = build_oracle(spec)
    arrs = {"dims": 2, "num_blocks": len(od.blocks), "dt": 0.005, "velm": np.array([[1.0, 0.0]]),
            "outflow": np.array(spec["outflow"])}
    _fixed_faces_from_oracle(od, arrs, np.random.default_rng(21), 0.2)
    return arrs


def case_skewed2d_scalar():
    from setups import rotate_distort, tensor_grid
    coords = rotate_distort(tensor_grid(np.linspace(0, 1.2, 13), np.linspace(0, 1.0, 11)), angle=0.4)
    od = po.ODomain(2, 1e-2, scalar_channels=2)
    od.create_block(coords=coords)
    od.close_all(0)
    rng = np.random.default_rng(22)
    ny, nx = 10, 12
    od.close_boundary(0, "-x", np.concatenate([1 + 0.1 * rng.random((1, 1, ny, 1)), 0.1 * rng.random((1, 1, ny, 1))], 1))
    od.close_boundary(0, "+x", 0.8 + 0.2 * rng.random((1, 2, ny, 1)))
    od.close_boundary(0, "+y", 0.3 + 0.2 * rng.random((1, 2, 1, nx)))
    arrs = {"dims": 2, "num_blocks": 1, "dt": 0.02, "outflow": np.array([[0, 1], [0, 3]]),
            "velm0": np.array([[0.7, 0.3]]), "velm1": 0.5 + rng.random((1, 2, 1, nx))}
    _fixed_faces_from_oracle(od, arrs, rng, 0.3)
    arrs["b0_scalar"] = rng.random((1, 2, ny, nx))
    arrs["f0_1_scalar"] = rng.random((1, 2, ny, 1))
    arrs["f0_3_scalar"] = rng.random((1, 2, 1, nx))
    return arrs


def _box3d(balanced):
    nz, ny, nx = 4, 5, 6
    od = po.ODomain(3, 1e-2)
    od.create_block(size=[nx, ny, nz])
    od.close_all(0)
    rng = np.random.default_rng(23)
    inflow = np.concatenate([1 + 0.1 * rng.random((1, 1, nz, ny, 1)), 0.1 * rng.random((1, 2, nz, ny, 1))], 1)
    od.close_boundary(0, "-x", inflow)
    od.close_boundary(0, "+x", inflow.copy() if balanced else 0.9 + 0.1 * rng.random((1, 3, nz, ny, 1)))
    od.close_boundary(0, "+y", np.array([[1.0, 0.0, 0.0]]))
    arrs = {"dims": 3, "num_blocks": 1, "dt": 0.0 if balanced else 0.05, "outflow": np.array([[0, 1]]),
            "velm": np.array([[1.2, 0.1, -0.1]])}
    _fixed_faces_from_oracle(od, arrs, rng, 0.0 if balanced else 0.3)
    return arrs


CASES = {"street16": case_street16, "skewed2d_scalar": case_skewed2d_scalar,
         "box3d": lambda: _box3d(False), "box3d_balanced": lambda: _box3d(True)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="checkout of the reference sources")
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    ns = reference_namespace(args.reference)
    os.makedirs(args.out, exist_ok=True)
    for name, make in CASES.items():
        arrs = make()
        dom, bounds, velm, dt = S.build_case(arrs)
        ns["update_advective_boundaries"](dom, bounds, velm, dt)
        out = dict(arrs)
        out.update(S.outputs(dom, arrs))
        np.savez_compressed(os.path.join(args.out, "ref_outflow_%s.npz" % name), **out)
        print("fixture", name, flush=True)


if __name__ == "__main__":
    main()
