"""Maximum-velocity fixtures from the reference's own CUDA build (run on a GPU machine).

Domain::getMaxVelocity / getMaxVelocityMagnitude (extensions/domain_structs.cpp:1564-1600, 2387-2410) with
and without the fixed boundaries and in physical or computational (transformed) coordinates: the
quantities the adaptive time step (PISOtorch_simulation.py:55-64, 1329-1372) is computed from.  For every
setup of tests/setups.py and the reduced cylinder street, built through the reference's ``PISOtorch`` API
(oracle/_ref) with seeded random block velocities and, on the street, a varying outflow face, the script
records the block velocities and the eight values per domain.  It also runs the adaptive step of
Simulation._PISO_adaptive_step (PISOtorch_simulation.py:1329-1372: substeps from the CFL number and the
domain's maximum computational velocity with its boundaries, the remaining time split evenly) with the
reference's operators (the orthogonal step of make_ref_fixtures.py) on a lid-driven cavity whose lid
moves at 4, for 3 major steps in FP64, and records the substep counts and fields.
tests/test_gpu_cfl.py compares.

Usage (GPU machine):  python tests/golden/make_ref_maxvel_fixtures.py --out <dir>
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
sys.path.insert(0, ROOT)

import torch  # noqa: E402

from make_ref_fixtures import block_fields, piso_step, ref_module  # noqa: E402

COMBOS = [(wb, comp) for wb in (False, True) for comp in (False, True)]


def domain_for(R, name):
    from setups import build_product, case
    if name == "street16":
        from pict_b200.cylinder_street import build_street, street_spec
        dom, _ = build_street(street_spec(16, 16, 0.5), module=R, dtype=torch.float64)
        return dom
    return build_product(case(name), torch.float64, module=R)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory the fixtures are written to")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    R = ref_module()
    from setups import ALL_CASES
    out = {}
    for ci, name in enumerate(list(ALL_CASES) + ["street16"]):
        dom = domain_for(R, name)
        g = torch.Generator(device="cpu").manual_seed(100 + ci)
        for bi, b in enumerate(dom.getBlocks()):
            v = torch.randn(b.velocity.shape, generator=g, dtype=torch.float64) * (0.5 + bi)
            b.setVelocity(v.cuda().contiguous())
            out["%s_b%d_velocity" % (name, bi)] = v.numpy()
        if name == "street16":
            bnd = dom.getBlock(dom.getNumBlocks() - 1).getBoundary("+x")
            ov = torch.randn(bnd.velocity.shape, generator=g, dtype=torch.float64) * 3.0
            bnd.setVelocity(ov.cuda().contiguous())
            out["%s_outflow" % name] = ov.numpy()
        has_t = all(b.hasTransform() for b in dom.getBlocks())
        vals = []
        for wb, comp in COMBOS:
            if comp and not has_t:
                vals += [np.nan, np.nan]
                continue
            vals.append(float(dom.getMaxVelocity(wb, comp).cpu()))
            vals.append(float(dom.getMaxVelocityMagnitude(wb, comp).cpu()))
        out["%s_values" % name] = np.array(vals)
        print(name, vals, flush=True)
    # adaptive major steps
    from setups import build_product, lid_cavity
    dom = build_product(lid_cavity(24, viscosity=1e-2, lid=4.0), torch.float64, module=R)
    target, cfl = 0.05, 0.8
    counts, steps_ts = [], []
    for _ in range(3):
        remaining, n = target, 0
        while remaining > 0 and not np.isclose(remaining, 0):
            max_vel = float(dom.getMaxVelocity(True, True).cpu())
            max_ts = remaining if np.isclose(max_vel, 0) else cfl / max_vel
            ts = remaining if max_ts >= remaining else remaining / int(np.ceil(remaining / max_ts))
            remaining -= ts
            piso_step(R, dom, ts, 1e-12)
            steps_ts.append(ts)
            n += 1
        counts.append(n)
    u, p = block_fields(dom)
    out.update({"adaptive_counts": np.array(counts), "adaptive_ts": np.array(steps_ts), "adaptive_velocity": u,
                "adaptive_pressure": p, "adaptive_target": target, "adaptive_cfl": cfl})
    print("adaptive substeps", counts, flush=True)
    np.savez_compressed(os.path.join(args.out, "ref_maxvel.npz"), **out)


if __name__ == "__main__":
    main()
