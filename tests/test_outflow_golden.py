"""Advective outflow (update_advective_boundaries + balance_boundary_fluxes) against the reference's own
functions (CPU).

Fixtures ``tests/golden/ref_outflow_<case>.npz`` hold inputs and the boundary tensors the reference's
functions produced from them (tests/golden/make_ref_outflow_fixtures.py, on the stand-ins of
tests/outflow_standins.py).  Checked: this package's restatement (pict_b200.PISOtorch_simulation) on
the same stand-ins, and the FP64 oracle's restatement (oracle/piso_oracle.py) on an oracle domain
holding the same arrays (static characteristic velocity, no passive scalar).
"""
import os

import numpy as np
import pytest

import outflow_standins as S
import piso_oracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["street16", "skewed2d_scalar", "box3d", "box3d_balanced"]


def _load(name):
    d = np.load(os.path.join(HERE, "golden", "ref_outflow_%s.npz" % name))
    return {k: d[k] for k in d.files}


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", CASES)
def test_restatement_matches_reference_functions(name):
    from pict_b200.PISOtorch_simulation import update_advective_boundaries
    arrs = _load(name)
    dom, bounds, velm, dt = S.build_case(arrs)
    update_advective_boundaries(dom, bounds, velm, dt)
    out = S.outputs(dom, arrs)
    keys = [k for k in arrs if k.startswith("out_")]
    assert sorted(keys) == sorted(out)
    for k in keys:
        assert out[k].shape == arrs[k].shape, k
        assert _rel(out[k], arrs[k]) < 1e-14, (k, _rel(out[k], arrs[k]))
    if name == "box3d_balanced":  # fluxes balanced and dt = 0: nothing changes
        for k in keys:
            assert np.array_equal(arrs[k], arrs[k[4:]])


def _oracle_domain(arrs):
    dims = int(arrs["dims"])
    od = po.ODomain(dims, 1.0)
    for i in range(int(arrs["num_blocks"])):
        v = arrs["b%d_velocity" % i]
        od.create_block(velocity=v)
        b = od.blocks[i]
        for f in range(2 * dims):
            key = "f%d_%d_velocity" % (i, f)
            if key in arrs:
                b.boundaries[f] = po.OBoundary("fixed", velocity=arrs[key].copy(),
                                               transform=arrs.get("f%d_%d_transform" % (i, f)))
            else:
                b.boundaries[f] = po.OBoundary("connected")
    return od


@pytest.mark.parametrize("name", ["street16", "box3d", "box3d_balanced"])
def test_oracle_matches_reference_functions(name):
    arrs = _load(name)
    od = _oracle_domain(arrs)
    faces = [tuple(int(v) for v in bf) for bf in arrs["outflow"].reshape(-1, 2)]
    po.advective_outflow(od, faces, arrs["velm"], float(arrs["dt"]))
    for i, b in enumerate(od.blocks):
        for f, bnd in enumerate(b.boundaries):
            k = "out_f%d_%d_velocity" % (i, f)
            if k in arrs:
                assert _rel(np.asarray(bnd.velocity), arrs[k]) < 1e-14, (k, _rel(np.asarray(bnd.velocity), arrs[k]))


def test_outflow_rejects_static_faces_and_foreign_bounds():
    from pict_b200.PISOtorch_simulation import update_advective_boundaries
    import torch
    arrs = _load("box3d")
    dom, bounds, velm, dt = S.build_case(arrs)
    bounds[0].setVelocity(torch.tensor([[1.0, 0.0, 0.0]], dtype=torch.float64))
    with pytest.raises(ValueError, match="must be varying"):
        update_advective_boundaries(dom, bounds, velm, dt)
    dom2, bounds2, _, _ = S.build_case(arrs)
    with pytest.raises(ValueError, match="not \\(all\\) part of the domain"):
        update_advective_boundaries(dom, bounds2, velm, dt)
