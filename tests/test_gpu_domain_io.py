"""Domain checkpoints (pict_b200.domain_io) against files written by the reference's own save_domain (GPU).

Fixtures: tests/golden/ref_domain_io_*.json / .npz, written by the reference's lib/util/domain_io.py through
tests/golden/make_ref_domain_io_fixtures.py for setups with block connections, periodic axes, block
viscosities and sources, vertex coordinates, and passive scalars with Neumann faces and varying
boundary scalars.  Loading one must give the domain the setup builds (fields, boundaries, and the
operators computed on it); saving the setup's domain must give the same JSON and arrays.
"""
import json
import os
import sys

import numpy as np
import pytest
import torch

from setups import build_product

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
from make_ref_domain_io_fixtures import IO_CASES, io_spec  # noqa: E402


def _path(name):
    p = os.path.join(GOLDEN, "ref_domain_io_%s" % name)
    if not os.path.exists(p + ".json"):
        pytest.skip("fixture missing")
    return p


def _np(t):
    return t.detach().double().cpu().numpy()


def _same_domain(a, b):
    assert a.getSpatialDims() == b.getSpatialDims()
    assert a.getPassiveScalarChannels() == b.getPassiveScalarChannels()
    from pict_b200 import PISOtorch as P
    for ba, bb in zip(a.getBlocks(), b.getBlocks()):
        for attr in ["velocity", "pressure", "transform", "viscosity", "velocitySource", "passiveScalar"]:
            ta, tb = getattr(ba, attr), getattr(bb, attr)
            assert (ta is None) == (tb is None), attr
            if ta is not None:
                assert np.allclose(_np(ta), _np(tb), rtol=1e-12, atol=1e-12), attr
        for f in range(2 * a.getSpatialDims()):
            fa, fb = ba.getBoundary(f), bb.getBoundary(f)
            assert type(fa) is type(fb)
            if isinstance(fa, P.FixedBoundary):
                assert np.array_equal(_np(fa.velocity), _np(fb.velocity))
                assert (fa.passiveScalar is None) == (fb.passiveScalar is None)
                if fa.passiveScalar is not None:
                    assert np.array_equal(_np(fa.passiveScalar), _np(fb.passiveScalar))
                    assert fa._scalar_neumann_mask(a.getPassiveScalarChannels()) == \
                        fb._scalar_neumann_mask(a.getPassiveScalarChannels())
            elif isinstance(fa, P.ConnectedBoundary):
                assert list(fa.axes) == list(fb.axes)
                assert a.getBlocks().index(fa.getConnectedBlock()) == b.getBlocks().index(fb.getConnectedBlock())


@pytest.mark.parametrize("name", IO_CASES)
def test_load_reference_checkpoint(name):
    from pict_b200 import PISOtorch as P
    from pict_b200.domain_io import load_domain
    dom = load_domain(_path(name), dtype=torch.float64, device="cuda")
    ref = build_product(io_spec(name), torch.float64)
    _same_domain(dom, ref)
    dom.PrepareSolve()
    ts = torch.tensor([0.05], dtype=torch.float64)
    for d in (dom, ref):
        P.SetupAdvectionMatrix(d, ts, 0)
    assert torch.equal(dom.C.coef, ref.C.coef)
    if dom.getPassiveScalarChannels():
        for d in (dom, ref):
            P.SetupAdvectionMatrix(d, ts, 0, forPassiveScalar=True, passiveScalarChannel=d.getPassiveScalarChannels() - 1)
        assert torch.equal(dom.C.coef, ref.C.coef)


@pytest.mark.parametrize("name", IO_CASES)
def test_save_matches_reference_checkpoint(name, tmp_path):
    from pict_b200.domain_io import load_domain, save_domain
    ref_path = _path(name)
    out = str(tmp_path / "dom")
    save_domain(build_product(io_spec(name), torch.float64), out)
    with open(ref_path + ".json") as fh:
        jr = json.load(fh)
    with open(out + ".json") as fh:
        jo = json.load(fh)
    info_r, info_o = jr.pop("data_info"), jo.pop("data_info")
    assert jo == jr
    assert sorted(info_o) == sorted(info_r)
    for k in info_r:
        assert info_o[k]["shape"] == info_r[k]["shape"] and info_o[k]["dtype"] == info_r[k]["dtype"], k
    with np.load(ref_path + ".npz") as zr, np.load(out + ".npz") as zo:
        assert sorted(zr.files) == sorted(zo.files)
        for k in zr.files:
            # boundary transforms: the reference file holds a restatement's values, equal to round-off
            assert np.allclose(zr[k], zo[k], rtol=1e-12, atol=1e-12), k
    # and back: the written checkpoint loads into the same domain
    _same_domain(load_domain(out, dtype=torch.float64, device="cuda"), build_product(io_spec(name), torch.float64))
