"""Domain checkpoint fixtures written by the reference's own ``save_domain`` (run in a checkout that has the
reference sources; no GPU needed).

``save_domain`` (lib/util/domain_io.py:44-149) is plain Python over the domain's accessors, so it is run
here on a stand-in object graph: the structure and tensors of a setup of ``tests/setups.py`` (blocks
with vertex coordinates or sizes, viscosities, sources, passive scalars, fixed faces with their
boundary transforms, periodic axes and block connections), with CPU tensors, and a stand-in for the
few ``PISOtorch`` enum names the function compares against.  The result, ``ref_domain_io_<setup>.json``
/ ``.npz`` in ``tests/golden``, is what the reference writes for that domain (device "cpu" in
``data_info`` where the reference would record "cuda"); ``tests/test_gpu_domain_io.py`` loads it with
``pict_b200.domain_io`` and writes the same domain back.

Usage:  python tests/golden/make_ref_domain_io_fixtures.py --reference <reference checkout>
"""
import argparse
import enum
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import torch  # noqa: E402

IO_CASES = ["twoblock2d_rotated", "periodic2d", "channel3d", "scalar_cavity2d", "scalar_inflow2d"]


class _BC(enum.IntEnum):
    DIRICHLET = 0
    NEUMANN = 1


def _stub_module():
    m = types.ModuleType("PISOtorch")
    m.BoundaryConditionType = _BC
    for k, name in enumerate(["DIRICHLET", "DIRICHLET_VARYING", "NEUMANN", "FIXED", "CONNECTED", "PERIODIC"]):
        setattr(m, name, "BT_" + name)
    return m


def _t(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64)


class _Fixed:
    def __init__(self, ob, channels):
        self.type = "BT_FIXED"
        self.velocityType = _BC.DIRICHLET
        self.velocity = _t(ob.velocity)
        self._scalar = _t(ob.scalar) if channels else None
        self.passiveScalarTypes = [(_BC.NEUMANN if t == "neumann" else _BC.DIRICHLET) for t in (ob.scalar_types or ["dirichlet"])]
        self.transform = None if ob.transform is None else _t(ob.transform)

    def hasPassiveScalar(self):
        return self._scalar is not None

    @property
    def passiveScalar(self):
        return self._scalar

    def hasTransform(self):
        return self.transform is not None


class _Connected:
    def __init__(self, other, axes):
        self.type = "BT_CONNECTED"
        self._other = other
        self.axes = list(axes)

    def getConnectedBlock(self):
        return self._other


class _Periodic:
    type = "BT_PERIODIC"


class _Block:
    def __init__(self, spec_block, ob, dims, channels):
        self.name = "block"
        self._dims = dims
        self.velocity = _t(ob.velocity)
        self.pressure = _t(ob.pressure)
        self.viscosity = None if spec_block.get("viscosity") is None else _t(spec_block["viscosity"])
        self.velocitySource = None if spec_block.get("source") is None else _t(spec_block["source"])
        self.passiveScalar = _t(ob.scalar) if channels else None
        self.vertexCoordinates = None if spec_block.get("coords") is None else _t(spec_block["coords"])
        self.transform = None if ob.transform is None else _t(ob.transform)
        self.boundaries = []

    def getSpatialDims(self):
        return self._dims

    def hasViscosity(self):
        return self.viscosity is not None

    def hasPassiveScalarViscosity(self):
        return False

    def hasPassiveScalar(self):
        return self.passiveScalar is not None

    def hasVelocitySource(self):
        return self.velocitySource is not None

    def hasVertexCoordinates(self):
        return self.vertexCoordinates is not None

    def hasTransform(self):
        return self.transform is not None

    def hasFaceTransform(self):
        return False

    def getBoundary(self, f):
        return self.boundaries[f]


class _Domain:
    def __init__(self, spec):
        from setups import build_oracle
        od = build_oracle(spec)
        self.name = "test"
        self._dims = spec["dims"]
        self.viscosity = _t([spec["viscosity"]])
        self._channels = spec.get("scalar_channels", 0)
        sv = spec.get("scalar_viscosity")
        self.passiveScalarViscosity = None if sv is None else _t(np.asarray(sv, dtype=np.float64).reshape(-1))
        self.blocks = [_Block(sb, ob, self._dims, self._channels) for sb, ob in zip(spec["blocks"], od.blocks)]
        for blk, ob in zip(self.blocks, od.blocks):
            for bnd in ob.boundaries:
                if bnd.kind == "fixed":
                    blk.boundaries.append(_Fixed(bnd, self._channels))
                elif bnd.kind == "connected":
                    blk.boundaries.append(_Connected(self.blocks[bnd.block], bnd.axes))
                else:
                    blk.boundaries.append(_Periodic())

    def getSpatialDims(self):
        return self._dims

    def getPassiveScalarChannels(self):
        return self._channels

    def hasPassiveScalarViscosity(self):
        return self.passiveScalarViscosity is not None

    def getBlocks(self):
        return self.blocks


def io_spec(name):
    from setups import case, scalar_case
    if name.startswith("scalar_"):
        return scalar_case(name)
    spec = case(name)
    spec["scalar_channels"] = 0
    return spec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="checkout of the reference (for lib/util/domain_io.py)")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    sys.modules["PISOtorch"] = _stub_module()
    src = os.path.join(args.reference, "lib", "util", "domain_io.py")
    spec = importlib.util.spec_from_file_location("ref_domain_io", src)
    ref_io = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref_io)
    for name in IO_CASES:
        ref_io.save_domain(_Domain(io_spec(name)), os.path.join(args.out, "ref_domain_io_%s" % name))
        print("domain checkpoint fixture", name, flush=True)


if __name__ == "__main__":
    main()
