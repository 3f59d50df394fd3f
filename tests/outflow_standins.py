"""CPU stand-ins with the PISOtorch boundary interface (test infrastructure).

The advective outflow functions of the reference driver (update_advective_boundaries,
balance_boundary_fluxes, get_advective_velocity; PISOtorch_simulation.py:80-312) are plain PyTorch over
a small part of the domain interface: blocks with velocity / passive scalar tensors, fixed boundaries
with velocity, transform, GetFluxes and setters.  These classes provide that interface on CPU tensors so
that the reference's own functions (tests/golden/make_ref_outflow_fixtures.py) and this package's
restatement (pict_b200.PISOtorch_simulation) run on identical inputs without a GPU.

``FixedBoundary.GetFluxes`` restates FixedBoundary::GetFluxes (extensions/domain_structs.cpp:527-542):
per face cell det * (M^-1 u)_axis of the boundary velocity (u_axis without a transform).
"""
from __future__ import annotations

import enum
import types

import numpy as np
import torch


class BoundaryConditionType(enum.IntEnum):
    DIRICHLET = 0
    NEUMANN = 1


class FixedBoundary:
    def __init__(self, dims, face, face_shape, velocity, transform=None, scalar=None, scalar_types=None):
        self._dims = dims
        self._face = face
        self._shape = list(face_shape)  # z, y, x of the face (1 along the face axis)
        self.velocityType = BoundaryConditionType.DIRICHLET
        self._velocity = velocity
        self.transform = transform
        self._scalar = scalar
        self.passiveScalarTypes = list(scalar_types or [BoundaryConditionType.DIRICHLET])
        self._parent = None

    def getSpatialDims(self):
        return self._dims

    def getSizes(self):
        xyz = list(reversed(self._shape)) + [1] * (3 - self._dims)
        return xyz + [self._dims]

    def hasTransform(self):
        return self.transform is not None

    @property
    def isVelocityStatic(self):
        return self._velocity.dim() == 2

    @property
    def velocity(self):
        return self._velocity

    def setVelocity(self, t):
        assert t.size(1) == self._dims
        self._velocity = t.contiguous()

    def _varying(self):
        v = self._velocity
        if v.dim() == 2:
            v = v.reshape([1, self._dims] + [1] * self._dims).expand([1, self._dims] + self._shape)
        return v

    def GetFluxes(self):
        v = self._varying()
        a = self._face >> 1
        if self.transform is None:
            return v[:, a:a + 1].clone()
        D = self._dims
        row = self.transform[..., D * D + a * D: D * D + (a + 1) * D]  # [1, zyx, D]
        det = self.transform[..., -1]
        flux = det * (row * torch.movedim(v, 1, -1)).sum(-1)
        return flux.unsqueeze(1)

    def hasPassiveScalar(self):
        return self._scalar is not None

    def isPassiveScalarStatic(self):
        return self._scalar.dim() == 2

    @property
    def passiveScalar(self):
        return self._scalar

    def setPassiveScalar(self, t):
        self._scalar = t.contiguous()

    def getParentDomain(self):
        return self._parent


class VaryingDirichletBoundary:  # deprecated reference classes, never instantiated here
    pass


class StaticDirichletBoundary:
    pass


class _Other:
    """A face that is not a fixed boundary (connected / periodic)."""


class Block:
    def __init__(self, velocity, scalar=None):
        self.velocity = velocity
        self.passiveScalar = scalar
        self.boundaries = []

    def getBoundary(self, i):
        return self.boundaries[i]

    def getFixedBoundaries(self):
        return [(i, b) for i, b in enumerate(self.boundaries) if isinstance(b, FixedBoundary)]

    def hasPassiveScalar(self):
        return self.passiveScalar is not None


class Domain:
    def __init__(self, dims, blocks, dtype=torch.float64):
        self._dims = dims
        self._blocks = blocks
        self._dtype = dtype
        for b in blocks:
            for bnd in b.boundaries:
                if isinstance(bnd, FixedBoundary):
                    bnd._parent = self

    def getSpatialDims(self):
        return self._dims

    def getBlocks(self):
        return list(self._blocks)

    def getNumBlocks(self):
        return len(self._blocks)

    def getBlock(self, i):
        return self._blocks[i]

    def getDtype(self):
        return self._dtype

    def getDevice(self):
        return torch.device("cpu")


def stub_module():
    m = types.ModuleType("PISOtorch")
    m.FixedBoundary = FixedBoundary
    m.VaryingDirichletBoundary = VaryingDirichletBoundary
    m.StaticDirichletBoundary = StaticDirichletBoundary
    m.BoundaryConditionType = BoundaryConditionType
    m.Domain = Domain
    return m


# ------------------------------------------------------------------ cases as arrays

def _t(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64)


def build_case(arrs):
    """Stand-in domain from a case's arrays (see tests/golden/make_ref_outflow_fixtures.py):
    dims, block velocities "b<i>_velocity" / scalars "b<i>_scalar", per fixed face "f<i>_<face>_velocity",
    "..._transform", "..._scalar"; "outflow" [(block, face)], "velm" ([1,D] or a list "velm<k>"), "dt"."""
    dims = int(arrs["dims"])
    nb = int(arrs["num_blocks"])
    blocks = []
    for i in range(nb):
        sc = arrs.get("b%d_scalar" % i)
        blk = Block(_t(arrs["b%d_velocity" % i]), None if sc is None else _t(sc))
        zyx = list(blk.velocity.shape[2:])
        for f in range(2 * dims):
            key = "f%d_%d_velocity" % (i, f)
            if key not in arrs:
                blk.boundaries.append(_Other())
                continue
            shape = list(zyx)
            shape[dims - 1 - (f >> 1)] = 1
            tr = arrs.get("f%d_%d_transform" % (i, f))
            fsc = arrs.get("f%d_%d_scalar" % (i, f))
            blk.boundaries.append(FixedBoundary(dims, f, shape, _t(arrs[key]), None if tr is None else _t(tr),
                                                None if fsc is None else _t(fsc)))
        blocks.append(blk)
    dom = Domain(dims, blocks)
    outflow = [tuple(int(v) for v in bf) for bf in np.asarray(arrs["outflow"]).reshape(-1, 2)]
    bounds = [blocks[b].boundaries[f] for b, f in outflow]
    if "velm" in arrs:
        velm = _t(arrs["velm"])
    else:
        velm = [_t(arrs["velm%d" % k]) for k in range(len(outflow))]
    return dom, bounds, velm, _t(np.asarray([float(arrs["dt"])]))


def outputs(dom, arrs):
    """Every fixed face's velocity (and scalar) after the update, keyed like the inputs."""
    out = {}
    for i, blk in enumerate(dom.getBlocks()):
        for f, bnd in enumerate(blk.boundaries):
            if isinstance(bnd, FixedBoundary):
                out["out_f%d_%d_velocity" % (i, f)] = bnd.velocity.numpy()
                if bnd.passiveScalar is not None:
                    out["out_f%d_%d_scalar" % (i, f)] = bnd.passiveScalar.numpy()
    return out
