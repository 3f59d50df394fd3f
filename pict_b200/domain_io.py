"""Domain checkpoints: a domain's structure as JSON plus its tensors as one NPZ archive.

The file pair ``<path>.json`` / ``<path>.npz`` is the format of the reference's ``save_domain`` /
``load_domain`` (lib/util/domain_io.py:44-235), so that checkpoints move between the two in both
directions:

* the JSON holds the domain (``name``, ``spatialDims``, ``passiveScalarChannels``), one entry per
  block (``name``, field references, ``boundaries`` per face) and ``data_info`` (shape, dtype and device
  of every stored tensor);
* a field reference is the string index of a tensor in the NPZ (keys ``"0"``, ``"1"``, ...); a tensor
  used several times (a shared static boundary velocity, say) is stored once;
* a fixed face stores ``velocityType``, its velocity, and with passive scalars ``passiveScalarType``
  (one name per stored type) and the scalar; a connected face stores the other block's index and the
  connection ``axes``; a periodic face only its type.  Blocks with vertex coordinates store those (the
  transforms follow from them), otherwise their transforms.

Loading builds the domain through the public API (CreateBlock, CloseBoundary, ConnectBlock,
MakePeriodic) and does not call PrepareSolve, as the reference leaves that to the caller.
"""
from __future__ import annotations

import json
import warnings

import numpy as np
import torch

from . import PISOtorch

_FACES = ["-x", "+x", "-y", "+y", "-z", "+z"]


def _dtype_name(dtype):
    if dtype == torch.float32:
        return "float32"
    if dtype == torch.float64:
        return "float64"
    raise TypeError("Unsupported dtype.")


def _bc_name(t):
    t = PISOtorch.BoundaryConditionType(t)
    return "DIRICHLET" if t == PISOtorch.BoundaryConditionType.DIRICHLET else "NEUMANN"


def _bc_type(name):
    if name == "DIRICHLET":
        return PISOtorch.BoundaryConditionType.DIRICHLET
    if name == "NEUMANN":
        return PISOtorch.BoundaryConditionType.NEUMANN
    raise TypeError("Unsupported boundary condition type.")


class _Store:
    """Tensors in first-use order, each stored once (identity, not value)."""

    def __init__(self):
        self.tensors = []

    def ref(self, t):
        for i, s in enumerate(self.tensors):
            if s is t:
                return str(i)
        self.tensors.append(t)
        return str(len(self.tensors) - 1)


def save_domain(domain, path):
    """Write ``<path>.json`` and ``<path>.npz`` (path without extension)."""
    store = _Store()
    blocks = domain.getBlocks()
    d = {"name": domain.name, "spatialDims": domain.getSpatialDims(), "viscosity": store.ref(domain.viscosity),
         "passiveScalarChannels": domain.getPassiveScalarChannels()}
    if domain.hasPassiveScalarViscosity():
        d["passiveScalarViscosity"] = store.ref(domain.passiveScalarViscosity)
    d["blocks"] = []
    for block in blocks:
        b = {"name": block.name}
        if block.hasViscosity():
            b["viscosity"] = store.ref(block.viscosity)
        b["velocity"] = store.ref(block.velocity)
        b["pressure"] = store.ref(block.pressure)
        if block.hasPassiveScalar() and block.passiveScalar is not None:
            b["scalar"] = store.ref(block.passiveScalar)
        if block.hasVelocitySource():
            b["velocitySource"] = store.ref(block.velocitySource)
        if block.hasVertexCoordinates():
            b["vertexCoordinates"] = store.ref(block.vertexCoordinates)
        elif block.hasTransform():
            b["transform"] = store.ref(block.transform)
            if block.hasFaceTransform():
                b["faceTransform"] = store.ref(block.faceTransform)
        faces = []
        for f in range(2 * block.getSpatialDims()):
            bnd = block.getBoundary(f)
            e = {}
            if isinstance(bnd, PISOtorch.FixedBoundary):
                e["type"] = "FIXED"
                e["velocityType"] = _bc_name(bnd.velocityType)
                e["velocity"] = store.ref(bnd.velocity)
                if bnd.hasPassiveScalar():
                    e["passiveScalarType"] = [_bc_name(t) for t in (bnd.passiveScalarTypes or [bnd.velocityType])]
                    e["scalar"] = store.ref(bnd.passiveScalar)
                if bnd.hasTransform():
                    e["transform"] = store.ref(bnd.transform)
            elif isinstance(bnd, PISOtorch.ConnectedBoundary):
                e["type"] = "CONNECTED"
                e["connectedBlock"] = blocks.index(bnd.getConnectedBlock())
                e["axes"] = [int(a) for a in bnd.axes]
            elif isinstance(bnd, PISOtorch.PeriodicBoundary):
                e["type"] = "PERIODIC"
            else:
                raise TypeError("Unknown boundary type.")
            faces.append(e)
        b["boundaries"] = faces
        d["blocks"].append(b)
    d["data_info"] = {str(i): {"shape": list(t.shape), "dtype": _dtype_name(t.dtype), "device": str(t.device.type)}
                      for i, t in enumerate(store.tensors)}
    np.savez_compressed(path + ".npz", **{str(i): t.detach().cpu().numpy() for i, t in enumerate(store.tensors)})
    with open(path + ".json", "w") as fh:
        json.dump(d, fh)


def load_domain(path, dtype=None, device=None, with_scalar=True):
    """Read a domain written by ``save_domain`` (or by the reference).  ``dtype`` / ``device`` default to
    float32 / the current CUDA device; ``with_scalar=False`` drops the passive scalars."""
    with open(path + ".json", "r") as fh:
        d = json.load(fh)
    dtype = torch.float32 if dtype is None else dtype
    device = torch.device("cuda") if device is None else torch.device(device)
    with np.load(path + ".npz") as npz:
        data = [torch.tensor(npz[str(i)]).to(device=device, dtype=dtype).contiguous() for i in range(len(npz.files))]

    def get(e, key):
        return data[int(e[key])] if key in e else None

    channels = d.get("passiveScalarChannels", 1) if with_scalar else 0
    # the domain viscosity is a host tensor; every other field lives on the device
    viscosity = get(d, "viscosity").cpu()
    domain = PISOtorch.Domain(d["spatialDims"], viscosity, d["name"], dtype=dtype, device=device,
                              passiveScalarChannels=channels,
                              scalarViscosity=get(d, "passiveScalarViscosity") if with_scalar else None)
    for b in d["blocks"]:
        block = domain.CreateBlock(get(b, "velocity"), get(b, "pressure"), get(b, "scalar") if with_scalar else None,
                                   vertexCoordinates=get(b, "vertexCoordinates"), name=b["name"])
        if "viscosity" in b:
            block.setViscosity(get(b, "viscosity"))
        if with_scalar and "passiveScalarViscosity" in b:
            warnings.warn("per-block passive scalar viscosity is not used by the scalar operators; ignored")
        if "velocitySource" in b:
            block.setVelocitySource(get(b, "velocitySource"))
        if "vertexCoordinates" not in b and "transform" in b:
            block.setTransform(get(b, "transform"), get(b, "faceTransform"))
    blocks = domain.getBlocks()
    for b, block in zip(d["blocks"], blocks):
        for f, e in enumerate(b["boundaries"]):
            kind = e["type"]
            if kind in ("DIRICHLET", "DIRICHLET_VARYING"):
                warnings.warn("%s boundaries are loaded as FixedBoundary." % kind)
                block.CloseBoundary(f, get(e, "velocity"), get(e, "scalar") if with_scalar else None)
            elif kind == "FIXED":
                has_scalar = with_scalar and "scalar" in e
                block.CloseBoundary(f, get(e, "velocity"), get(e, "scalar") if has_scalar else None)
                if has_scalar:
                    types = e["passiveScalarType"]
                    types = [_bc_type(t) for t in types] if isinstance(types, list) else _bc_type(types)
                    block.getBoundary(f).setPassiveScalarType(types)
            elif kind == "CONNECTED":
                block.ConnectBlock(_FACES[f], blocks[e["connectedBlock"]], *[_FACES[a] for a in e["axes"]])
            elif kind == "PERIODIC":
                block.MakePeriodic(f // 2)
            elif kind == "NEUMANN":
                raise NotImplementedError("NEUMANN boundaries")
            else:
                raise TypeError("Unknown boundary type: " + kind)
    return domain
