"""Drop-in host mirror of the reference's ``PISOtorch`` extension module.

Same class names, method names, argument names, defaults and error behaviour as
the reference's pybind11 module (extensions/PISOtorch.cpp:25-655, backed by
extensions/domain_structs.{h,cpp}), implemented as a thin Python layer over the
C ABI of ``libpict_b200.so`` (include/pict_b200.h).  Field memory stays in
torch tensors owned by Python; the native code receives raw device pointers in
a packed block table (the reference's "atlas", extensions/domain_structs.cpp:2992-3261),
re-packed by ``Domain.UpdateDomainData()`` exactly when the reference requires
it.

Differences in representation (not in results):

* ``Domain.C`` / ``Domain.P`` are :class:`StencilMatrix` objects: the system
  matrices are stored as per-cell stencil coefficients ``coef[K][N]``; the
  reference's CSR arrays ``value/index/row`` are materialised on demand in the
  reference's row layout (rows sorted by column).
* Linear solves run as persistent CUDA kernels; ``SolveLinear`` still returns
  one ``LinearSolverResultInfo`` per right-hand side.

Scope: the PISO path (orthogonal, and the non-orthogonal terms of ``nonOrthoFlags``) with fixed Dirichlet,
periodic and connected block boundaries, per-cell transforms, block/global
viscosity and velocity sources, in 2D and 3D, float32 and float64, with the gradients of all of it;
velocity correctors 0/1 (finite differences), 4, 5 and 6 (finite volumes); passive scalar transport
with its raw gradient operators.  ``SolveLinear``'s CG takes every ``ConvergenceCriterion``, residual
resets, ``returnBestResult`` and ``matrixRankDeficient``; BiCGStab takes every criterion too, unpreconditioned
or preconditioned (``BiCGPreconditioner``).  Face-transform pressure assembly raises ``NotImplementedError``.
"""
from __future__ import annotations

import ctypes
import enum
import warnings
import weakref
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._lib import BlockDesc, DomainDesc, Face, SolveInfo, SolveParams, check

# ------------------------------------------------------------------------------------------------
# enums and small types (extensions/PISOtorch.cpp:30-58, 544-558)
# ------------------------------------------------------------------------------------------------


class BoundaryType(enum.IntEnum):
    DIRICHLET = 0
    DIRICHLET_VARYING = 1
    NEUMANN = 10
    FIXED = 30
    CONNECTED = 20
    PERIODIC = 21


class BoundaryConditionType(enum.IntEnum):
    DIRICHLET = 0
    NEUMANN = 1


class ConvergenceCriterion(enum.IntEnum):
    NORM2 = 0
    NORM2_NORMALIZED = 1
    ABS_SUM = 2
    ABS_MEAN = 3
    ABS_MAX = 4


class BiCGPreconditioner(enum.IntEnum):
    """Preconditioner of SolveLinear(useBiCG=True, BiCGwithPreconditioner=True); no counterpart in the
    reference's module, which has one fixed behaviour.  AS_REFERENCE (default): the operator the
    reference's build applies, M = T T with T the lower triangle of the matrix including its diagonal
    (extensions/bicgstab_solver_kernel.cu:150-208 sets up csrilu02 factors, but its triangular solves apply
    the unfactorised lower triangle twice), so solves, iteration counts and reports equal the reference's.
    ILU0: M = L U of the zero-fill incomplete LU factors, the preconditioner the reference's set-up
    intends (fewer iterations)."""
    AS_REFERENCE = 0
    ILU0 = 1


_bicg_preconditioner = BiCGPreconditioner.AS_REFERENCE


def SetBiCGPreconditioner(kind):
    """Select the preconditioner of preconditioned BiCGStab solves (BiCGPreconditioner); returns the
    previous one."""
    global _bicg_preconditioner
    prev = _bicg_preconditioner
    _bicg_preconditioner = BiCGPreconditioner(kind)
    return prev


def GetBiCGPreconditioner():
    return _bicg_preconditioner


class NonOrthoFlags(enum.IntFlag):
    """Bits of the ``nonOrthoFlags`` argument (extensions/PISO_multiblock_cuda.h:9-13).  The reference
    declares a pybind11 enum of this name but leaves it commented out (extensions/PISOtorch.cpp:491-501),
    so its callers pass plain ints; these members are the same ints, and the operators take either."""
    NONE = 0
    DIRECT_MATRIX = 1
    DIRECT_RHS = 2
    DIAGONAL_MATRIX = 4
    DIAGONAL_RHS = 8
    CENTER_MATRIX = 16


# pybind11 export_values(): enum members are also module attributes
DIRICHLET_VARYING = BoundaryType.DIRICHLET_VARYING
FIXED = BoundaryType.FIXED
CONNECTED = BoundaryType.CONNECTED
PERIODIC = BoundaryType.PERIODIC
DIRICHLET = BoundaryConditionType.DIRICHLET
NEUMANN = BoundaryConditionType.NEUMANN
NORM2 = ConvergenceCriterion.NORM2
NORM2_NORMALIZED = ConvergenceCriterion.NORM2_NORMALIZED
ABS_SUM = ConvergenceCriterion.ABS_SUM
ABS_MEAN = ConvergenceCriterion.ABS_MEAN
ABS_MAX = ConvergenceCriterion.ABS_MAX


class Int4:
    """I4 (extensions/domain_structs_gpu.h:120-125)."""

    def __init__(self, x=0, y=0, z=0, w=0):
        self.x, self.y, self.z, self.w = int(x), int(y), int(z), int(w)

    def __getitem__(self, i):
        if 0 <= i < 4:
            return (self.x, self.y, self.z, self.w)[i]
        raise IndexError(i)

    def __len__(self):
        return 4

    def __str__(self):
        return "I4(%d,%d,%d,%d)" % (self.x, self.y, self.z, self.w)

    __repr__ = __str__


class LinearSolverResultInfo:
    """extensions/bicgstab_solver.h:20-34."""

    def __init__(self, finalResidual=0.0, usedIterations=-1, converged=False, isFiniteResidual=True):
        self.finalResidual = float(finalResidual)
        self.usedIterations = int(usedIterations)
        self.converged = bool(converged)
        self.isFiniteResidual = bool(isFiniteResidual)

    def __str__(self):
        return "LinearSolverResultInfo(finalResidual=%g, usedIterations=%d, converged=%d, isFiniteResidual=%d)" % (
            self.finalResidual, self.usedIterations, self.converged, self.isFiniteResidual)

    __repr__ = __str__


FACE_NAMES = ["-x", "+x", "-y", "+y", "-z", "+z"]
AXIS_NAMES = ["x", "y", "z"]


def _face_index(face) -> int:
    """BoundarySideToIndex, extensions/domain_structs.cpp:134-155."""
    if isinstance(face, str):
        if face not in FACE_NAMES:
            raise ValueError("Invalid boundary side '%s'" % face)
        return FACE_NAMES.index(face)
    return int(face)


def _axis_index(axis) -> int:
    if isinstance(axis, str):
        if axis not in AXIS_NAMES:
            raise ValueError("Invalid axis '%s'" % axis)
        return AXIS_NAMES.index(axis)
    return int(axis)


def _check(cond, msg):
    if not cond:
        raise RuntimeError(msg)


def _dtype_code(dtype):
    if dtype == torch.float32:
        return _lib.PICT_F32
    if dtype == torch.float64:
        return _lib.PICT_F64
    raise TypeError("dtype must be torch.float32 or torch.float64")


def _stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


TILE_CELLS = 1024  # cells per Krylov work tile (1..2048; the kernels hold at most 2048)


def build_tiles(host_blocks, num_blocks, num_sims, device, tile_cells=TILE_CELLS):
    """Krylov work tiles of a block table (pict_build_tiles): returns (tiles [T,4] int32, sim_tiles [S+1])."""
    lib = _lib.load()
    cnt = ctypes.c_int32(0)
    sim_tiles = torch.empty(num_sims + 1, dtype=torch.int32)
    lib.pict_build_tiles(host_blocks, num_blocks, num_sims, tile_cells, None, 0, sim_tiles.data_ptr(), ctypes.byref(cnt))
    tiles = torch.empty((max(cnt.value, 1), 4), dtype=torch.int32)
    check(lib.pict_build_tiles(host_blocks, num_blocks, num_sims, tile_cells, tiles.data_ptr(), cnt.value,
                               sim_tiles.data_ptr(), ctypes.byref(cnt)), "build_tiles")
    return tiles[:cnt.value].to(device), sim_tiles.to(device), cnt.value


def _transform_size(dims):
    return 2 * dims * dims + 1


def _as_scalar(v, default=None):
    if v is None:
        return default
    if isinstance(v, torch.Tensor):
        return v.reshape(-1)[0].item()
    return v


# ------------------------------------------------------------------------------------------------
# CSR / stencil matrices (extensions/domain_structs.h:54-90)
# ------------------------------------------------------------------------------------------------


class CSRmatrix:
    """Generic CSR matrix container with the reference's interface."""

    def __init__(self, value, index=None, row=None, device=None):
        if isinstance(value, torch.Tensor):
            self.value = value
            self.index = index
            self.row = row
        else:  # CSRmatrix(numValues, numRows, dtype, device)
            numValues, numRows, dtype = int(value), int(index), row
            self.value = torch.zeros(numValues, dtype=dtype, device=device)
            self.index = torch.zeros(numValues, dtype=torch.int32, device=device)
            self.row = torch.zeros(numRows + 1, dtype=torch.int32, device=device)
        self._changed = False

    def setValue(self, tensor):
        _check(tensor.dim() == 1 and tensor.size(0) == self.getSize(), "CSR value size must not change.")
        self.value = tensor
        self._changed = True

    def CreateValue(self):
        self.setValue(torch.zeros_like(self.value))

    def getDevice(self):
        return self.value.device

    def getDtype(self):
        return self.value.dtype

    def copy(self):
        return CSRmatrix(self.value, self.index, self.row)

    def clone(self):
        return CSRmatrix(self.value.clone(), self.index, self.row)

    def detach(self):
        self.value = self.value.detach()

    def WithZeroValue(self):
        return CSRmatrix(torch.zeros_like(self.value), self.index, self.row)

    def toType(self, dtype):
        return CSRmatrix(self.value.to(dtype), self.index, self.row)

    def getSize(self):
        return self.value.size(0)

    def getRows(self):
        return self.row.size(0) - 1

    def IsTensorChanged(self):
        return self._changed

    def __str__(self):
        return "CSRmatrix(rows=%d, nnz=%d)" % (self.getRows(), self.getSize())


class StencilMatrix(CSRmatrix):
    """System matrix of a prepared domain stored as stencil coefficients ``coef[K][N]``.

    ``value``/``index``/``row`` give the reference CSR layout (computed on demand);
    assigning ``value`` (``setValue``) converts back to stencil storage.
    """

    def __init__(self, domain, coef: torch.Tensor):
        self._domain_ref = weakref.ref(domain)
        self.coef = coef
        self._changed = False

    # -- CSR views --
    def _domain(self):
        d = self._domain_ref()
        if d is None:
            raise RuntimeError("StencilMatrix: the domain is expired.")
        return d

    def _csr(self):
        d = self._domain()
        row, index = d._csr_structure()
        value = torch.empty(index.numel(), dtype=self.coef.dtype, device=self.coef.device)
        check(_lib.load().pict_stencil_to_csr(ctypes.byref(d._desc), _ptr(self.coef.contiguous()), _ptr(row),
                                              _ptr(value), _ptr(index), _stream_ptr()), "stencil_to_csr")
        return value, index, row

    @property
    def value(self):
        return self._csr()[0]

    @property
    def index(self):
        return self._domain()._csr_structure()[1]

    @property
    def row(self):
        return self._domain()._csr_structure()[0]

    def setValue(self, tensor):
        d = self._domain()
        row, index = d._csr_structure()
        _check(tensor.dim() == 1 and tensor.size(0) == index.numel(), "CSR value size must not change.")
        coef = torch.empty_like(self.coef)
        check(_lib.load().pict_csr_to_stencil(ctypes.byref(d._desc), _ptr(tensor.contiguous()), _ptr(row),
                                              _ptr(index), _ptr(coef), _stream_ptr()), "csr_to_stencil")
        self.coef = coef
        self._changed = True

    def setCoef(self, coef):
        _check(coef.shape == self.coef.shape, "stencil shape must not change.")
        self.coef = coef
        self._changed = True

    def CreateValue(self):
        self.setCoef(torch.zeros_like(self.coef))

    def getDevice(self):
        return self.coef.device

    def getDtype(self):
        return self.coef.dtype

    def getSize(self):
        return self._domain()._csr_structure()[1].numel()

    def getRows(self):
        return self.coef.size(1)

    def copy(self):
        return StencilMatrix(self._domain(), self.coef)

    def clone(self):
        return StencilMatrix(self._domain(), self.coef.clone())

    def detach(self):
        self.coef = self.coef.detach()

    def WithZeroValue(self):
        return StencilMatrix(self._domain(), torch.zeros_like(self.coef))

    def toType(self, dtype):
        return StencilMatrix(self._domain(), self.coef.to(dtype))

    def __str__(self):
        return "StencilMatrix(K=%d, rows=%d)" % (self.coef.size(0), self.coef.size(1))


# ------------------------------------------------------------------------------------------------
# boundaries (extensions/domain_structs.h:92-375)
# ------------------------------------------------------------------------------------------------


class Boundary:
    def __init__(self, btype, domain):
        self.type = btype
        self._domain_ref = weakref.ref(domain)
        self._changed = True

    def getParentDomain(self):
        d = self._domain_ref()
        _check(d is not None, "Parent domain expired.")
        return d

    def getSpatialDims(self):
        return self.getParentDomain().getSpatialDims()

    def getDtype(self):
        return self.getParentDomain().getDtype()

    def getDevice(self):
        return self.getParentDomain().getDevice()

    def IsTensorChanged(self):
        return self._changed

    def __str__(self):
        return "%s()" % self.type.name


class PeriodicBoundary(Boundary):
    def __init__(self, domain):
        super().__init__(BoundaryType.PERIODIC, domain)

    def Copy(self):
        return PeriodicBoundary(self.getParentDomain())

    Clone = Copy


class ConnectedBoundary(Boundary):
    """extensions/domain_structs.h:329-352; ``axes`` starts with the connected face of the other block."""

    def __init__(self, block, axes, domain):
        super().__init__(BoundaryType.CONNECTED, domain)
        self._block_ref = weakref.ref(block)
        self.axes = list(axes)

    def getConnectedBlock(self):
        b = self._block_ref()
        _check(b is not None, "ConnectedBlock is expired.")
        return b

    def getConnectedFace(self):
        return self.axes[0] >> 1

    def getConnectionAxis(self, axis):
        return self.axes[axis] >> 1

    def getConnectionAxisDirection(self, axis):
        return self.axes[axis] & 1

    def __str__(self):
        s = 'CONNECTED(to="%s", face=%s' % (self.getConnectedBlock().name, FACE_NAMES[self.axes[0]])
        for k in range(1, len(self.axes)):
            s += ", axis%d=%s" % (k, FACE_NAMES[self.axes[k]])
        return s + ")"


class FixedBoundary(Boundary):
    """Prescribed boundary: Dirichlet velocity, 0-Neumann pressure (extensions/domain_structs.cpp:304-796)."""

    def __init__(self, domain, velocity=None, velocityType=BoundaryConditionType.DIRICHLET, passiveScalar=None,
                 transform=None):
        super().__init__(BoundaryType.FIXED, domain)
        self._size = None  # x,y,z with 1 along the face axis
        self._axis = -1
        self.velocityGrad = torch.empty(0)
        self.passiveScalar = None
        self.passiveScalarGrad = None
        self.passiveScalarTypes = None
        self.transform = None
        dims = domain.getSpatialDims()
        if velocity is not None and velocity.dim() > 2:
            self._setSizeFromTensor(velocity, True)
        elif passiveScalar is not None and passiveScalar.dim() > 2:
            self._setSizeFromTensor(passiveScalar, True)
        elif transform is not None:
            self._setSizeFromTensor(transform, False)
        elif velocity is not None:
            _check(velocity.dim() > 1, "Velocity must be 1-3D and either static (shape NC) or varying (shape NCDHW).")
        elif passiveScalar is not None:
            raise RuntimeError("Can't create FixedBoundary from static passive scalar alone.")
        if velocity is not None:
            self.setVelocity(velocity)
        else:
            self.CreateVelocity(True)
        self.setVelocityType(velocityType)
        if passiveScalar is not None:
            self.setPassiveScalar(passiveScalar)
        elif domain.hasPassiveScalar():
            self.CreatePassiveScalar(True)
        if transform is not None:
            self.setTransform(transform)

    # -- size --
    def _setSizeFromTensor(self, t, channelsFirst):
        dims = self.getSpatialDims()
        _check(t.dim() == dims + 2, "Invalid tensor for boundary shape.")
        off = 1 if channelsFirst else 0
        size = [t.size(dims + off - d) for d in range(dims)]
        self._setSize(size)

    def _setSize(self, size):
        _check(self._size is None, "Internal Error: FixedBoundary already has a size set.")
        dims = self.getSpatialDims()
        has1 = False
        for d in range(dims):
            if size[d] == 1:
                _check(not has1, "Invalid boundary shape: only one dimension must be 1.")
                has1 = True
                self._axis = d
            else:
                _check(size[d] > 2, "Invalid boundary shape: grid size must be at least 3.")
        _check(has1, "Invalid boundary shape: one dimension must be 1.")
        self._size = list(size) + [1] * (3 - dims)

    def hasSize(self):
        return self._size is not None

    def getSizes(self):
        dims = self.getSpatialDims()
        s = self._size if self._size is not None else [1, 1, 1]
        return Int4(s[0], s[1], s[2], dims)

    def getStrides(self):
        s = self.getSizes()
        return Int4(1, s.x, s.x * s.y, s.x * s.y * s.z)

    def _face_cells(self):
        s = self.getSizes()
        return s.x * s.y * s.z

    # -- velocity --
    @property
    def velocity(self):
        return self._velocity

    @property
    def velocityType(self):
        return self._velocityType

    @property
    def isVelocityStatic(self):
        return self._velocityStatic

    def setVelocity(self, t):
        dims = self.getSpatialDims()
        _check(t.is_cuda, "velocity must be a CUDA tensor")
        _check(t.is_contiguous(), "velocity must be contiguous")
        _check(t.size(0) == 1, "Batches are not yet supported (velocity).")
        _check(t.size(1) == dims, "Velocity channels are invalid. Velocity must be %dD and either static (shape NC) or varying (shape NCDHW)." % dims)
        _check(t.dim() == 2 or t.dim() == 2 + dims,
               "Velocity spatial dimensions are invalid. Velocity must be %dD and either static (shape NC) or varying (shape NCDHW)." % dims)
        _check(t.dtype == self.getDtype(), "Velocity dtype must match domain.")
        static = t.dim() == 2
        if not static and self.hasSize():
            s = self.getSizes()
            _check(all(t.size(dims + 1 - d) == [s.x, s.y, s.z][d] for d in range(dims)),
                   "New velocity spatial dimensions must match existing fields.")
        if self.velocityGrad is not None and self.velocityGrad.numel() > 0:
            _check(self.velocityGrad.dim() == t.dim(), "New velocity does not match existing gradient tensor.")
        self._velocity = t
        self._velocityStatic = static
        self._changed = True

    def setVelocityType(self, velocityType):
        _check(velocityType == BoundaryConditionType.DIRICHLET,
               "Invalid velocity boundary type: Currently only Dirichlet boundaries are supported")
        self._velocityType = BoundaryConditionType(velocityType)

    def CreateVelocity(self, createStatic):
        dims = self.getSpatialDims()
        if createStatic:
            v = torch.zeros((1, dims), dtype=self.getDtype(), device=self.getDevice())
        else:
            _check(self.hasSize(), "FixedBoundary is missing size to create a varying velocity.")
            s = self.getSizes()
            v = torch.zeros([1, dims] + [[s.x, s.y, s.z][dims - 1 - d] for d in range(dims)], dtype=self.getDtype(),
                            device=self.getDevice())
        self.setVelocity(v)

    def getVelocityVarying(self, size=None):
        if self._velocityStatic:
            _check(self.hasSize() or size is not None,
                   "FixedBoundary has no fields with spatial dimensions to infer varying velocity shape.")
            s = self.getSizes() if self.hasSize() else size
            dims = self.getSpatialDims()
            shape = [[s[0], s[1], s[2]][dims - 1 - d] for d in range(dims)]
            v = self._velocity.reshape([1, dims] + [1] * dims)
            return v.repeat([1, 1] + shape).clone().contiguous()
        return self._velocity

    def makeVelocityVarying(self, size=None):
        if self._velocityStatic:
            self.setVelocity(self.getVelocityVarying(size))

    def getVelocity(self, computational):
        _check(self.hasSize(), "FixedBoundary has no size set.")
        v = self.getVelocityVarying(None)
        if computational and self.hasTransform():
            return TransformVectors(v, self.transform, True)
        return v

    def GetFluxes(self):
        """Boundary-normal fluxes det * (Minv u)_axis (extensions/domain_structs.cpp:527-542)."""
        _check(self.hasSize(), "FixedBoundary has no size set.")
        v = self.getVelocityVarying(None)
        if self.hasTransform():
            det = self.transform[..., -1]
            f = det.unsqueeze(1) * TransformVectors(v, self.transform, True)
        else:
            f = v
        return f[:, self._axis:self._axis + 1].clone()

    def setVelocityGrad(self, t):
        _check(t.shape == self._velocity.shape, "FixedBoundary.velocity_grad must match velocity.")
        self.velocityGrad = t
        self._changed = True

    def CreateVelocityGrad(self):
        self.setVelocityGrad(torch.zeros_like(self._velocity))

    def setPassiveScalarGrad(self, t):
        _check(self.passiveScalar is not None, "FixedBoundary does not have a passive scalar.")
        _check(t.shape == self.passiveScalar.shape, "FixedBoundary passive scalar gradient must match the passive scalar.")
        self.passiveScalarGrad = t
        self._changed = True

    def CreatePassiveScalarGrad(self):
        if self.passiveScalar is not None:
            self.setPassiveScalarGrad(torch.zeros_like(self.passiveScalar))

    # -- passive scalar --
    def setPassiveScalar(self, t):
        dims = self.getSpatialDims()
        _check(t.is_cuda, "passiveScalar must be a CUDA tensor")
        _check(t.size(0) == 1, "Batches are not yet supported (passiveScalar).")
        _check(t.size(1) == self.getPassiveScalarChannels(), "Passive scalar channels must match domain.")
        _check(t.dim() == 2 or t.dim() == 2 + dims, "Passive Scalar spatial dimensions are invalid. Passive Scalar must be "
               "1-3D and either static (shape NC) or varying (shape NCDHW). Varying dimensionality must match velocity.")
        _check(t.dtype == self.getDtype(), "Passive Scalar dtype must match domain.")
        self.passiveScalar = t
        if self.passiveScalarTypes is None:
            self.passiveScalarTypes = [self._velocityType]
        self._changed = True

    def CreatePassiveScalar(self, createStatic):
        ch = self.getParentDomain().getPassiveScalarChannels()
        if createStatic:
            shape = [1, ch]
        else:
            _check(self.hasSize(), "FixedBoundary is missing size to create a varying PassiveScalar.")
            shape = [1, ch] + [self._size[d] for d in reversed(range(self.getSpatialDims()))]
        self.setPassiveScalar(torch.zeros(shape, dtype=self.getDtype(), device=self.getDevice()))

    def hasPassiveScalar(self):
        return self.passiveScalar is not None

    def getPassiveScalarChannels(self):
        return self.getParentDomain().getPassiveScalarChannels()

    def isPassiveScalarStatic(self):
        return self.passiveScalar is None or self.passiveScalar.dim() == 2

    def isPassiveScalarBoundaryTypeStatic(self):
        return self.passiveScalarTypes is None or len(set(self.passiveScalarTypes)) < 2

    def _scalar_neumann_mask(self, channels):
        """Bit c set where passive scalar channel c has a Neumann boundary (one type for all channels when
        a single type is given)."""
        types = self.passiveScalarTypes or [self._velocityType]
        mask = 0
        for c in range(channels):
            if BoundaryConditionType(types[c] if len(types) > 1 else types[0]) == BoundaryConditionType.NEUMANN:
                mask |= 1 << c
        return mask

    def setPassiveScalarType(self, t):
        """One type for every channel, or a list with one type per channel (FixedBoundary::setPassiveScalarType,
        extensions/domain_structs.cpp:622-643)."""
        _check(self.hasPassiveScalar(), "FixedBoundary has not passive scalar.")
        types = list(t) if isinstance(t, (list, tuple)) else [t]
        _check(len(types) == 1 or len(types) == self.getPassiveScalarChannels(),
               "Passive scalar boundary conditions must be static or match channels.")
        self.passiveScalarTypes = [BoundaryConditionType(x) for x in types]
        self._changed = True

    # -- transform --
    def hasTransform(self):
        return self.transform is not None

    def setTransform(self, t):
        dims = self.getSpatialDims()
        _check(t.is_cuda and t.is_contiguous(), "transform must be a contiguous CUDA tensor")
        _check(t.size(0) == 1, "Batches are not yet supported (transform).")
        _check(t.dim() == 2 + dims, "Transform spatial dimensions are invalid. Transform must be 1-3D and have shape NDHWT. Dimensionality must match velocity.")
        if self.hasSize():
            s = self.getSizes()
            _check(all(t.size(dims - d) == [s.x, s.y, s.z][d] for d in range(dims)),
                   "Transform spatial dimensions must match existing fields.")
        else:
            self._setSizeFromTensor(t, False)
        _check(t.size(-1) == _transform_size(dims), "Transform channels must match spatial dimensions")
        self.transform = t
        self._changed = True

    def clearTransform(self):
        if self.transform is not None:
            self.transform = None
            self._changed = True

    def DetachFwd(self):
        self._velocity = self._velocity.detach()
        if self.transform is not None:
            self.transform = self.transform.detach()

    def DetachGrad(self):
        self.velocityGrad = self.velocityGrad.detach()

    def Detach(self):
        self.DetachFwd()
        self.DetachGrad()

    def Copy(self):
        return FixedBoundary(self.getParentDomain(), self._velocity, self._velocityType, self.passiveScalar, self.transform)

    def Clone(self):
        return FixedBoundary(self.getParentDomain(), self._velocity.clone(), self._velocityType,
                             None if self.passiveScalar is None else self.passiveScalar.clone(),
                             None if self.transform is None else self.transform.clone())

    def __str__(self):
        return "FIXED(%dD, size=%s, vStatic=%s, transform=%s)" % (
            self.getSpatialDims(), self.getSizes() if self.hasSize() else "?", self._velocityStatic, self.hasTransform())


# ------------------------------------------------------------------------------------------------
# blocks (extensions/domain_structs.h:354-540)
# ------------------------------------------------------------------------------------------------


class Block:
    def __init__(self, domain, velocity=None, pressure=None, passiveScalar=None, vertexCoordinates=None, name="Block",
                 size=None):
        self._domain_ref = weakref.ref(domain)
        self.name = name
        dims = domain.getSpatialDims()
        dtype, device = domain.getDtype(), domain.getDevice()
        if size is None:
            _check(velocity is not None or pressure is not None or passiveScalar is not None or vertexCoordinates is not None,
                   "At least one field (velocity, pressure, passiveScalar, vertexCoordinates) or the size must be given to create a block.")
        if velocity is not None:
            _check(velocity.is_cuda and velocity.is_contiguous(), "velocity must be a contiguous CUDA tensor")
            _check(velocity.dim() == dims + 2, "Velocity dimensionality must match domain. Layout should be NC<spatial-dims>, e.g. NCDHW for 3D.")
            _check(velocity.size(1) == dims, "The velocity channels must match the spatial dimensions.")
            _check(velocity.size(0) == 1, "Batches are not yet supported.")
            for d in range(2, velocity.dim()):
                _check(velocity.size(d) > 2, "all spatial dimensions must be at least 3.")
            _check(velocity.dtype == dtype, "Velocity dtype must match domain.")
            self.velocity = velocity
        else:
            if size is not None:
                zyx = [size[dims - 1 - d] for d in range(dims)]
            elif pressure is not None:
                zyx = list(pressure.shape[2:])
            elif passiveScalar is not None:
                zyx = list(passiveScalar.shape[2:])
            else:
                zyx = [s - 1 for s in vertexCoordinates.shape[2:]]
            _check(len(zyx) == dims, "Field dimensionality must match domain. Layout should be NC<spatial-dims>, e.g. NCDHW for 3D.")
            for s in zyx:
                _check(s > 2, "all spatial dimensions must be at least 3.")
            self.velocity = torch.zeros([1, dims] + zyx, dtype=dtype, device=device)
        self.boundaries = [PeriodicBoundary(domain) for _ in range(2 * dims)]
        self.pressure = None
        if pressure is not None:
            self.setPressure(pressure)
        else:
            self.CreatePressure()
        self.passiveScalar = None
        if passiveScalar is not None:
            self.setPassiveScalar(passiveScalar)
        elif domain.hasPassiveScalar():
            self.CreatePassiveScalar()
        self.viscosity = None
        self.velocitySource = None
        self.isVelocitySourceStatic = False
        self.vertexCoordinates = None
        self.transform = None
        self.faceTransform = None
        self.velocityGrad = torch.empty(0)
        self.pressureGrad = torch.empty(0)
        self.viscosityGrad = None
        self.velocitySourceGrad = None
        self.passiveScalarGrad = torch.empty(0)
        self.globalOffset = 0
        self.csrOffset = 0
        self._changed = True
        if vertexCoordinates is not None:
            self.setVertexCoordinates(vertexCoordinates)

    def getParentDomain(self):
        d = self._domain_ref()
        _check(d is not None, "Parent domain expired.")
        return d

    def getSpatialDims(self):
        return self.getParentDomain().getSpatialDims()

    def getDtype(self):
        return self.velocity.dtype

    def getDevice(self):
        return self.velocity.device

    def getDim(self, dim):
        return self.velocity.size(dim)

    def getAxis(self, dim):
        _check(0 <= dim < self.getSpatialDims(), "Axis index must be within spatial dimensions")
        return self.velocity.size(self.velocity.dim() - 1 - dim)

    def getSizes(self):
        dims = self.getSpatialDims()
        s = [self.getAxis(d) for d in range(dims)] + [1] * (3 - dims)
        return Int4(s[0], s[1], s[2], dims)

    def getStrides(self):
        s = self.getSizes()
        return Int4(1, s.x, s.x * s.y, s.x * s.y * s.z)

    def _ncells(self):
        return self.getStrides().w

    def _check_tensor(self, t, channels, allow_static, name):
        dims = self.getSpatialDims()
        _check(t.is_cuda, "%s must be a CUDA tensor" % name)
        _check(t.is_contiguous(), "%s must be contiguous" % name)
        _check(t.dtype == self.getDtype(), "%s dtype must match the domain." % name)
        _check(t.size(0) == 1, "%s: batches are not yet supported." % name)
        _check(t.size(1) == channels, "%s: channel dimension must be %d." % (name, channels))
        if allow_static and t.dim() == 2:
            return
        _check(t.dim() == dims + 2, "%s: spatial dimensions must match the block." % name)
        _check(list(t.shape[2:]) == list(self.velocity.shape[2:]), "%s: spatial size must match the block." % name)

    # -- fields --
    def setVelocity(self, v):
        self._check_tensor(v, self.getSpatialDims(), False, "Velocity")
        self.velocity = v
        self._changed = True

    def getVelocity(self, computational):
        if computational:
            _check(self.hasTransform(), "Coordinates or Transformations are required to compute computational velocities.")
            return TransformVectors(self.velocity, self.transform, True)
        return self.velocity

    def CreateVelocity(self):
        self.setVelocity(torch.zeros_like(self.velocity))

    def setPressure(self, p):
        self._check_tensor(p, 1, False, "Pressure")
        self.pressure = p
        self._changed = True

    def CreatePressure(self):
        self.pressure = torch.zeros([1, 1] + list(self.velocity.shape[2:]), dtype=self.getDtype(), device=self.getDevice())
        self._changed = True

    def setPassiveScalar(self, s):
        ch = self.getPassiveScalarChannels()
        _check(ch > 0, "Passive scalars are not active.")
        self._check_tensor(s, ch, False, "Passive Scalar")
        self.passiveScalar = s
        self._changed = True

    def CreatePassiveScalar(self):
        ch = self.getPassiveScalarChannels()
        _check(ch > 0, "Passive scalars are not active.")
        self.passiveScalar = torch.zeros([1, ch] + list(self.velocity.shape[2:]), dtype=self.getDtype(), device=self.getDevice())
        self._changed = True

    def hasPassiveScalar(self):
        return self.getParentDomain().hasPassiveScalar()

    def getPassiveScalarChannels(self):
        return self.getParentDomain().getPassiveScalarChannels()

    def hasPassiveScalarViscosity(self):
        return False

    def setVelocitySource(self, t):
        self._check_tensor(t, self.getSpatialDims(), True, "VelocitySource")
        if self.velocitySourceGrad is not None:
            _check(self.velocitySourceGrad.dim() == t.dim(), "New velocity source does not match existing gradient tensor.")
        self.velocitySource = t
        self.isVelocitySourceStatic = t.dim() == 2
        self._changed = True

    def hasVelocitySource(self):
        return self.velocitySource is not None

    def CreateVelocitySource(self, createStatic):
        dims = self.getSpatialDims()
        if createStatic:
            t = torch.zeros((1, dims), dtype=self.getDtype(), device=self.getDevice())
        else:
            t = torch.zeros_like(self.velocity)
        self.setVelocitySource(t)

    def clearVelocitySource(self):
        if self.velocitySource is not None:
            self.velocitySource = None
            self._changed = True

    def setViscosity(self, v):
        self._check_tensor(v, 1, True, "BlockViscosity")
        if self.viscosityGrad is not None:
            _check(self.viscosityGrad.dim() == v.dim(), "New block viscosity does not match existing gradient tensor.")
        self.viscosity = v
        self._changed = True

    def hasViscosity(self):
        return self.viscosity is not None

    def isViscosityStatic(self):
        return self.viscosity is None or self.viscosity.dim() == 2

    def clearViscosity(self):
        if self.viscosity is not None:
            self.viscosity = None
            self._changed = True

    # -- gradients (adjoint fields) --
    def setVelocityGrad(self, t):
        self._check_tensor(t, self.getSpatialDims(), False, "VelocityGrad")
        self.velocityGrad = t
        self._changed = True

    def CreateVelocityGrad(self):
        self.setVelocityGrad(torch.zeros_like(self.velocity))

    def setPassiveScalarGrad(self, t):
        _check(self.passiveScalar is not None, "Block does not have a passive scalar.")
        _check(t.shape == self.passiveScalar.shape, "Block passive scalar gradient must match the passive scalar.")
        self.passiveScalarGrad = t
        self._changed = True

    def CreatePassiveScalarGrad(self):
        if self.passiveScalar is not None:
            self.setPassiveScalarGrad(torch.zeros_like(self.passiveScalar))

    def setPressureGrad(self, t):
        self._check_tensor(t, 1, False, "PressureGrad")
        self.pressureGrad = t
        self._changed = True

    def CreatePressureGrad(self):
        self.setPressureGrad(torch.zeros_like(self.pressure))

    def setVelocitySourceGrad(self, t):
        self.velocitySourceGrad = t
        self._changed = True

    def hasVelocitySourceGrad(self):
        return self.velocitySourceGrad is not None

    def CreateVelocitySourceGrad(self):
        if self.velocitySource is not None:
            self.setVelocitySourceGrad(torch.zeros_like(self.velocitySource))
        else:
            self.clearVelocitySourceGrad()

    def clearVelocitySourceGrad(self):
        if self.velocitySourceGrad is not None:
            self.velocitySourceGrad = None
            self._changed = True

    def setViscosityGrad(self, t):
        self.viscosityGrad = t
        self._changed = True

    def CreateViscosityGrad(self):
        if self.viscosity is not None:
            self.setViscosityGrad(torch.zeros_like(self.viscosity))

    def hasViscosityGrad(self):
        return self.viscosityGrad is not None

    def clearViscosityGrad(self):
        if self.viscosityGrad is not None:
            self.viscosityGrad = None
            self._changed = True

    def CreateVelocityGradOnBoundaries(self):
        for b in self.boundaries:
            if isinstance(b, FixedBoundary):
                b.CreateVelocityGrad()

    def CreatePassiveScalarGradOnBoundaries(self):
        for b in self.boundaries:
            if isinstance(b, FixedBoundary):
                b.CreatePassiveScalarGrad()

    def DetachFwd(self):
        self.velocity = self.velocity.detach()
        self.pressure = self.pressure.detach()
        if self.velocitySource is not None:
            self.velocitySource = self.velocitySource.detach()
        if self.viscosity is not None:
            self.viscosity = self.viscosity.detach()
        for b in self.boundaries:
            if isinstance(b, FixedBoundary):
                b.DetachFwd()

    def DetachGrad(self):
        self.velocityGrad = self.velocityGrad.detach()
        self.pressureGrad = self.pressureGrad.detach()
        for b in self.boundaries:
            if isinstance(b, FixedBoundary):
                b.DetachGrad()

    def Detach(self):
        self.DetachFwd()
        self.DetachGrad()

    def IsTensorChanged(self):
        return self._changed or any(b.IsTensorChanged() for b in self.boundaries)

    def _set_unchanged(self):
        self._changed = False
        for b in self.boundaries:
            b._changed = False

    # -- coordinates and transforms --
    def setVertexCoordinates(self, coords):
        """Block::setVertexCoordinates, extensions/domain_structs.cpp:2001-2019."""
        _check(coords.is_cuda and coords.is_contiguous(), "vertex coordinates must be a contiguous CUDA tensor")
        _check(coords.dim() == self.velocity.dim(), "new vertex coordinates dimensions must match velocity.")
        _check(coords.size(0) == 1, "batches are not yet supported.")
        _check(coords.size(1) == self.getSpatialDims(), "vertex coordinates channel dimension must match spatial dimensions.")
        for d in range(2, self.velocity.dim()):
            _check(self.velocity.size(d) == coords.size(d) - 1, "vertex coordinates spatial dimension must match velocity's +1.")
        _check(coords.dtype == self.velocity.dtype, "Vertex coordinates and velocity must have same dtype.")
        self.clearCoordsTransforms()
        self.vertexCoordinates = coords
        self.transform = CoordsToTransforms(coords)
        self.faceTransform = CoordsToFaceTransforms(coords)
        self._UpdateBoundaryTransforms()
        self._changed = True

    def hasVertexCoordinates(self):
        return self.vertexCoordinates is not None

    def getCellCoordinates(self):
        _check(self.hasVertexCoordinates(), "VertexCoordinates are required to compute cell coordinates.")
        dims = self.getSpatialDims()
        pool = {1: torch.nn.functional.avg_pool1d, 2: torch.nn.functional.avg_pool2d, 3: torch.nn.functional.avg_pool3d}[dims]
        return pool(self.vertexCoordinates, 2, 1)

    def setTransform(self, transform, faceTransform=None):
        dims = self.getSpatialDims()
        _check(transform.is_cuda and transform.is_contiguous(), "transform must be a contiguous CUDA tensor")
        _check(transform.dim() == self.velocity.dim(), "new ransform dimensions must match velocity.")
        _check(transform.size(-1) == _transform_size(dims), "Transform channels must match spatial dimensions")
        self.clearCoordsTransforms()
        self.transform = transform
        self.faceTransform = faceTransform
        self._UpdateBoundaryTransforms()
        self._changed = True

    def hasTransform(self):
        return self.transform is not None

    def hasFaceTransform(self):
        return self.faceTransform is not None

    def getCellSizes(self):
        if self.hasTransform():
            return torch.abs(self.transform[..., -1]).unsqueeze(1)
        return torch.ones_like(self.pressure)

    def clearCoordsTransforms(self):
        self._changed = self._changed or self.hasTransform() or self.hasFaceTransform() or self.hasVertexCoordinates()
        self.transform = None
        self.faceTransform = None
        self.vertexCoordinates = None

    def GetCoordinateOrientation(self):
        if not self.hasTransform():
            return 1
        s = torch.sign(self.transform[..., -1])
        smin, smax = int(s.min().item()), int(s.max().item())
        return 0 if smin != smax else smin

    def _GetFaceTransformBoundarySlice(self, face):
        """extensions/domain_structs.cpp:1809-1835."""
        _check(self.hasFaceTransform(), "faceTransform missing to slice for boundary.")
        dims = self.getSpatialDims()
        axis, upper = face >> 1, face & 1
        idx = [slice(None), axis]
        for d in range(dims - 1, -1, -1):
            if d == axis:
                idx.append(slice(-1, None) if upper else slice(0, 1))
            else:
                idx.append(slice(0, -1))
        idx.append(slice(None))
        return self.faceTransform[tuple(idx)].clone().contiguous()

    def _UpdateBoundaryTransforms(self):
        if not self.hasFaceTransform():
            return
        for f, b in enumerate(self.boundaries):
            if isinstance(b, FixedBoundary):
                b.setTransform(self._GetFaceTransformBoundarySlice(f))

    # -- boundaries --
    def _check_face(self, face):
        _check(0 <= face < 2 * self.getSpatialDims(),
               "Face index must be in [0, dims*2) or one of {-x, +x, -y, +y, -z, +z} for exising spatial dimensions.")

    def _setBoundary(self, faceIndex, boundary):
        """Block::setBoundary, extensions/domain_structs.cpp:1653-1741."""
        face = _face_index(faceIndex)
        self._check_face(face)
        dims = self.getSpatialDims()
        if isinstance(boundary, FixedBoundary):
            if boundary.hasSize():
                _check(boundary.getSizes()[face >> 1] == 1, "Boundary axis size must be 1.")
                for k in range(1, dims):
                    ax = ((face >> 1) + k) % dims
                    _check(boundary.getSizes()[ax] == self.getAxis(ax), "Boundary size must match block.")
            else:
                s = [self.getAxis(d) for d in range(dims)]
                s[face >> 1] = 1
                boundary._setSize(s)
            if self.hasTransform() != boundary.hasTransform():
                print("Warning: Only one of Block and FixedBoundary has a transformation set.")
        elif isinstance(boundary, ConnectedBoundary):
            other = boundary.getConnectedBlock()
            for k in range(1, dims):
                ax = ((face >> 1) + k) % dims
                _check(self.getAxis(ax) == other.getAxis(boundary.getConnectionAxis(k)),
                       "%s connection axis size does not match." % ("First" if k == 1 else "Second"))
        self.boundaries[face] = boundary
        self._changed = True

    def getBoundary(self, faceIndex):
        face = _face_index(faceIndex)
        _check(0 <= face < 2 * self.getSpatialDims(), "Invalid boundary location specified.")
        return self.boundaries[face]

    def getBoundaries(self):
        return list(self.boundaries)

    def hasPrescribedBoundary(self):
        return any(isinstance(b, FixedBoundary) for b in self.boundaries)

    def getFixedBoundaries(self):
        return [(i, b) for i, b in enumerate(self.boundaries) if isinstance(b, FixedBoundary)]

    def isAllFixedBoundariesPassiveScalarTypeStatic(self):
        return all(b.isPassiveScalarBoundaryTypeStatic() for _, b in self.getFixedBoundaries())

    def _MakeFixedBoundary(self, face, velocity=None, passiveScalar=None):
        """extensions/domain_structs.cpp:1897-1922."""
        d = self.getParentDomain()
        transform = self._GetFaceTransformBoundarySlice(face) if self.hasFaceTransform() else None
        fb = FixedBoundary(d, velocity, BoundaryConditionType.DIRICHLET, passiveScalar, transform)
        self._setBoundary(face, fb)

    def _CloseConnectedBoundary(self, face):
        """Block::CloseConnectedBoudary with useFixed, extensions/domain_structs.cpp:1773-1807."""
        b = self.boundaries[face]
        if isinstance(b, ConnectedBoundary):
            b.getConnectedBlock()._MakeFixedBoundary(b.axes[0])
        elif isinstance(b, PeriodicBoundary):
            self._MakeFixedBoundary(face ^ 1)

    def CloseBoundary(self, faceIndex, velocity=None, passiveScalar=None):
        face = _face_index(faceIndex)
        self._check_face(face)
        self._CloseConnectedBoundary(face)
        self._MakeFixedBoundary(face, velocity, passiveScalar)

    def CloseAllBoundaries(self):
        for f in range(2 * self.getSpatialDims()):
            self.CloseBoundary(f)

    def ConnectBlock(self, faceIndex, otherBlock, otherFaceIndex, axis1Index=-1, axis2Index=-1):
        """Block::ConnectBlock -> ConnectBlocks, extensions/domain_structs.cpp:1064-1097, 1924-1930."""
        face1 = _face_index(faceIndex)
        face2 = _face_index(otherFaceIndex)
        a1 = _face_index(axis1Index) if axis1Index not in (-1, "") else -1
        a2 = _face_index(axis2Index) if axis2Index not in (-1, "") else -1
        self._check_face(face1)
        self._CloseConnectedBoundary(face1)
        otherBlock._check_face(face2)
        otherBlock._CloseConnectedBoundary(face2)
        _check(self.getParentDomain() is otherBlock.getParentDomain(), "The blocks must belong to the same domain.")
        dims = self.getSpatialDims()
        axes1, axes2 = [face2], [face1]
        if dims > 1:
            axes1.append(a1)
            f1d, f2d = face1 >> 1, face2 >> 1
            swapped = False
            if dims == 2 or (a1 >> 1) == (f2d + 1) % dims:
                axes2.append((((f1d + 1) % dims) << 1) | (a1 & 1))
            else:
                _check((a2 >> 1) == (f2d + 1) % dims, "Invalid connection.")
                axes2.append((((f1d + 2) % dims) << 1) | (a2 & 1))
                swapped = True
            if dims > 2:
                axes1.append(a2)
                if not swapped:
                    axes2.append((((f1d + 2) % dims) << 1) | (a2 & 1))
                else:
                    axes2.append((((f1d + 1) % dims) << 1) | (a1 & 1))
        d = self.getParentDomain()
        self._setBoundary(face1, ConnectedBoundary(otherBlock, axes1, d))
        otherBlock._setBoundary(face2, ConnectedBoundary(self, axes2, d))

    def MakePeriodic(self, axisIndex):
        axis = _axis_index(axisIndex)
        _check(0 <= axis < self.getSpatialDims(), "Axis index must be in [0, dims) or one of {x, y, z} for exising spatial dimensions.")
        lo, hi = axis << 1, (axis << 1) | 1
        bl, bh = self.boundaries[lo], self.boundaries[hi]
        if not (isinstance(bl, PeriodicBoundary) and isinstance(bh, PeriodicBoundary)):
            if isinstance(bl, ConnectedBoundary):
                self._CloseConnectedBoundary(lo)
            if isinstance(bh, ConnectedBoundary):
                self._CloseConnectedBoundary(hi)
            d = self.getParentDomain()
            if not isinstance(self.boundaries[lo], PeriodicBoundary):
                self._setBoundary(lo, PeriodicBoundary(d))
            if not isinstance(self.boundaries[hi], PeriodicBoundary):
                self._setBoundary(hi, PeriodicBoundary(d))

    def MakeAllPeriodic(self):
        for a in range(self.getSpatialDims()):
            self.MakePeriodic(a)

    def ComputeCSRSize(self):
        """extensions/domain_structs.cpp:2151-2161."""
        s = self.getSizes()
        sz = [s.x, s.y, s.z]
        n = s.x * s.y * s.z * (2 * self.getSpatialDims() + 1)
        for d in range(self.getSpatialDims()):
            area = sz[(d + 1) % 3] * sz[(d + 2) % 3]
            if isinstance(self.boundaries[2 * d], FixedBoundary):
                n -= area
            if isinstance(self.boundaries[2 * d + 1], FixedBoundary):
                n -= area
        return n

    # -- velocity statistics --
    def getMaxVelocity(self, withBounds=True, computational=False):
        m = torch.max(torch.abs(self.getVelocity(computational)))
        if withBounds:
            for b in self.boundaries:
                if isinstance(b, FixedBoundary):
                    m = torch.maximum(m, torch.max(torch.abs(b.getVelocity(computational))))
        return m

    def getMaxVelocityMagnitude(self, withBounds=True, computational=False):
        m = torch.max(torch.linalg.vector_norm(self.getVelocity(computational), dim=1))
        if withBounds:
            for b in self.boundaries:
                if isinstance(b, FixedBoundary):
                    m = torch.maximum(m, torch.max(torch.linalg.vector_norm(b.getVelocity(computational), dim=1)))
        return m

    def __str__(self):
        s = self.getSizes()
        return 'Block("%s", size=%s, boundaries=[%s])' % (self.name, s, ", ".join(str(b) for b in self.boundaries))


# ------------------------------------------------------------------------------------------------
# domain (extensions/domain_structs.h:563-787)
# ------------------------------------------------------------------------------------------------


class Domain:
    def __init__(self, spatialDims, viscosity, name="Domain", dtype=torch.float32, device=None,
                 passiveScalarChannels=1, scalarViscosity=None):
        _check(0 < spatialDims < 4, "spatialDims must be 1, 2, or 3.")
        _check(passiveScalarChannels >= 0, "passiveScalarChannels can't be negative.")
        self.name = name
        self._dims = int(spatialDims)
        self._dtype = dtype
        _dtype_code(dtype)
        device = torch.device("cuda") if device is None else torch.device(device)
        _check(device.type == "cuda", "device must be a CUDA device.")
        if device.index is None:
            device = torch.device("cuda", 0)
        self._device = device
        self._psc = int(passiveScalarChannels)
        self.blocks: List[Block] = []
        self.passiveScalarViscosity = scalarViscosity
        self.setViscosity(viscosity)
        self._initialized = False
        self._changed = True
        self._csr_struct = None
        self.viscosityGrad = None
        self.passiveScalarViscosityGrad = None

    # -- basic properties --
    def getSpatialDims(self):
        return self._dims

    def getDtype(self):
        return self._dtype

    def getDevice(self):
        return self._device

    def getPassiveScalarChannels(self):
        return self._psc

    def hasPassiveScalar(self):
        return self._psc > 0

    def getNumBlocks(self):
        return len(self.blocks)

    def getBlock(self, index):
        return self.blocks[index]

    def getBlocks(self):
        return list(self.blocks)

    def getTotalSize(self):
        return sum(b._ncells() for b in self.blocks)

    def getMaxBlockSize(self):
        return max(b._ncells() for b in self.blocks)

    def IsInitialized(self):
        return self._initialized

    def IsTensorChanged(self):
        return self._changed or any(b.IsTensorChanged() for b in self.blocks)

    def setViscosity(self, viscosity):
        _check(isinstance(viscosity, torch.Tensor) and not viscosity.is_cuda, "viscosity must be a host tensor")
        _check(viscosity.dim() == 1 and viscosity.size(0) == 1, "viscosity must be a scalar.")
        self.viscosity = viscosity
        if getattr(self, "_initialized", False):
            with torch.no_grad():
                self._sim_visc.copy_(viscosity.detach().to(self._dtype), non_blocking=False)

    def hasBlockViscosity(self):
        return any(b.hasViscosity() for b in self.blocks)

    def hasPassiveScalarViscosity(self):
        return self.passiveScalarViscosity is not None

    def isPassiveScalarViscosityStatic(self):
        return self.passiveScalarViscosity is None or self.passiveScalarViscosity.size(0) == 1

    def setScalarViscosity(self, v):
        self.passiveScalarViscosity = v

    def clearScalarViscosity(self):
        self.passiveScalarViscosity = None

    def hasPassiveScalarBlockViscosity(self):
        return False

    # -- blocks --
    def CreateBlock(self, velocity=None, pressure=None, passiveScalar=None, vertexCoordinates=None, name="Block"):
        b = Block(self, velocity, pressure, passiveScalar, vertexCoordinates, name)
        _check(b.getDevice() == self._device, "Block has wrong device")
        self.AddBlock(b)
        return b

    def CreateBlockWithSize(self, size, name="Block"):
        size = [size[0], size[1], size[2]] if not isinstance(size, Int4) else [size.x, size.y, size.z]
        _check(size[0] > 2, "size.x must be at least 3.")
        if self._dims > 1:
            _check(size[1] > 2, "size.y must be at least 3.")
        if self._dims > 2:
            _check(size[2] > 2, "size.z must be at least 3.")
        b = Block(self, name=name, size=size[:self._dims])
        self.AddBlock(b)
        return b

    def AddBlock(self, block):
        _check(block.getSpatialDims() == self._dims, "Number of block spatial dimensions does not match domain.")
        _check(block.getDtype() == self._dtype, "Data typ does not match.")
        self.blocks.append(block)
        self._initialized = False

    def _block_index(self, block):
        for i, b in enumerate(self.blocks):
            if b is block:
                return i
        return -1

    # -- statistics --
    def getMaxVelocity(self, withBounds=True, computational=False):
        _check(len(self.blocks) > 0, "Domain does not contain any blocks.")
        m = self.blocks[0].getMaxVelocity(withBounds, computational)
        for b in self.blocks[1:]:
            m = torch.maximum(m, b.getMaxVelocity(withBounds, computational))
        return m

    def getMaxVelocityMagnitude(self, withBounds=True, computational=False):
        _check(len(self.blocks) > 0, "Domain does not contain any blocks.")
        m = self.blocks[0].getMaxVelocityMagnitude(withBounds, computational)
        for b in self.blocks[1:]:
            m = torch.maximum(m, b.getMaxVelocityMagnitude(withBounds, computational))
        return m

    def hasVertexCoordinates(self):
        return len(self.blocks) > 0 and all(b.hasVertexCoordinates() for b in self.blocks)

    def getVertexCoordinates(self):
        _check(len(self.blocks) > 0, "Domain does not contain any blocks.")
        out = []
        for b in self.blocks:
            _check(b.hasVertexCoordinates(), "a block is missing vertex coordinates")
            out.append(b.vertexCoordinates)
        return out

    def GetCoordinateOrientation(self):
        _check(len(self.blocks) > 0, "Domain does not contain any blocks.")
        s = self.blocks[0].GetCoordinateOrientation()
        for b in self.blocks[1:]:
            if b.GetCoordinateOrientation() != s:
                return 0
        return s

    def hasPrescribedBoundary(self):
        return any(b.hasPrescribedBoundary() for b in self.blocks)

    def isAllFixedBoundariesPassiveScalarTypeStatic(self):
        return all(b.isAllFixedBoundariesPassiveScalarTypeStatic() for b in self.blocks)

    def GetBoundaryFluxBalance(self):
        """Domain::GetGlobalFluxBalance, extensions/domain_structs.cpp:2460-2493."""
        s = torch.zeros([1], dtype=self._dtype, device=self._device)
        for b in self.blocks:
            for i, bnd in enumerate(b.boundaries):
                if isinstance(bnd, FixedBoundary):
                    f = torch.sum(bnd.GetFluxes())
                    s = s + (f if (i & 1) else -f)
        return s

    def CheckBoundaryFluxBalance(self, eps=1e-5):
        return abs(self.GetBoundaryFluxBalance().item()) < eps

    # -- preparation (Domain::PrepareSolve, extensions/domain_structs.cpp:2554-2676) --
    def PrepareSolve(self):
        _check(len(self.blocks) > 0, "Domain does not contain any blocks.")
        _check(self.viscosity.dtype == self._dtype, "Data type of viscosity does not match.")
        dims = self._dims
        N = 0
        csr = 0
        for b in self.blocks:
            b.globalOffset = N
            b.csrOffset = csr
            csr += b.ComputeCSRSize()
            N += b._ncells()
            for f, bnd in enumerate(b.boundaries):
                if isinstance(bnd, ConnectedBoundary):
                    other = bnd.getConnectedBlock()
                    _check(self._block_index(other) >= 0, "Connected block is not part of this domain.")
                    ob = other.boundaries[bnd.axes[0]]
                    _check(isinstance(ob, ConnectedBoundary),
                           "Mismatch in block connection: connected block is not connected at the target face.")
                    _check(ob.getConnectedBlock() is b,
                           "Mismatch in block connection: connected block is connected to a different block at the target face.")
                    _check(ob.axes[0] == f,
                           "Mismatch in block connection: connected block is connected to a different face of the source block.")
                elif isinstance(bnd, PeriodicBoundary):
                    _check(isinstance(b.boundaries[f ^ 1], PeriodicBoundary), "Opposite boundary must also be periodic.")
        self._N = N
        self._K = 2 * dims + 1
        opts = dict(dtype=self._dtype, device=self._device)
        self.C = StencilMatrix(self, torch.zeros((self._K, N), **opts))
        self.P = StencilMatrix(self, torch.zeros((self._K, N), **opts))
        self.CGrad = self.C.WithZeroValue()
        self.PGrad = self.P.WithZeroValue()
        self.A = torch.zeros(N, **opts)
        self.AGrad = torch.empty(0)
        if self.hasPassiveScalar():
            self.scalarRHS = torch.zeros(N * self._psc, **opts)
            self.scalarResult = torch.zeros(N * self._psc, **opts)
        else:
            self.scalarRHS = torch.empty(0, **opts)
            self.scalarResult = torch.empty(0, **opts)
        self.velocityRHS = torch.zeros(N * dims, **opts)
        self.velocityResult = torch.zeros(N * dims, **opts)
        self.pressureRHS = torch.zeros(N * dims, **opts)
        self.pressureRHSdiv = torch.zeros(N, **opts)
        self.pressureResult = torch.zeros(N, **opts)
        for name in ["scalarRHSGrad", "scalarResultGrad", "velocityRHSGrad", "velocityResultGrad", "pressureRHSGrad",
                     "pressureRHSdivGrad", "pressureResultGrad"]:
            setattr(self, name, torch.empty(0))
        # topology on the host (native), then upload
        self._sim_visc = self.viscosity.to(self._dtype).to(self._device)
        self._sim_cells = torch.tensor([0, N], dtype=torch.int32, device=self._device)
        self._sim_blocks = torch.tensor([0, len(self.blocks)], dtype=torch.int32, device=self._device)
        host_blocks = self._pack_blocks()
        nbr = torch.empty((2 * dims, N), dtype=torch.int32)
        cell_block = torch.empty(N, dtype=torch.int32)
        check(_lib.load().pict_build_topology(host_blocks, len(self.blocks), dims, N, nbr.data_ptr(),
                                              cell_block.data_ptr()), "build_topology")
        self._nbr = nbr.to(self._device)
        self._cell_block = cell_block.to(self._device)
        self._tile_cells = getattr(self, "_tile_cells", TILE_CELLS)
        self._tiles, self._sim_tiles, self._num_tiles = build_tiles(host_blocks, len(self.blocks), 1, self._device,
                                                                    self._tile_cells)
        self._csr_struct = None
        self._initialized = True
        self.UpdateDomainData()

    def set_tile_cells(self, tile_cells):
        """Cells per Krylov work tile (1..2048): rebuilds the tile table of a prepared domain.  Steppers
        created before the change must be re-created (their workspace depends on the tile count)."""
        tile_cells = int(tile_cells)
        _check(1 <= tile_cells <= 2048, "tile_cells must be in [1, 2048]")
        self._tile_cells = tile_cells
        if self._initialized:
            self._tiles, self._sim_tiles, self._num_tiles = build_tiles(self._pack_blocks(), len(self.blocks), 1,
                                                                        self._device, tile_cells)
            self._desc = self._make_desc()

    def _pack_blocks(self):
        """Host block table with raw device pointers (Domain::UpdateDomainGPU, extensions/domain_structs.cpp:3040-3261)."""
        arr = (BlockDesc * len(self.blocks))()
        index = {id(b): i for i, b in enumerate(self.blocks)}
        psc = self._psc if self.hasPassiveScalar() else 0
        for bi, b in enumerate(self.blocks):
            d = arr[bi]
            s = b.getSizes()
            d.size[0], d.size[1], d.size[2] = s.x, s.y, s.z
            d.offset = b.globalOffset
            d.sim = 0
            d.velocity = _ptr(b.velocity)
            d.pressure = _ptr(b.pressure)
            d.transform = _ptr(b.transform) if b.hasTransform() else None
            d.face_transform = _ptr(b.faceTransform) if b.hasFaceTransform() else None
            if b.viscosity is not None:
                d.viscosity = _ptr(b.viscosity)
                d.viscosity_static = 1 if b.viscosity.dim() == 2 else 0
            if b.velocitySource is not None:
                d.source = _ptr(b.velocitySource)
                d.source_static = 1 if b.isVelocitySourceStatic else 0
            d.velocity_grad = _ptr(b.velocityGrad) if b.velocityGrad.numel() > 0 else None
            d.pressure_grad = _ptr(b.pressureGrad) if b.pressureGrad.numel() > 0 else None
            d.viscosity_grad = _ptr(b.viscosityGrad) if b.viscosityGrad is not None else None
            d.source_grad = _ptr(b.velocitySourceGrad) if b.velocitySourceGrad is not None else None
            if psc and b.passiveScalar is not None:
                d.scalar = _ptr(b.passiveScalar)
                g = b.passiveScalarGrad
                d.scalar_grad = _ptr(g) if g is not None and g.numel() > 0 else None
            for f, bnd in enumerate(b.boundaries):
                F = d.face[f]
                if isinstance(bnd, FixedBoundary):
                    F.type = _lib.PICT_FACE_FIXED
                    F.vel_static = 1 if bnd.isVelocityStatic else 0
                    F.velocity = _ptr(bnd.velocity)
                    F.transform = _ptr(bnd.transform) if bnd.hasTransform() else None
                    F.velocity_grad = _ptr(bnd.velocityGrad) if bnd.velocityGrad is not None and bnd.velocityGrad.numel() > 0 else None
                    if psc and bnd.passiveScalar is not None:
                        F.scalar = _ptr(bnd.passiveScalar)
                        F.scalar_static = 1 if bnd.passiveScalar.dim() == 2 else 0
                        F.scalar_neumann = bnd._scalar_neumann_mask(psc)
                        g = bnd.passiveScalarGrad
                        F.scalar_grad = _ptr(g) if g is not None and g.numel() > 0 else None
                elif isinstance(bnd, PeriodicBoundary):
                    F.type = _lib.PICT_FACE_PERIODIC
                elif isinstance(bnd, ConnectedBoundary):
                    F.type = _lib.PICT_FACE_CONNECTED
                    F.conn_block = index[id(bnd.getConnectedBlock())]
                    for k in range(len(bnd.axes)):
                        F.conn_axes[k] = bnd.axes[k]
                else:
                    raise NotImplementedError("boundary type %s is not supported" % type(bnd).__name__)
        return arr

    def UpdateDomainData(self):
        """Re-pack raw pointers after tensors were replaced (Domain::UpdateDomain, extensions/domain_structs.cpp:3031-3038)."""
        _check(self._initialized, "Domain is not initialized.")
        host = self._pack_blocks()
        raw = bytes(host)
        if getattr(self, "_blocks_raw", None) != raw:
            buf = torch.frombuffer(bytearray(raw), dtype=torch.uint8).pin_memory()
            if getattr(self, "_blocks_dev", None) is None or self._blocks_dev.numel() != buf.numel():
                self._blocks_dev = torch.empty(buf.numel(), dtype=torch.uint8, device=self._device)
            self._blocks_dev.copy_(buf, non_blocking=True)
            self._blocks_raw = raw
            self._blocks_host = buf
        self._desc = self._make_desc()
        self._changed = False
        for b in self.blocks:
            b._set_unchanged()

    def _make_desc(self, C=None, P=None):
        d = DomainDesc()
        d.dims = self._dims
        d.num_blocks = len(self.blocks)
        d.num_cells = self._N
        d.num_sims = 1
        d.dtype = _dtype_code(self._dtype)
        d.max_sim_cells = self._N
        d.blocks = self._blocks_dev.data_ptr()
        d.nbr = _ptr(self._nbr)
        d.cell_block = _ptr(self._cell_block)
        d.sim_cells = _ptr(self._sim_cells)
        d.sim_blocks = _ptr(self._sim_blocks)
        d.tiles = _ptr(self._tiles)
        d.sim_tiles = _ptr(self._sim_tiles)
        d.num_tiles = self._num_tiles
        d.tile_cells = self._tile_cells
        d.sim_viscosity = _ptr(self._sim_visc)
        d.sim_dt = None
        d.C = _ptr(self.C.coef if C is None else C)
        d.A = _ptr(self.A)
        d.P = _ptr(self.P.coef if P is None else P)
        d.velocity_rhs = _ptr(self.velocityRHS)
        d.velocity_result = _ptr(self.velocityResult)
        d.pressure_rhs = _ptr(self.pressureRHS)
        d.pressure_rhs_div = _ptr(self.pressureRHSdiv)
        d.pressure_result = _ptr(self.pressureResult)
        if self.hasPassiveScalar():
            d.scalar_channels = self._psc
            sv = self._scalar_viscosity_device()
            if sv is not None:
                d.scalar_viscosity = _ptr(sv)
                d.scalar_viscosity_static = 1 if sv.numel() == 1 else 0
            d.scalar_rhs = _ptr(self.scalarRHS) if self.scalarRHS.numel() > 0 else None
            d.scalar_result = _ptr(self.scalarResult) if self.scalarResult.numel() > 0 else None
        return d

    def _scalar_viscosity_device(self):
        """The scalar viscosity as a contiguous tensor on the domain's device and dtype (a cached copy when
        it was given elsewhere)."""
        sv = self.passiveScalarViscosity
        if sv is None:
            return None
        if sv.device == self._device and sv.dtype == self._dtype and sv.is_contiguous():
            return sv
        key = (id(sv), sv._version)
        if getattr(self, "_sv_key", None) != key:
            self._sv_dev = sv.detach().to(device=self._device, dtype=self._dtype).contiguous()
            self._sv_key = key
        return self._sv_dev

    def _check_ready(self):
        _check(len(self.blocks) > 0, "Domain does not contain blocks.")
        _check(self._initialized, "Domain is not initialized.")
        _check(not self.IsTensorChanged(), "Domain's tensors have been changed, use UpdateDomain() to set the new pointers.")
        # keep the packed global pointers in sync with the current tensors
        self._desc = self._make_desc()

    def _csr_structure(self):
        if self._csr_struct is None:
            row = torch.empty(self._N + 1, dtype=torch.int32, device=self._device)
            check(_lib.load().pict_csr_row_ptr(ctypes.byref(self._desc), _ptr(row), _stream_ptr()), "csr_row_ptr")
            nnz = int(row[-1].item())
            index = torch.empty(nnz, dtype=torch.int32, device=self._device)
            tmp = torch.empty(nnz, dtype=self._dtype, device=self._device)
            check(_lib.load().pict_stencil_to_csr(ctypes.byref(self._desc), _ptr(self.C.coef), _ptr(row), _ptr(tmp),
                                                  _ptr(index), _stream_ptr()), "stencil_to_csr")
            self._csr_struct = (row, index)
        return self._csr_struct

    # -- global field setters (extensions/domain_structs.cpp:2750-2828) --
    def _set_global(self, name, t, size):
        _check(t.is_cuda and t.is_contiguous() and t.dim() == 1, "%s must be a contiguous 1D CUDA tensor" % name)
        _check(t.size(0) == size, "%s has the wrong size (%d, expected %d)" % (name, t.size(0), size))
        _check(t.dtype == self._dtype, "%s dtype must match the domain" % name)
        setattr(self, name, t)
        self._changed = True

    def setA(self, t):
        self._set_global("A", t, self._N)

    def CreateA(self):
        self.setA(torch.zeros(self._N, dtype=self._dtype, device=self._device))

    def setVelocityRHS(self, t):
        self._set_global("velocityRHS", t, self._N * self._dims)

    def setVelocityResult(self, t):
        self._set_global("velocityResult", t, self._N * self._dims)

    def setPressureRHS(self, t):
        self._set_global("pressureRHS", t, self._N * self._dims)

    def setPressureRHSdiv(self, t):
        self._set_global("pressureRHSdiv", t, self._N)

    def setPressureResult(self, t):
        self._set_global("pressureResult", t, self._N)

    def CreateScalarRHS(self):
        self.scalarRHS = torch.zeros(self._N * self._psc, dtype=self._dtype, device=self._device)

    def CreateScalarResult(self):
        self.scalarResult = torch.zeros(self._N * self._psc, dtype=self._dtype, device=self._device)

    def setScalarRHS(self, t):
        self._set_global("scalarRHS", t, self._N * self._psc)

    def setScalarResult(self, t):
        self._set_global("scalarResult", t, self._N * self._psc)

    def CreateVelocityRHS(self):
        self.setVelocityRHS(torch.zeros(self._N * self._dims, dtype=self._dtype, device=self._device))

    def CreateVelocityResult(self):
        self.setVelocityResult(torch.zeros(self._N * self._dims, dtype=self._dtype, device=self._device))

    def CreatePressureRHS(self):
        self.setPressureRHS(torch.zeros(self._N * self._dims, dtype=self._dtype, device=self._device))

    def CreatePressureRHSdiv(self):
        self.setPressureRHSdiv(torch.zeros(self._N, dtype=self._dtype, device=self._device))

    def CreatePressureResult(self):
        self.setPressureResult(torch.zeros(self._N, dtype=self._dtype, device=self._device))

    def CreateVelocityOnBlocks(self):
        for b in self.blocks:
            b.CreateVelocity()

    def CreatePressureOnBlocks(self):
        for b in self.blocks:
            b.CreatePressure()

    def CreateVelocityGradOnBlocks(self):
        for b in self.blocks:
            b.CreateVelocityGrad()

    def CreatePressureGradOnBlocks(self):
        for b in self.blocks:
            b.CreatePressureGrad()

    def CreateVelocitySourceGradOnBlocks(self):
        for b in self.blocks:
            b.CreateVelocitySourceGrad()

    def CreateVelocityGradOnBoundaries(self):
        for b in self.blocks:
            b.CreateVelocityGradOnBoundaries()

    def CreatePassiveScalarGradOnBlocks(self):
        for b in self.blocks:
            b.CreatePassiveScalarGrad()

    def CreatePassiveScalarGradOnBoundaries(self):
        for b in self.blocks:
            b.CreatePassiveScalarGradOnBoundaries()

    def CreateViscosityGrad(self):
        """Zero gradient of the domain viscosity, of every block viscosity and of the passive scalar
        viscosity (Domain::CreateViscosityGrad, extensions/domain_structs.cpp:2875-2882)."""
        self.viscosityGrad = torch.zeros_like(self.viscosity)
        for b in self.blocks:
            b.CreateViscosityGrad()
        self.CreatePassiveScalarViscosityGrad()

    def CreatePassiveScalarViscosityGrad(self):
        if self.passiveScalarViscosity is not None:
            self.passiveScalarViscosityGrad = torch.zeros_like(self.passiveScalarViscosity)

    def hasPassiveScalarViscosityGrad(self):
        return self.passiveScalarViscosityGrad is not None

    def setPassiveScalarViscosityGrad(self, t):
        _check(self.passiveScalarViscosity is not None and t.shape == self.passiveScalarViscosity.shape,
               "Scalar viscosity grad shape must match Scalar viscosity.")
        self.passiveScalarViscosityGrad = t

    def clearPassiveScalarViscosityGrad(self):
        self.passiveScalarViscosityGrad = None

    def setScalarRHSGrad(self, t):
        self._grad_vec("scalarRHSGrad", t, self._N * self._psc)

    def CreateScalarRHSGrad(self):
        self.scalarRHSGrad = torch.zeros(self._N * self._psc, dtype=self._dtype, device=self._device)

    def setScalarResultGrad(self, t):
        self._grad_vec("scalarResultGrad", t, self._N * self._psc)

    def CreateScalarResultGrad(self):
        self.scalarResultGrad = torch.zeros(self._N * self._psc, dtype=self._dtype, device=self._device)

    def setViscosityGrad(self, t):
        self.viscosityGrad = t

    # -- gradient fields of the global vectors (extensions/PISOtorch.cpp:456-484) --
    def _grad_vec(self, name, t, n):
        _check(isinstance(t, torch.Tensor) and t.dim() == 1 and t.numel() == n,
               "%s must be a 1D tensor with %d elements" % (name, n))
        _check(t.dtype == self._dtype and t.device == self._device, "%s: dtype/device mismatch" % name)
        setattr(self, name, t)

    def setAGrad(self, t):
        self._grad_vec("AGrad", t, self._N)

    def CreateAGrad(self):
        self.AGrad = torch.zeros(self._N, dtype=self._dtype, device=self._device)

    def setVelocityRHSGrad(self, t):
        self._grad_vec("velocityRHSGrad", t, self._N * self._dims)

    def CreateVelocityRHSGrad(self):
        self.velocityRHSGrad = torch.zeros(self._N * self._dims, dtype=self._dtype, device=self._device)

    def setVelocityResultGrad(self, t):
        self._grad_vec("velocityResultGrad", t, self._N * self._dims)

    def CreateVelocityResultGrad(self):
        self.velocityResultGrad = torch.zeros(self._N * self._dims, dtype=self._dtype, device=self._device)

    def setPressureRHSGrad(self, t):
        self._grad_vec("pressureRHSGrad", t, self._N * self._dims)

    def CreatePressureRHSGrad(self):
        self.pressureRHSGrad = torch.zeros(self._N * self._dims, dtype=self._dtype, device=self._device)

    def setPressureRHSdivGrad(self, t):
        self._grad_vec("pressureRHSdivGrad", t, self._N)

    def CreatePressureRHSdivGrad(self):
        self.pressureRHSdivGrad = torch.zeros(self._N, dtype=self._dtype, device=self._device)

    def setPressureResultGrad(self, t):
        self._grad_vec("pressureResultGrad", t, self._N)

    def CreatePressureResultGrad(self):
        self.pressureResultGrad = torch.zeros(self._N, dtype=self._dtype, device=self._device)

    def hasViscosityGrad(self):
        return self.viscosityGrad is not None

    def clearViscosityGrad(self):
        self.viscosityGrad = None

    # -- copies --
    def DetachFwd(self):
        for b in self.blocks:
            b.DetachFwd()
        for name in ["A", "velocityRHS", "velocityResult", "pressureRHS", "pressureRHSdiv", "pressureResult"]:
            if hasattr(self, name):
                setattr(self, name, getattr(self, name).detach())
        if hasattr(self, "C"):
            self.C.detach()
            self.P.detach()

    def DetachGrad(self):
        for b in self.blocks:
            b.DetachGrad()

    def Detach(self):
        self.DetachFwd()
        self.DetachGrad()

    def _copy_structure(self, clone, newName):
        d = Domain(self._dims, self.viscosity.clone() if clone else self.viscosity, newName or (self.name + "_copy"),
                   self._dtype, self._device, self._psc)
        mapping = {}
        for b in self.blocks:
            nb = Block(d, b.velocity.clone() if clone else b.velocity, b.pressure.clone() if clone else b.pressure,
                       None, None, b.name)
            nb.transform = None if b.transform is None else (b.transform.clone() if clone else b.transform)
            nb.faceTransform = None if b.faceTransform is None else (b.faceTransform.clone() if clone else b.faceTransform)
            nb.vertexCoordinates = None if b.vertexCoordinates is None else (b.vertexCoordinates.clone() if clone else b.vertexCoordinates)
            if b.viscosity is not None:
                nb.viscosity = b.viscosity.clone() if clone else b.viscosity
            if b.velocitySource is not None:
                nb.velocitySource = b.velocitySource.clone() if clone else b.velocitySource
                nb.isVelocitySourceStatic = b.isVelocitySourceStatic
            d.AddBlock(nb)
            mapping[id(b)] = nb
        for b in self.blocks:
            nb = mapping[id(b)]
            for f, bnd in enumerate(b.boundaries):
                if isinstance(bnd, FixedBoundary):
                    fb = FixedBoundary(d, bnd.velocity.clone() if clone else bnd.velocity, bnd.velocityType, None,
                                       None if bnd.transform is None else (bnd.transform.clone() if clone else bnd.transform))
                    nb.boundaries[f] = fb
                    fb._size = list(bnd._size) if bnd._size is not None else None
                    fb._axis = bnd._axis
                elif isinstance(bnd, ConnectedBoundary):
                    nb.boundaries[f] = ConnectedBoundary(mapping[id(bnd.getConnectedBlock())], bnd.axes, d)
                else:
                    nb.boundaries[f] = PeriodicBoundary(d)
        return d

    def Copy(self, newName=None):
        return self._copy_structure(False, newName)

    def Clone(self, newName=None):
        return self._copy_structure(True, newName)

    def __str__(self):
        return 'Domain("%s", %dD, blocks=%d, cells=%d, dtype=%s)' % (
            self.name, self._dims, len(self.blocks), self.getTotalSize(), self._dtype)


# ------------------------------------------------------------------------------------------------
# operators (extensions/PISOtorch.cpp:529-601)
# ------------------------------------------------------------------------------------------------


def _time_step(timeStep, domain):
    _check(isinstance(timeStep, torch.Tensor), "timeStep must be a tensor")
    _check(not timeStep.is_cuda, "timeStep must be a host tensor")
    _check(timeStep.dim() == 1 and timeStep.size(0) == 1, "timeStep must be 1D." if timeStep.dim() != 1 else "timeStep must be a scalar.")
    _check(timeStep.dtype == domain.getDtype(), "Data type of timeStep does not match.")
    return float(timeStep.item())


# nonOrthoFlags bits (extensions/PISO_multiblock_cuda.h:9-13); NON_ORTHO_DIAGONAL_MATRIX has no effect in the
# reference either
NON_ORTHO_DIRECT_MATRIX = 1
NON_ORTHO_DIRECT_RHS = 2
NON_ORTHO_DIAGONAL_MATRIX = 4
NON_ORTHO_DIAGONAL_RHS = 8
NON_ORTHO_CENTER_MATRIX = 16


def _non_ortho(flags):
    flags = int(flags)
    _check(0 <= flags < 32, "invalid nonOrthoFlags %d" % flags)
    return flags


def _check_scalar(domain, what):
    _check(domain.hasPassiveScalar(), "%s: the domain has no passive scalar channels." % what)
    for b in domain.getBlocks():
        _check(b.passiveScalar is not None, "%s: block %s has no passive scalar." % (what, b.name))


def SetupAdvectionMatrix(domain, timeStep, nonOrthoFlags, forPassiveScalar=False, passiveScalarChannel=0):
    """Implicit advection-diffusion matrix C and its diagonal A (extensions/PISO_multiblock_cuda_kernel.cu:3601-3865); with
    ``forPassiveScalar`` the matrix of passive scalar channel ``passiveScalarChannel`` (scalar viscosity, no
    diffusion through the channel's Neumann faces)."""
    flags = _non_ortho(nonOrthoFlags)
    domain._check_ready()
    dt = _time_step(timeStep, domain)
    if forPassiveScalar:
        _check_scalar(domain, "SetupAdvectionMatrix")
        ch = int(passiveScalarChannel)
        _check(0 <= ch < domain.getPassiveScalarChannels(), "passiveScalarChannel out of range.")
        check(_lib.load().pict_setup_scalar_matrix(ctypes.byref(domain._desc), dt, flags, ch, _stream_ptr()),
              "SetupAdvectionMatrix")
        return
    check(_lib.load().pict_setup_advection_matrix(ctypes.byref(domain._desc), dt, flags, _stream_ptr()),
          "SetupAdvectionMatrix")


def SetupAdvectionVelocity(domain, timeStep, nonOrthoFlags, applyPressureGradient=False):
    """Velocity RHS of the advection-diffusion solve (extensions/PISO_multiblock_cuda_kernel.cu:4281-4385).  With
    non-orthogonal RHS flags the explicit terms are taken from ``domain.velocityResult`` (as in the reference,
    the caller copies the block velocity there first)."""
    flags = _non_ortho(nonOrthoFlags)
    domain._check_ready()
    dt = _time_step(timeStep, domain)
    check(_lib.load().pict_setup_advection_velocity(ctypes.byref(domain._desc), dt, flags,
                                                    int(bool(applyPressureGradient)), _stream_ptr()),
          "SetupAdvectionVelocity")


def SetupAdvectionScalar(domain, timeStep, nonOrthoFlags):
    """scalarRHS of every passive scalar channel (extensions/PISO_multiblock_cuda_kernel.cu:4079-4183).  With
    non-orthogonal RHS flags the explicit terms are taken from ``domain.scalarResult``."""
    flags = _non_ortho(nonOrthoFlags)
    domain._check_ready()
    _check_scalar(domain, "SetupAdvectionScalar")
    dt = _time_step(timeStep, domain)
    check(_lib.load().pict_setup_scalar_rhs(ctypes.byref(domain._desc), dt, flags, _stream_ptr()), "SetupAdvectionScalar")


def SetupPressureCorrection(domain, timeStep, nonOrthoMode=0, useFaceTransform=False, timeStepNorm=False):
    """Pressure matrix, H/A RHS and its divergence (extensions/PISO_multiblock_cuda_kernel.cu:4797-5419); with
    non-orthogonal RHS flags the explicit terms of ``domain.pressureResult`` are added to the divergence."""
    flags = _non_ortho(nonOrthoMode)
    if useFaceTransform:
        raise NotImplementedError("face-transform pressure assembly is not implemented in pict_b200")
    domain._check_ready()
    dt = _time_step(timeStep, domain)
    check(_lib.load().pict_setup_pressure_correction(ctypes.byref(domain._desc), dt, flags, int(bool(timeStepNorm)),
                                                     _stream_ptr()), "SetupPressureCorrection")


def SetupPressureMatrix(domain, timeStep, nonOrthoMode=0, useFaceTransform=False):
    flags = _non_ortho(nonOrthoMode)
    if useFaceTransform:
        raise NotImplementedError("face-transform pressure assembly is not implemented in pict_b200")
    domain._check_ready()
    _time_step(timeStep, domain)
    check(_lib.load().pict_setup_pressure_matrix(ctypes.byref(domain._desc), flags, _stream_ptr()),
          "SetupPressureMatrix")


def SetupPressureRHS(domain, timeStep, nonOrthoMode=0, useFaceTransform=False, timeStepNorm=False):
    flags = _non_ortho(nonOrthoMode)
    if useFaceTransform:
        raise NotImplementedError("face-transform pressure assembly is not implemented in pict_b200")
    domain._check_ready()
    dt = _time_step(timeStep, domain)
    check(_lib.load().pict_setup_pressure_rhs(ctypes.byref(domain._desc), dt, flags, int(bool(timeStepNorm)),
                                              _stream_ptr()), "SetupPressureRHS")


def SetupPressureRHSdiv(domain, timeStep, nonOrthoMode=0, useFaceTransform=False, timeStepNorm=False):
    flags = _non_ortho(nonOrthoMode)
    if useFaceTransform:
        raise NotImplementedError("face-transform pressure assembly is not implemented in pict_b200")
    domain._check_ready()
    dt = _time_step(timeStep, domain)
    check(_lib.load().pict_setup_pressure_rhs_div(ctypes.byref(domain._desc), dt, flags, int(bool(timeStepNorm)),
                                                  _stream_ptr()), "SetupPressureRHSdiv")


def CorrectVelocity(domain, timeStep, version=0, timeStepNorm=False):
    """u = H/A - grad(p)/A (extensions/PISO_multiblock_cuda_kernel.cu:6163-6201).  version 0/1: finite-difference
    pressure gradient (:5947-5980); 4: mean of the two face fluxes with orthogonal metrics (:6053-6160,
    always scaled by the time step); 5 / 6: finite-volume pressure gradient from interpolated cell
    fluxes / staggered face transforms (:6013-6050).  Every other number, including 2 and 3 (the
    reference's smoothing kernels, which it marks as not to be used and does not dispatch), takes the
    reference's default branch: the finite-difference corrector of version 1."""
    version = int(version)
    if version not in (4, 5, 6):
        version = 1
    domain._check_ready()
    if version in (5, 6):
        for b in domain.getBlocks():
            if not b.hasTransform():
                continue
            _check(version != 6 or b.hasFaceTransform(),
                   "CorrectVelocity version 6 needs the face transforms of transformed blocks (block %s)" % b.name)
            for f, bnd in enumerate(b.boundaries):
                _check(not isinstance(bnd, FixedBoundary) or bnd.hasTransform(),
                       "CorrectVelocity version %d needs the transform of fixed boundary %d of block %s" % (version, f, b.name))
    dt = _time_step(timeStep, domain)
    check(_lib.load().pict_correct_velocity(ctypes.byref(domain._desc), dt, version if version else 1,
                                            int(bool(timeStepNorm)), 0, _stream_ptr()), "CorrectVelocity")


def _copy(domain, fn, what):
    domain._check_ready()
    check(getattr(_lib.load(), fn)(ctypes.byref(domain._desc), _stream_ptr()), what)


def CopyVelocityResultToBlocks(domain):
    _copy(domain, "pict_copy_velocity_result_to_blocks", "CopyVelocityResultToBlocks")


def CopyVelocityResultFromBlocks(domain):
    _copy(domain, "pict_copy_velocity_result_from_blocks", "CopyVelocityResultFromBlocks")


def CopyPressureResultToBlocks(domain):
    _copy(domain, "pict_copy_pressure_result_to_blocks", "CopyPressureResultToBlocks")


def CopyPressureResultFromBlocks(domain):
    _copy(domain, "pict_copy_pressure_result_from_blocks", "CopyPressureResultFromBlocks")


def CopyScalarResultToBlocks(domain):
    """The blocks' passive scalar = scalarResult (extensions/PISO_multiblock_cuda_kernel.cu:6543-6733)."""
    domain._check_ready()
    _check_scalar(domain, "CopyScalarResultToBlocks")
    check(_lib.load().pict_copy_scalar_result(ctypes.byref(domain._desc), 1, _stream_ptr()), "CopyScalarResultToBlocks")


def CopyScalarResultFromBlocks(domain):
    """scalarResult = the blocks' passive scalar."""
    domain._check_ready()
    _check_scalar(domain, "CopyScalarResultFromBlocks")
    check(_lib.load().pict_copy_scalar_result(ctypes.byref(domain._desc), 0, _stream_ptr()), "CopyScalarResultFromBlocks")


# ------------------------------------------------------------------------------------------------
# gradient operators (extensions/PISOtorch.cpp:566-593).  They read the gradient fields of the domain
# (AGrad, CGrad, PGrad, velocityRHSGrad, velocityResultGrad, pressureRHSGrad, pressureRHSdivGrad,
# pressureResultGrad) and add to the gradient fields of their inputs (blocks' velocity / source /
# viscosity / pressure gradients, boundaries' velocity gradients, the domain's viscosity gradient and
# the global gradient vectors), except where the reference assigns: CorrectVelocityGrad writes
# AGrad and pressureRHSGrad, the Copy*GradFromBlocks / ToBlocks operators copy.  As with the
# reference, call the matching Create*Grad first for a fresh gradient.  Computed by the same adjoint
# kernels as the autograd Functions of pict_b200.PISOtorch_diff; with nonOrthoFlags the gradients of
# the non-orthogonal terms are added as the reference adds them: the explicit right-hand-side terms
# to velocityResultGrad / pressureResultGrad, the coefficients to the viscosity gradients / AGrad.
# Passive scalars have raw gradient operators (SetupAdvectionScalarGrad, the forPassiveScalar matrix
# gradient, CopyScalarResultGrad*).
# ------------------------------------------------------------------------------------------------

def _need_grad(domain, name, n):
    t = getattr(domain, name)
    if t is None or t.numel() != n:
        setattr(domain, name, torch.zeros(n, dtype=domain.getDtype(), device=domain.getDevice()))
    return getattr(domain, name)


def _nonortho_grad(domain, flags, what, out_bar, A_bar=None, data_bar=None, coef_bar=None, vb=None, name=""):
    """Add the gradient of the non-orthogonal terms of one operator (pict_nonortho_grad)."""
    from .PISOtorch_diff import _p, _stream
    if flags == 0:
        return
    check(_lib.load().pict_nonortho_grad(ctypes.byref(domain._desc), flags, what, _p(out_bar), _p(A_bar), _p(data_bar),
                                         _p(coef_bar), _p(vb), _stream()), name)


def _add_parameter_grads(domain, g):
    """Add the accumulators of a PISOtorch_diff._Grads to the blocks', boundaries' and domain's gradients."""
    blocks = domain.getBlocks()
    D = domain.getSpatialDims()

    def same(t, like):
        return t is not None and like is not None and t.numel() > 0 and t.shape == like.shape

    old_v = [b.velocityGrad if same(b.velocityGrad, b.velocity) else None for b in blocks]
    old_s = [b.velocitySourceGrad if same(b.velocitySourceGrad, b.velocitySource) else None for b in blocks]
    old_n = [b.viscosityGrad if same(b.viscosityGrad, b.viscosity) else None for b in blocks]
    old_f = [[b.boundaries[f].velocityGrad if (isinstance(b.boundaries[f], FixedBoundary)
              and same(b.boundaries[f].velocityGrad, b.boundaries[f].velocity)) else None for f in range(2 * D)]
             for b in blocks]
    keys = [("VISCOSITY",)]
    nu = g.to_inputs(keys)[0]
    for b, ov, os_, on, of in zip(blocks, old_v, old_s, old_n, old_f):
        if ov is not None:
            b.setVelocityGrad(b.velocityGrad + ov)
        if os_ is not None and b.velocitySourceGrad is not None:
            b.setVelocitySourceGrad(b.velocitySourceGrad + os_)
        if on is not None and b.viscosityGrad is not None:
            b.setViscosityGrad(b.viscosityGrad + on)
        for f in range(2 * D):
            if of[f] is not None:
                b.boundaries[f].setVelocityGrad(b.boundaries[f].velocityGrad + of[f])
    nu = nu.reshape(domain.viscosity.shape).to(domain.viscosity.device, domain.viscosity.dtype)
    if domain.viscosityGrad is not None and domain.viscosityGrad.shape == nu.shape:
        domain.viscosityGrad = domain.viscosityGrad + nu
    else:
        domain.viscosityGrad = nu
    domain.UpdateDomainData()


def _face_cells(block, f):
    """Global indices of the block's cells on face f, in the face's flat order (x fastest, face axis dropped)."""
    key = (f, block.globalOffset)
    cache = block.__dict__.setdefault("_face_cells_cache", {})
    if key not in cache:
        dims = block.getSpatialDims()
        zyx = list(block.pressure.shape[2:])
        idx = np.arange(int(np.prod(zyx))).reshape(zyx)
        ax = dims - 1 - (f >> 1)
        sl = [slice(None)] * dims
        sl[ax] = slice(-1, None) if f & 1 else slice(0, 1)
        cache[key] = torch.as_tensor(idx[tuple(sl)].reshape(-1) + block.globalOffset, device=block.velocity.device)
    return cache[key]


def _add_boundary_scalar_grads(domain, sb):
    """Per-adjacent-cell boundary scalar adjoints sb [2D][C][N] to the fixed faces' passive scalar gradients
    (static scalars receive the sum; extensions/PISO_multiblock_cuda_kernel.cu:2448-2476)."""
    C = domain.getPassiveScalarChannels()
    for b in domain.getBlocks():
        for f, bnd in enumerate(b.boundaries):
            if not isinstance(bnd, FixedBoundary) or bnd.passiveScalar is None:
                continue
            g = bnd.passiveScalarGrad
            if g is None or g.shape != bnd.passiveScalar.shape:
                continue
            vals = sb[f][:, _face_cells(b, f)]
            add = vals.sum(dim=1).reshape(g.shape) if bnd.passiveScalar.dim() == 2 else vals.reshape(g.shape)
            bnd.setPassiveScalarGrad(g + add)


def _add_scalar_viscosity_grad(domain, per_channel):
    """Scalar viscosity adjoint per channel [C] to passiveScalarViscosityGrad when it exists, else to the domain
    viscosity gradient (scatterViscosity_GRAD, extensions/PISO_multiblock_cuda_kernel.cu:1832-1849)."""
    g = domain.passiveScalarViscosityGrad
    if g is not None:
        add = per_channel.sum() if g.numel() == 1 else per_channel
        domain.passiveScalarViscosityGrad = g + add.reshape(g.shape).to(g.device, g.dtype)
    else:
        v = domain.viscosityGrad if domain.viscosityGrad is not None else torch.zeros_like(domain.viscosity)
        domain.viscosityGrad = v + per_channel.sum().reshape(v.shape).to(v.device, v.dtype)


def SetupAdvectionScalarGrad(domain, timeStep, nonOrthoFlags):
    """Gradient of SetupAdvectionScalar (extensions/PISO_multiblock_cuda_kernel.cu:4185-4278): scalarRHSGrad to the
    blocks' passive scalar gradients (assigned, as in the reference), the fixed faces' scalar and velocity
    gradients, the scalar viscosity gradient and, with non-orthogonal RHS flags, scalarResultGrad."""
    from .PISOtorch_diff import _Grads, _p, _stream
    flags = _non_ortho(nonOrthoFlags)
    domain._check_ready()
    _check_scalar(domain, "SetupAdvectionScalarGrad")
    dt = _time_step(timeStep, domain)
    g = _Grads(domain)
    C, N, D = domain.getPassiveScalarChannels(), g.N, g.D
    rb = _need_grad(domain, "scalarRHSGrad", C * N).contiguous()
    sres = _need_grad(domain, "scalarResultGrad", C * N)
    s_bar, sb, nu = g.z(C * N), g.z(2 * D * C * N), g.z(C * N)
    check(_lib.load().pict_scalar_grad(ctypes.byref(domain._desc), dt, flags, 1, 0, _p(rb), None, None, _p(s_bar),
                                       _p(sres), _p(sb), _p(g.vb), _p(nu), _stream()), "SetupAdvectionScalarGrad")
    s_bar = s_bar.reshape(C, N)
    for b in domain.getBlocks():
        n = b.pressure.numel()
        b.setPassiveScalarGrad(s_bar[:, b.globalOffset:b.globalOffset + n].reshape(b.passiveScalar.shape).contiguous())
    _add_boundary_scalar_grads(domain, sb.reshape(2 * D, C, N))
    _add_scalar_viscosity_grad(domain, nu.reshape(C, N).sum(dim=1))
    _add_parameter_grads(domain, g)


def SetupAdvectionMatrixGrad(domain, timeStep, nonOrthoFlags, forPassiveScalar=False, passiveScalarChannel=0):
    """Gradient of SetupAdvectionMatrix (extensions/PISO_multiblock_cuda_kernel.cu:3869-4077): AGrad and CGrad to the
    velocity, viscosity and boundary velocity gradients; with ``forPassiveScalar`` to the velocity and the
    scalar viscosity gradient of ``passiveScalarChannel``."""
    from .PISOtorch_diff import _Grads, _p, _stream
    flags = _non_ortho(nonOrthoFlags)
    if forPassiveScalar:
        domain._check_ready()
        _check_scalar(domain, "SetupAdvectionMatrixGrad")
        dt = _time_step(timeStep, domain)
        ch = int(passiveScalarChannel)
        _check(0 <= ch < domain.getPassiveScalarChannels(), "passiveScalarChannel out of range.")
        g = _Grads(domain)
        nu = g.z(g.N)
        check(_lib.load().pict_scalar_grad(ctypes.byref(domain._desc), dt, flags, 0, ch, _p(domain.CGrad.coef.contiguous()),
                                           _p(_need_grad(domain, "AGrad", g.N).contiguous()), _p(g.un), None, None,
                                           None, None, _p(nu), _stream()), "SetupAdvectionMatrixGrad")
        per = torch.zeros(domain.getPassiveScalarChannels(), dtype=nu.dtype, device=nu.device)
        per[ch] = nu.sum()
        _add_scalar_viscosity_grad(domain, per)
        _add_parameter_grads(domain, g)
        return
    domain._check_ready()
    dt = _time_step(timeStep, domain)
    g = _Grads(domain)
    zD = g.z(g.D * g.N)
    Ab = _need_grad(domain, "AGrad", g.N).contiguous()
    Cb = domain.CGrad.coef.contiguous()
    check(_lib.load().pict_advection_grad(ctypes.byref(domain._desc), dt, _p(zD), _p(zD), _p(Cb),
                                          _p(Ab), _p(g.un), _p(g.nu), _p(g.vb), None, _stream()),
          "SetupAdvectionMatrixGrad")
    _nonortho_grad(domain, flags, 0, Cb, A_bar=Ab, coef_bar=g.nu, name="SetupAdvectionMatrixGrad")
    _add_parameter_grads(domain, g)


def SetupAdvectionVelocityGrad(domain, timeStep, nonOrthoFlags, applyPressureGradient=False):
    """Gradient of SetupAdvectionVelocity (extensions/PISO_multiblock_cuda_kernel.cu:4388-4478): velocityRHSGrad to the
    velocity, source, viscosity and boundary velocity gradients, and with non-orthogonal RHS flags to
    velocityResultGrad (the explicit terms read domain.velocityResult).  applyPressureGradient is accepted
    like the reference's kernel accepts it, which does not differentiate the pressure term (-dt grad p):
    the outputs are the same with and without it.  PISOtorch_diff.SetupAdvectionVelocity adds the
    gradient of that term with respect to the blocks' pressure."""
    from .PISOtorch_diff import _Grads, _p, _stream
    flags = _non_ortho(nonOrthoFlags)
    domain._check_ready()
    dt = _time_step(timeStep, domain)
    g = _Grads(domain)
    zD = g.z(g.D * g.N)
    rb = _need_grad(domain, "velocityRHSGrad", g.D * g.N).contiguous()
    check(_lib.load().pict_advection_grad(ctypes.byref(domain._desc), dt, _p(zD), _p(rb), _p(g.z((2 * g.D + 1) * g.N)),
                                          _p(g.z(g.N)), _p(g.un), _p(g.nu), _p(g.vb), _p(g.src), _stream()),
          "SetupAdvectionVelocityGrad")
    if flags & (NON_ORTHO_DIRECT_RHS | NON_ORTHO_DIAGONAL_RHS):
        ub = _need_grad(domain, "velocityResultGrad", g.D * g.N)
        _nonortho_grad(domain, flags, 1, rb, data_bar=ub, coef_bar=g.nu, vb=g.vb, name="SetupAdvectionVelocityGrad")
    _add_parameter_grads(domain, g)


def SetupPressureMatrixGrad(domain, timeStep, nonOrthoMode=0, useFaceTransform=False):
    """Gradient of SetupPressureMatrix (extensions/PISO_multiblock_cuda_kernel.cu:4967-5117): PGrad to AGrad."""
    from .PISOtorch_diff import _p, _stream
    flags = _non_ortho(nonOrthoMode)
    if useFaceTransform:
        raise NotImplementedError("face-transform pressure assembly is not implemented in pict_b200")
    domain._check_ready()
    _time_step(timeStep, domain)
    Ab = _need_grad(domain, "AGrad", domain.getTotalSize())
    add = torch.zeros_like(Ab)
    Pb = domain.PGrad.coef.contiguous()
    check(_lib.load().pict_pressure_matrix_grad(ctypes.byref(domain._desc), _p(domain.A), _p(Pb),
                                                _p(add), _stream()), "SetupPressureMatrixGrad")
    _nonortho_grad(domain, flags, 2, Pb, coef_bar=add, name="SetupPressureMatrixGrad")
    domain.AGrad = Ab + add


def _pressure_rhs_grad(domain, dt, with_rhs, what, flags=0, time_step_norm=False):
    from .PISOtorch_diff import _Grads, _p, _stream
    lib = _lib.load()
    g = _Grads(domain)
    N, D = g.N, g.D
    desc = ctypes.byref(domain._desc)
    st = _stream()
    hb = _need_grad(domain, "pressureRHSGrad", D * N).detach().clone().contiguous()
    div_grad = _need_grad(domain, "pressureRHSdivGrad", N).contiguous()
    if flags & (NON_ORTHO_DIRECT_RHS | NON_ORTHO_DIAGONAL_RHS):
        # explicit terms of pressureResult (k_pressureRHSaddNonOrthoComponents_GRAD)
        pb = _need_grad(domain, "pressureResultGrad", N)
        Ab = _need_grad(domain, "AGrad", N)
        _nonortho_grad(domain, flags, 3, div_grad, data_bar=pb, coef_bar=Ab, name=what)
    if time_step_norm:
        # the divergence was divided by the time step, the non-orthogonal terms added after it are not
        # (k_computePressureRHSdivergenceFromFlux_GRAD, extensions/PISO_multiblock_cuda_kernel.cu:5424-5448)
        div_grad = (div_grad / dt).contiguous()
    check(lib.pict_divergence_grad(desc, _p(div_grad), _p(hb), _p(g.vb), st), what)
    # the divergence gradient stays in pressureRHSGrad, as the reference scatters it there in place
    domain.pressureRHSGrad = hb
    if not with_rhs:
        _add_parameter_grads(domain, g)
        return
    Ab, Cb, Ub = g.z(N), g.z((2 * D + 1) * N), g.z(D * N)
    zN = g.z(N)
    check(lib.pict_pressure_rhs_grad(desc, dt, _p(hb), _p(domain.pressureRHS), _p(domain.A), _p(domain.C.coef),
                                     _p(domain.velocityResult), _p(zN), _p(zN), _p(Ab), _p(Cb), _p(Ub), _p(g.un),
                                     _p(g.src), _p(g.nu), _p(g.vb), st), what)
    domain.AGrad = _need_grad(domain, "AGrad", N) + Ab
    domain.CGrad.setCoef(domain.CGrad.coef + Cb.reshape(domain.CGrad.coef.shape))
    domain.velocityResultGrad = _need_grad(domain, "velocityResultGrad", D * N) + Ub
    _add_parameter_grads(domain, g)


def SetupPressureRHSGrad(domain, timeStep, nonOrthoMode=0, useFaceTransform=False, timeStepNorm=False):
    """Gradient of SetupPressureRHS (h = H/A and its divergence, extensions/PISO_multiblock_cuda_kernel.cu:5243-5453):
    pressureRHSGrad and pressureRHSdivGrad to AGrad, CGrad, velocityResultGrad and the velocity, source,
    viscosity and boundary velocity gradients; with timeStepNorm the divergence's gradient is divided by
    the time step."""
    flags = _non_ortho(nonOrthoMode)
    if useFaceTransform:
        raise NotImplementedError("SetupPressureRHSGrad: no gradient with face transforms")
    domain._check_ready()
    _pressure_rhs_grad(domain, _time_step(timeStep, domain), True, "SetupPressureRHSGrad", flags, bool(timeStepNorm))


def SetupPressureRHSdivGrad(domain, timeStep, nonOrthoMode=0, useFaceTransform=False, timeStepNorm=False):
    """Gradient of SetupPressureRHSdiv (extensions/PISO_multiblock_cuda_kernel.cu:5423-5453): pressureRHSdivGrad to
    pressureRHSGrad and the boundary velocity gradients."""
    flags = _non_ortho(nonOrthoMode)
    if useFaceTransform:
        raise NotImplementedError("SetupPressureRHSdivGrad: no gradient with face transforms")
    domain._check_ready()
    _pressure_rhs_grad(domain, _time_step(timeStep, domain), False, "SetupPressureRHSdivGrad", flags,
                       bool(timeStepNorm))


def SetupPressureCorrectionGrad(domain, timeStep, nonOrthoMode=0, useFaceTransform=False, timeStepNorm=False):
    """Gradient of SetupPressureCorrection: SetupPressureMatrixGrad followed by SetupPressureRHSGrad."""
    SetupPressureMatrixGrad(domain, timeStep, nonOrthoMode, useFaceTransform)
    SetupPressureRHSGrad(domain, timeStep, nonOrthoMode, useFaceTransform, timeStepNorm)


def CorrectVelocityGrad(domain, timeStep, timeStepNorm=False):
    """Gradient of CorrectVelocity (FD version, extensions/PISO_multiblock_cuda_kernel.cu:6251-6293): velocityResultGrad
    to pressureRHSGrad and AGrad (assigned, as in the reference) and the blocks' pressure gradients (added);
    with timeStepNorm the pressure and A gradients carry the time step factor."""
    from .PISOtorch_diff import _p, _stream
    domain._check_ready()
    dt = _time_step(timeStep, domain)
    lib = _lib.load()
    N, D = domain.getTotalSize(), domain.getSpatialDims()
    z = lambda n: torch.zeros(n, dtype=domain.getDtype(), device=domain.getDevice())
    ug = _need_grad(domain, "velocityResultGrad", D * N).contiguous()
    p_glob = z(N)
    check(lib.pict_copy_field(ctypes.byref(domain._desc), 1, 0, _p(p_glob), 0, _stream()), "CorrectVelocityGrad")
    Ab, pb, hb = z(N), z(N), z(D * N)
    # timeStepNorm: the pressure update was multiplied by the time step, the pressureRHS term was not
    # (PISO_update_velocity_GRAD, extensions/PISO_multiblock_cuda_kernel.cu:6270-6283)
    ug_update = (ug * dt).contiguous() if timeStepNorm else ug
    check(lib.pict_correct_velocity_grad(ctypes.byref(domain._desc), _p(domain.A), _p(p_glob), _p(ug_update), _p(Ab),
                                         _p(pb), _p(hb), _stream()), "CorrectVelocityGrad")
    domain.AGrad = Ab
    domain.pressureRHSGrad = ug.clone() if timeStepNorm else hb
    for b in domain.getBlocks():
        if b.pressureGrad is None or b.pressureGrad.shape != b.pressure.shape:
            b.setPressureGrad(torch.zeros_like(b.pressure))
    domain.UpdateDomainData()
    check(lib.pict_copy_field(ctypes.byref(domain._desc), 4, 1, _p(pb), 1, _stream()), "CorrectVelocityGrad")


def _copy_grad(domain, which, to_blocks, name, n):
    from .PISOtorch_diff import _p, _stream
    domain._check_ready()
    if to_blocks:
        vec = _need_grad(domain, name, n).contiguous()
        for b in domain.getBlocks():
            if which == 3 and (b.velocityGrad is None or b.velocityGrad.shape != b.velocity.shape):
                b.setVelocityGrad(torch.zeros_like(b.velocity))
        domain.UpdateDomainData()
        check(_lib.load().pict_copy_field(ctypes.byref(domain._desc), which, 1, _p(vec), 0, _stream()), name)
    else:
        out = torch.zeros(n, dtype=domain.getDtype(), device=domain.getDevice())
        check(_lib.load().pict_copy_field(ctypes.byref(domain._desc), which, 0, _p(out), 0, _stream()), name)
        setattr(domain, name, out)


def CopyVelocityResultGradFromBlocks(domain):
    """velocityResultGrad = the blocks' velocity gradients (gradient of CopyVelocityResultToBlocks)."""
    _copy_grad(domain, 3, False, "velocityResultGrad", domain.getTotalSize() * domain.getSpatialDims())


def CopyVelocityResultGradToBlocks(domain):
    """The blocks' velocity gradients = velocityResultGrad (gradient of CopyVelocityResultFromBlocks)."""
    _copy_grad(domain, 3, True, "velocityResultGrad", domain.getTotalSize() * domain.getSpatialDims())


def CopyPressureResultGradFromBlocks(domain):
    """pressureResultGrad = the blocks' pressure gradients (gradient of CopyPressureResultToBlocks)."""
    _copy_grad(domain, 4, False, "pressureResultGrad", domain.getTotalSize())


def CopyScalarResultGradFromBlocks(domain):
    """scalarResultGrad = the blocks' passive scalar gradients (gradient of CopyScalarResultToBlocks)."""
    domain._check_ready()
    _check_scalar(domain, "CopyScalarResultGradFromBlocks")
    C = domain.getPassiveScalarChannels()
    parts = [(b.passiveScalarGrad if b.passiveScalarGrad is not None and b.passiveScalarGrad.numel() > 0
              else torch.zeros_like(b.passiveScalar)).reshape(C, -1) for b in domain.getBlocks()]
    domain.scalarResultGrad = torch.cat(parts, dim=1).reshape(-1).contiguous()


def CopyScalarResultGradToBlocks(domain):
    """The blocks' passive scalar gradients = scalarResultGrad (gradient of CopyScalarResultFromBlocks)."""
    domain._check_ready()
    _check_scalar(domain, "CopyScalarResultGradToBlocks")
    C, N = domain.getPassiveScalarChannels(), domain.getTotalSize()
    g = _need_grad(domain, "scalarResultGrad", C * N).reshape(C, N)
    for b in domain.getBlocks():
        n = b.pressure.numel()
        b.setPassiveScalarGrad(g[:, b.globalOffset:b.globalOffset + n].reshape(b.passiveScalar.shape).clone())
    domain.UpdateDomainData()


def SGSviscosityIncompressibleSmagorinsky(domain, coefficient):
    """Smagorinsky sub-grid-scale viscosity per block (extensions/PISO_multiblock_cuda_kernel.cu:6896-7019): for each
    block a tensor shaped like its pressure with coefficient * delta * |S|, |S| = sqrt(2 S:S) of the
    blocks' velocity and delta the largest squared column length of the cell transform (1 without one).
    ``coefficient`` is a host tensor of shape [1]."""
    domain._check_ready()
    _check(isinstance(coefficient, torch.Tensor) and not coefficient.is_cuda, "coefficient must be a host tensor")
    _check(coefficient.dim() == 1 and coefficient.size(0) == 1, "coefficient tensor must have shape [1]")
    out = torch.empty(domain.getTotalSize(), dtype=domain.getDtype(), device=domain.getDevice())
    check(_lib.load().pict_sgs_smagorinsky(ctypes.byref(domain._desc), float(coefficient[0]), _ptr(out), _stream_ptr()),
          "SGSviscosityIncompressibleSmagorinsky")
    res = []
    for b in domain.getBlocks():
        n = b.pressure.numel()
        res.append(out[b.globalOffset:b.globalOffset + n].reshape(b.pressure.shape).clone())
    return res


def ComputeVelocityDivergence(domain):
    """Flux divergence of the blocks' velocity (extensions/PISO_multiblock_cuda_kernel.cu:6333-6388)."""
    domain._check_ready()
    out = torch.zeros_like(domain.pressureResult)
    check(_lib.load().pict_velocity_divergence(ctypes.byref(domain._desc), _ptr(out), _stream_ptr()),
          "ComputeVelocityDivergence")
    return out


def CoordsToTransforms(coords):
    """Cell transforms (M, Minv, det) from vertex coordinates (extensions/grid_gen.cu:341-375)."""
    _check(coords.is_cuda and coords.is_contiguous(), "coords must be a contiguous CUDA tensor")
    _check(2 < coords.dim() < 6, "coords must have batch and channel dimension and be 1-3D.")
    _check(coords.size(0) == 1, "coords batch dimension must be 1.")
    dims = coords.dim() - 2
    _check(coords.size(1) == dims, "coords channel dimension must match spatial dimensionality.")
    size = [coords.size(-1 - d) - 1 for d in range(dims)]
    out = torch.zeros([1] + [size[dims - 1 - d] for d in range(dims)] + [_transform_size(dims)],
                      dtype=coords.dtype, device=coords.device)
    sz = (ctypes.c_int32 * 3)(*(size + [1] * (3 - dims)))
    check(_lib.load().pict_coords_to_transforms(_ptr(coords), dims, sz, _dtype_code(coords.dtype), _ptr(out),
                                                _stream_ptr()), "CoordsToTransforms")
    return out


def CoordsToFaceTransforms(coords):
    """Staggered face transforms from vertex coordinates (extensions/grid_gen.cu:468-514)."""
    _check(coords.is_cuda and coords.is_contiguous(), "coords must be a contiguous CUDA tensor")
    dims = coords.dim() - 2
    size = [coords.size(-1 - d) - 1 for d in range(dims)]
    out = torch.zeros([1, dims] + list(coords.shape[2:]) + [_transform_size(dims)], dtype=coords.dtype,
                      device=coords.device)
    sz = (ctypes.c_int32 * 3)(*(size + [1] * (3 - dims)))
    check(_lib.load().pict_coords_to_face_transforms(_ptr(coords), dims, sz, _dtype_code(coords.dtype), _ptr(out),
                                                     _stream_ptr()), "CoordsToFaceTransforms")
    return out


def TransformVectors(vectors, transforms, inverse=False):
    """Per-cell vector transform (extensions/PISO_multiblock_cuda_kernel.cu:7152-7224): M u, or Minv u with ``inverse``."""
    dims = vectors.size(1)
    tr = transforms.reshape(-1, _transform_size(dims))
    off = dims * dims if inverse else 0
    M = tr[:, off:off + dims * dims].reshape(-1, dims, dims)
    v = torch.movedim(vectors, 1, -1).reshape(-1, dims, 1)
    out = torch.bmm(M, v).reshape(list(vectors.shape[:1]) + list(vectors.shape[2:]) + [dims])
    return torch.movedim(out, -1, 1).contiguous()


# ------------------------------------------------------------------------------------------------
# linear solves (extensions/PISOtorch.cpp:559-563 -> extensions/PISO_multiblock_cuda_kernel.cu:7021-7103)
# ------------------------------------------------------------------------------------------------

_warned = set()


def _warn_once(key, msg):
    if key not in _warned:
        _warned.add(key)
        warnings.warn(msg)


class _Workspace:
    """Scratch memory for the Krylov kernels, allocated through torch's caching allocator."""

    def __init__(self):
        self.buf = None

    def get(self, nbytes, device):
        if self.buf is None or self.buf.numel() < nbytes or self.buf.device != device:
            self.buf = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        return self.buf


def _solve_params(nrhs, maxit, tol, conv, use_bicg, transpose, x_zero=False, subtract_mean=False,
                  write_block_pressure=False, group_size=0, threads=0, variant=0, residual_reset=0,
                  return_best=False, rank_deficient=False):
    p = SolveParams()
    p.max_iterations = int(maxit)
    p.use_bicg = int(bool(use_bicg))
    p.nrhs = int(nrhs)
    p.x_is_zero = int(bool(x_zero))
    p.transpose = int(bool(transpose))
    p.convergence = int(conv)
    p.group_size = int(group_size)
    p.threads = int(threads)
    p.subtract_mean = int(bool(subtract_mean))
    p.write_block_pressure = int(bool(write_block_pressure))
    p.variant = int(variant)
    p.residual_reset_steps = max(int(residual_reset), 0)
    p.return_best_result = int(bool(return_best))
    p.rank_deficient = int(bool(rank_deficient))
    p.tolerance = float(tol)
    return p


def solve_stencil(domain, coef, rhs, x, params, info=None, stream=None):
    """Launch one stencil solve on the domain's topology (no host synchronisation).

    rhs and x are [nrhs*N] device vectors; returns the device info tensor ([nrhs] SolveInfo records).
    """
    lib = _lib.load()
    desc = domain._desc
    ws_bytes = lib.pict_solve_workspace_bytes(ctypes.byref(desc), ctypes.byref(params))
    _check(ws_bytes > 0, "solve: invalid workspace size")
    ws = domain.__dict__.setdefault("_ws", _Workspace()).get(ws_bytes, coef.device)
    if info is None:
        info = torch.empty(params.nrhs * desc.num_sims * _lib.SOLVE_INFO_BYTES, dtype=torch.uint8, device=coef.device)
    st = _stream_ptr() if stream is None else stream
    check(lib.pict_solve(ctypes.byref(desc), _ptr(coef), _ptr(rhs), _ptr(x), ctypes.byref(params), _ptr(info),
                         _ptr(ws), ws_bytes, st), "SolveLinear")
    return info


def decode_infos(info_tensor):
    raw = info_tensor.cpu().numpy().tobytes()
    n = len(raw) // _lib.SOLVE_INFO_BYTES
    arr = (SolveInfo * n).from_buffer_copy(raw)
    out = []
    for r in arr:
        li = LinearSolverResultInfo(r.final_residual, r.used_iterations, bool(r.converged), bool(r.finite))
        li.status = int(r.status)
        out.append(li)
    return out


def SolveLinear(A, RHS, x, maxIterations=1000, tolerance=1e-8, convergenceCriterion=ConvergenceCriterion.NORM2_NORMALIZED,
                useBiCG=False, matrixRankDeficient=False, residualResetSteps=0, transposeA=False, printResidual=False,
                returnBestResult=False, BiCGwithPreconditioner=True):
    """Solve A x = RHS for every length-n slice of RHS; returns one LinearSolverResultInfo per slice."""
    _check(isinstance(A, StencilMatrix), "SolveLinear: A must be a system matrix of a prepared domain (domain.C, domain.P or a copy).")
    domain = A._domain()
    n = A.getRows()
    _check(RHS.is_cuda and RHS.is_contiguous(), "RHS must be a contiguous CUDA tensor")
    _check(RHS.dim() == 1, "RHS must be a vector.")
    _check(RHS.size(0) % n == 0, "Size of RHS must be a multiple of the matrix size.")
    _check(RHS.dtype == A.getDtype(), "Data type of RHS must match A.")
    _check(x.is_cuda and x.is_contiguous() and x.dim() == 1, "x must be a vector.")
    _check(x.size(0) == RHS.size(0), "Size of x must match RHS.")
    _check(x.dtype == A.getDtype(), "Data type of x must match A.")
    maxit = int(_as_scalar(maxIterations))
    tol = float(_as_scalar(tolerance))
    conv = int(convergenceCriterion)
    _check(0 <= conv <= 4, "Unknown convergence criterion.")
    if domain.IsTensorChanged():
        raise RuntimeError("Domain's tensors have been changed, use UpdateDomain() to set the new pointers.")
    domain._desc = domain._make_desc()
    nb = RHS.size(0) // n
    if useBiCG and BiCGwithPreconditioner:
        infos = _solve_bicgstab_ilu(domain, A, RHS, x, nb, maxit, tol, conv, bool(transposeA))
        if printResidual:
            for i, inf in enumerate(infos):
                print("BiCG (ILU) RHS %d: %s" % (i, inf))
        return infos
    infos = []
    coef = A.coef.contiguous()
    if useBiCG:
        p = _solve_params(nb, maxit, tol, conv, True, transposeA)
        info = solve_stencil(domain, coef, RHS, x, p)
        infos = decode_infos(info)
    else:
        for k in range(nb):
            p = _solve_params(1, maxit, tol, conv, False, transposeA, residual_reset=int(residualResetSteps),
                              return_best=bool(returnBestResult), rank_deficient=bool(matrixRankDeficient))
            info = solve_stencil(domain, coef, RHS[k * n:(k + 1) * n], x[k * n:(k + 1) * n], p)
            infos.extend(decode_infos(info))
    if printResidual:
        for i, inf in enumerate(infos):
            print("%sCG RHS %d: %s" % ("Bi" if useBiCG else "", i, inf))
    return infos


def _ilu_plan(domain):
    """Host analysis of the domain's CSR pattern for the ILU(0) solves (pict_ilu_analyze), once per domain:
    device arrays of the pattern, diagonal and transposed positions and level orders, host level starts."""
    plan = getattr(domain, "_ilu", None)
    row, index = domain._csr_structure()
    if plan is not None and plan["row"] is row:
        return plan
    lib = _lib.load()
    rh = row.cpu().numpy().astype(np.int32)
    ih = index.cpu().numpy().astype(np.int32)
    n, nnz = rh.size - 1, ih.size
    diag = np.empty(n, np.int32)
    tpos = np.empty(nnz, np.int32)
    of, ob = np.empty(n, np.int32), np.empty(n, np.int32)
    pf, pb = np.empty(n + 1, np.int32), np.empty(n + 1, np.int32)
    nlf, nlb = ctypes.c_int32(0), ctypes.c_int32(0)
    check(lib.pict_ilu_analyze(n, rh.ctypes.data, ih.ctypes.data, diag.ctypes.data, tpos.ctypes.data, of.ctypes.data,
                               pf.ctypes.data, ob.ctypes.data, pb.ctypes.data, ctypes.byref(nlf), ctypes.byref(nlb)),
          "ilu_analyze")
    dev = domain.getDevice()
    t = lambda a: torch.from_numpy(a).to(dev)
    plan = {"row": row, "index": index, "index_out": torch.empty_like(index), "n": n, "nnz": nnz, "diag": t(diag),
            "tpos": t(tpos), "order_f": t(of),
            "order_b": t(ob), "ptr_f": pf[:nlf.value + 1].copy(), "ptr_b": pb[:nlb.value + 1].copy(),
            "nlf": nlf.value, "nlb": nlb.value}
    domain._ilu = plan
    return plan


def _solve_bicgstab_ilu(domain, A, RHS, x, nb, maxit, tol, conv, transpose):
    """BiCGStab with the right preconditioner selected by SetBiCGPreconditioner (pict_bicgstab_ilu) on the
    CSR form of A; nb right-hand sides solved one after another with the same preconditioner, as the
    reference's bicgstabSolveGPU does."""
    _check(domain._desc.num_sims == 1, "SolveLinear: the preconditioned BiCGStab takes single-simulation domains")
    lib = _lib.load()
    plan = _ilu_plan(domain)
    n, nnz = plan["n"], plan["nnz"]
    dtype = domain.getDtype()
    aval = torch.empty(nnz, dtype=dtype, device=domain.getDevice())
    check(lib.pict_stencil_to_csr(ctypes.byref(domain._desc), _ptr(A.coef.contiguous()), _ptr(plan["row"]), _ptr(aval),
                                  _ptr(plan["index_out"]), _stream_ptr()), "stencil_to_csr")
    ws = torch.empty(int(lib.pict_bicgstab_ilu_workspace_bytes(n, nnz, _dtype_code(dtype))), dtype=torch.uint8,
                     device=domain.getDevice())
    info = (ctypes.c_uint8 * (_lib.SOLVE_INFO_BYTES * nb))()
    check(lib.pict_bicgstab_ilu(n, nnz, _dtype_code(dtype), _ptr(plan["row"]), _ptr(plan["index"]), _ptr(plan["diag"]),
                                _ptr(plan["tpos"]), _ptr(plan["order_f"]), plan["ptr_f"].ctypes.data, plan["nlf"],
                                _ptr(plan["order_b"]), plan["ptr_b"].ctypes.data, plan["nlb"], _ptr(aval), _ptr(RHS),
                                _ptr(x), nb, maxit, tol, conv, 0, int(transpose), int(_bicg_preconditioner),
                                ctypes.addressof(info), _ptr(ws),
                                ws.numel(), _stream_ptr()), "bicgstab_ilu")
    return decode_infos(torch.frombuffer(bytearray(info), dtype=torch.uint8))


def SparseOuterProduct(a, b, out_pattern):
    """out.value[ij] = a_i * b_j on the sparsity pattern of out (extensions/cg_solver_kernel.cu:869-908)."""
    _check(isinstance(out_pattern, StencilMatrix), "SparseOuterProduct: out_pattern must be a domain matrix")
    d = out_pattern._domain()
    N = out_pattern.getRows()
    coef = torch.empty_like(out_pattern.coef)
    coef[0] = a * b
    nbr = d._nbr.long()
    for f in range(2 * d.getSpatialDims()):
        j = nbr[f]
        ok = j >= 0
        coef[f + 1] = torch.where(ok, a * b[j.clamp(min=0)], torch.zeros_like(a))
    out_pattern.setCoef(coef)
