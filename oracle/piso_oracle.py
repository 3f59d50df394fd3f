"""FP64 CPU oracle of PICT's PISO time step (test infrastructure only).

This module is the checker for the CUDA implementation in ``pict_b200``: a
NumPy / SciPy-sparse restatement of the reference discretisation for the
PISO path (orthogonal, and with the non-orthogonal terms of ``nonOrthoFlags``), on single- and multi-block
structured grids with fixed (Dirichlet), periodic and connected boundaries and
optional per-cell coordinate transforms.  It is imported only by ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``; the
product path never calls it.

Every function cites the reference source it restates (paths relative to the
PICT repository):

* kernel.cu   = extensions/PISO_multiblock_cuda_kernel.cu
* cg.cu       = extensions/cg_solver_kernel.cu
* bicg.cu     = extensions/bicgstab_solver_kernel.cu
* grid_gen.cu = extensions/grid_gen.cu
* sim.py      = PISOtorch_simulation.py

Layout conventions (identical to the reference):

* faces / boundaries are indexed ``[-x, +x, -y, +y, -z, +z]`` = 0..2D-1,
  axis = face >> 1, upper side = face & 1 (extensions/PISO_multiblock_cuda_kernel.cu:196-225);
* cells of a block are flattened x-fastest; global vectors concatenate the
  blocks (``globalOffset``) and vector fields are component-major
  ``[D][N]`` (extensions/PISO_multiblock_cuda_kernel.cu:166-172);
* stencil coefficients are stored as ``coef[K][N]`` with K = 2D+1 in the order
  ``[diag, -x, +x, -y, +y, -z, +z]`` (the reference's ``rowValues`` order,
  extensions/PISO_multiblock_cuda_kernel.cu:3693-3694, before its CSR sort).

Pinning: golden fixtures produced by the reference's own CUDA build
(``tests/golden/``, generated by ``tests/golden/make_ref_fixtures.py``) are
compared against this oracle in ``tests/test_oracle_golden.py``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

FACE_NAMES = ["-x", "+x", "-y", "+y", "-z", "+z"]
AXIS_NAMES = ["x", "y", "z"]


def face_index(face) -> int:
    """Face string or index -> index (extensions/domain_structs.cpp:134-155)."""
    if isinstance(face, str):
        return FACE_NAMES.index(face)
    return int(face)


def axis_index(axis) -> int:
    if isinstance(axis, str):
        return AXIS_NAMES.index(axis)
    return int(axis)


# --------------------------------------------------------------------------
# transforms from vertex coordinates (grid_gen.cu)
# --------------------------------------------------------------------------

def _det_inv(M):
    """Determinant and inverse of a stack of DxD matrices."""
    det = np.linalg.det(M)
    inv = np.linalg.inv(M)
    return det, inv


def coords_to_transforms(coords: np.ndarray) -> np.ndarray:
    """Cell transforms from vertex coordinates, extensions/grid_gen.cu:284-339.

    coords: [1, D, (z+1), y+1, x+1] -> transforms [1, (z), y, x, 2D^2+1] with
    per cell M (row-major, M[i][k] = d x_i / d xi_k from the difference of the
    opposite face centres), Minv and det(M).
    """
    c = np.asarray(coords, dtype=np.float64)
    D = c.shape[1]
    v = c[0]  # [D, (z+1), y+1, x+1]
    # face centres: average of the 2^(D-1) vertices of each face
    sl = lambda lo_hi, ax: tuple(
        (slice(1, None) if lo_hi else slice(0, -1)) if a == ax else slice(None) for a in range(D))
    # move to cell-centred index space with explicit loops over the vertex corners
    cell_shape = tuple(s - 1 for s in v.shape[1:])
    M = np.zeros(cell_shape + (D, D))
    for k in range(D):  # direction
        # numpy axis of direction k in the spatial array (zyx order)
        nax = D - 1 - k
        upper = np.zeros((D,) + cell_shape)
        lower = np.zeros((D,) + cell_shape)
        for corner in range(1 << D):
            idx = []
            for n in range(D):  # numpy spatial axis n -> direction D-1-n
                kk = D - 1 - n
                bit = (corner >> kk) & 1
                idx.append(slice(1, None) if bit else slice(0, -1))
            val = v[(slice(None),) + tuple(idx)]
            if (corner >> k) & 1:
                upper += val
            else:
                lower += val
        norm = 1.0 / (1 << (D - 1))
        diff = (upper - lower) * norm  # [D(comp), cells]
        for i in range(D):
            M[..., i, k] = diff[i]
    det, inv = _det_inv(M)
    T = np.concatenate([M.reshape(cell_shape + (D * D,)), inv.reshape(cell_shape + (D * D,)),
                        det[..., None]], axis=-1)
    return T[None]


def coords_to_face_transforms(coords: np.ndarray) -> np.ndarray:
    """Face transforms (staggered), extensions/grid_gen.cu:383-466.

    Returns [1, D, (z+1), y+1, x+1, 2D^2+1]; channel ``dim`` holds the transform
    of the lower face of cell ``pos`` along ``dim``.  Entries whose tangential
    index is the last vertex index are left zero (extensions/grid_gen.cu:392-397).
    """
    c = np.asarray(coords, dtype=np.float64)
    D = c.shape[1]
    v = c[0]
    vshape = v.shape[1:]  # zyx vertex grid
    size = np.array(list(reversed(vshape)))  # x,y,z vertex counts
    n = int(np.prod(vshape))
    grids = np.meshgrid(*[np.arange(s) for s in vshape], indexing="ij")
    P = np.stack([grids[D - 1 - a].reshape(-1) for a in range(D)], 1)  # (n, D) xyz
    nfv = 1 << (D - 1)
    nev = 1 << max(D - 2, 0)

    def gather(Q):
        Qc = np.clip(Q, 0, size - 1)
        idx = tuple(Qc[:, D - 1 - m] for m in range(D))
        return v[(slice(None),) + idx].T  # (n, D comp)

    out = np.zeros((D, n, 2 * D * D + 1))
    for dim in range(D):
        valid = np.ones(n, dtype=bool)
        for i in range(1, D):
            t_ax = (dim + i) % D
            valid &= P[:, t_ax] != size[t_ax] - 1
        t = np.zeros((n, D, D))
        norm_w = np.full(n, 0.5)
        for is_upper in range(2):
            sign = 2 * is_upper - 1
            at_b = (P[:, dim] == size[dim] - 1) if is_upper else (P[:, dim] == 0)
            F = P.copy()
            F[:, dim] += np.where(at_b, 0, sign)
            norm_w = np.where(at_b, 1.0, norm_w)
            for vi in range(nfv):
                Vp = F.copy()
                for i in range(1, D):
                    Vp[:, (dim + i) % D] += 1 if (vi & i) != 0 else 0
                t[:, :, dim] += gather(Vp) * sign
        t[:, :, dim] *= (norm_w / nfv)[:, None]
        for k in range(1, D):
            tdim = (dim + k) % D
            for vi in range(nfv):
                Vp = P.copy()
                for i in range(1, D):
                    Vp[:, (dim + i) % D] += 1 if (vi & i) != 0 else 0
                tsign = 1.0 if (vi & k) else -1.0
                t[:, :, tdim] += gather(Vp) * tsign
            t[:, :, tdim] *= 1.0 / nev
        tv = t[valid]
        det = np.linalg.det(tv)
        inv = np.linalg.inv(tv)
        out[dim, valid] = np.concatenate([tv.reshape(-1, D * D), inv.reshape(-1, D * D), det[:, None]], 1)
    return out.reshape((1, D) + tuple(vshape) + (2 * D * D + 1,))


def boundary_transform_from_face_transforms(face_T: np.ndarray, face: int) -> np.ndarray:
    """Slice of the face transforms on a block face, extensions/domain_structs.cpp:1809-1835.

    face_T: [1, D, (z+1), y+1, x+1, T] -> [1, (z'), y', x', T] with the face axis of size 1.
    """
    D = face_T.shape[1]
    axis = face >> 1
    upper = face & 1
    idx = [slice(None), axis]
    for dim in range(D - 1, -1, -1):
        if dim == axis:
            idx.append(slice(-1, None) if upper else slice(0, 1))
        else:
            idx.append(slice(0, -1))
    idx.append(slice(None))
    return np.ascontiguousarray(face_T[tuple(idx)])


# --------------------------------------------------------------------------
# domain model
# --------------------------------------------------------------------------

@dataclass
class OBoundary:
    kind: str  # 'fixed' | 'periodic' | 'connected'
    velocity: Optional[np.ndarray] = None  # fixed: [1,D] static or [1,D,face zyx]
    transform: Optional[np.ndarray] = None  # fixed: [1, face zyx, T]
    block: int = -1  # connected: other block index
    axes: Optional[List[int]] = None  # connected: axes as in ConnectedBoundary (extensions/domain_structs.h:329-338)
    scalar: Optional[np.ndarray] = None  # fixed: passive scalar [1,C] static or [1,C,face zyx]
    scalar_types: Optional[List[str]] = None  # fixed: 'dirichlet' / 'neumann', one for all channels or one per channel


@dataclass
class OBlock:
    size: List[int]  # x,y,z (len D)
    velocity: np.ndarray  # [1, D, zyx]
    pressure: np.ndarray  # [1, 1, zyx]
    transform: Optional[np.ndarray] = None  # [1, zyx, T]
    face_transform: Optional[np.ndarray] = None
    viscosity: Optional[np.ndarray] = None  # None, [1] static, or [1,1,zyx]
    source: Optional[np.ndarray] = None  # None, [1,D] static, or [1,D,zyx]
    scalar: Optional[np.ndarray] = None  # passive scalar [1,C,zyx]
    boundaries: List[OBoundary] = field(default_factory=list)

    @property
    def ncells(self):
        return int(np.prod(self.size))


class ODomain:
    """Host model of a PICT domain (extensions/domain_structs.h:563-787), FP64."""

    def __init__(self, dims: int, viscosity: float, scalar_channels: int = 0, scalar_viscosity=None):
        self.dims = dims
        self.viscosity = float(viscosity)
        self.blocks: List[OBlock] = []
        self.scalar_channels = int(scalar_channels)
        self.scalar_viscosity = None if scalar_viscosity is None else np.asarray(scalar_viscosity, dtype=np.float64).reshape(-1)

    # ---- construction, mirroring Domain::CreateBlock / Block::* ----
    def create_block(self, size=None, velocity=None, pressure=None, coords=None):
        D = self.dims
        if velocity is not None:
            velocity = np.asarray(velocity, dtype=np.float64)
            zyx = velocity.shape[2:]
        elif coords is not None:
            zyx = tuple(s - 1 for s in np.asarray(coords).shape[2:])
        else:
            zyx = tuple(reversed(size))
        size_xyz = list(reversed(zyx))
        if velocity is None:
            velocity = np.zeros((1, D) + tuple(zyx))
        if pressure is None:
            pressure = np.zeros((1, 1) + tuple(zyx))
        b = OBlock(size=size_xyz, velocity=np.array(velocity, dtype=np.float64),
                   pressure=np.array(pressure, dtype=np.float64))
        b.boundaries = [OBoundary("periodic") for _ in range(2 * D)]
        if coords is not None:
            b.transform = coords_to_transforms(coords)
            b.face_transform = coords_to_face_transforms(coords)
        self.blocks.append(b)
        return len(self.blocks) - 1

    def _fixed(self, bi, face, velocity=None, scalar=None, scalar_types=None):
        b = self.blocks[bi]
        D = self.dims
        vel = np.zeros((1, D)) if velocity is None else np.asarray(velocity, dtype=np.float64)
        tr = None
        if b.face_transform is not None:
            tr = boundary_transform_from_face_transforms(b.face_transform, face)
        sc = None
        if self.scalar_channels:
            sc = np.zeros((1, self.scalar_channels)) if scalar is None else np.asarray(scalar, dtype=np.float64)
        b.boundaries[face] = OBoundary("fixed", velocity=vel, transform=tr, scalar=sc,
                                       scalar_types=list(scalar_types) if scalar_types else ["dirichlet"])

    def _close_connected(self, bi, face):
        """Block::CloseConnectedBoudary with useFixed=True, extensions/domain_structs.cpp:1773-1807."""
        bnd = self.blocks[bi].boundaries[face]
        if bnd.kind == "connected":
            self._fixed(bnd.block, bnd.axes[0])
        elif bnd.kind == "periodic":
            self._fixed(bi, face ^ 1)

    def close_boundary(self, bi, face, velocity=None, scalar=None, scalar_types=None):
        """Block::CloseBoundary(face, velocity, passiveScalar), extensions/domain_structs.cpp:1979-1986, and
        FixedBoundary::setPassiveScalarType (extensions/domain_structs.cpp:622-643)."""
        face = face_index(face)
        self._close_connected(bi, face)
        self._fixed(bi, face, velocity, scalar, scalar_types)

    def close_all(self, bi):
        for f in range(2 * self.dims):
            self.close_boundary(bi, f)

    def make_periodic(self, bi, axis):
        """Block::MakePeriodic, extensions/domain_structs.cpp:1936-1955."""
        axis = axis_index(axis)
        lo, hi = axis << 1, (axis << 1) | 1
        b = self.blocks[bi]
        if not (b.boundaries[lo].kind == "periodic" and b.boundaries[hi].kind == "periodic"):
            if b.boundaries[lo].kind == "connected":
                self._close_connected(bi, lo)
            if b.boundaries[hi].kind == "connected":
                self._close_connected(bi, hi)
            b.boundaries[lo] = OBoundary("periodic")
            b.boundaries[hi] = OBoundary("periodic")

    def connect(self, b1, face1, b2, face2, axis1=-1, axis2=-1):
        """Block::ConnectBlock -> ConnectBlocks, extensions/domain_structs.cpp:1064-1097, 1924-1930."""
        face1, face2 = face_index(face1), face_index(face2)
        axis1 = face_index(axis1) if axis1 != -1 else -1
        axis2 = face_index(axis2) if axis2 != -1 else -1
        self._close_connected(b1, face1)
        self._close_connected(b2, face2)
        D = self.dims
        axes1 = [face2]
        axes2 = [face1]
        if D > 1:
            axes1.append(axis1)
            f1d, f2d = face1 >> 1, face2 >> 1
            swapped = False
            if D == 2 or (axis1 >> 1) == (f2d + 1) % D:
                axes2.append((((f1d + 1) % D) << 1) | (axis1 & 1))
            else:
                assert (axis2 >> 1) == (f2d + 1) % D, "Invalid connection."
                axes2.append((((f1d + 2) % D) << 1) | (axis2 & 1))
                swapped = True
            if D > 2:
                axes1.append(axis2)
                if not swapped:
                    axes2.append((((f1d + 2) % D) << 1) | (axis2 & 1))
                else:
                    axes2.append((((f1d + 1) % D) << 1) | (axis1 & 1))
        self.blocks[b1].boundaries[face1] = OBoundary("connected", block=b2, axes=axes1)
        self.blocks[b2].boundaries[face2] = OBoundary("connected", block=b1, axes=axes2)

    # ---- topology ----
    def prepare(self):
        """Global offsets and per-cell neighbour tables (Domain::PrepareSolve, extensions/domain_structs.cpp:2554-2676;
        neighbour resolution extensions/PISO_multiblock_cuda_kernel.cu:326-345, 432-477)."""
        D = self.dims
        self.offsets = []
        n = 0
        for b in self.blocks:
            self.offsets.append(n)
            n += b.ncells
        self.N = n
        N = n
        self.blk = np.zeros(N, dtype=np.int64)
        self.loc = np.zeros(N, dtype=np.int64)
        self.pos = np.zeros((N, 3), dtype=np.int64)
        for bi, b in enumerate(self.blocks):
            o = self.offsets[bi]
            nb = b.ncells
            l = np.arange(nb)
            sx = b.size[0]
            sy = b.size[1] if D > 1 else 1
            self.blk[o:o + nb] = bi
            self.loc[o:o + nb] = l
            self.pos[o:o + nb, 0] = l % sx
            self.pos[o:o + nb, 1] = (l // sx) % sy
            self.pos[o:o + nb, 2] = l // (sx * sy)
        K = 2 * D
        self.nb = np.full((K, N), -1, dtype=np.int64)  # neighbour global index, -1 for fixed
        self.fixed = np.zeros((K, N), dtype=bool)
        self.ncomp = np.zeros((K, N), dtype=np.int64)  # component used at the neighbour
        self.flip = np.ones((K, N))  # flux sign flip across connections
        for f in range(K):
            a = f >> 1
            up = f & 1
            for bi, b in enumerate(self.blocks):
                o = self.offsets[bi]
                sl = slice(o, o + b.ncells)
                p = self.pos[sl]
                stride = [1, b.size[0], b.size[0] * (b.size[1] if D > 1 else 1)]
                at = (p[:, a] == (b.size[a] - 1)) if up else (p[:, a] == 0)
                gi = np.arange(o, o + b.ncells)
                nbv = gi + (stride[a] if up else -stride[a])
                ncomp = np.full(b.ncells, a)
                flip = np.ones(b.ncells)
                fixed = np.zeros(b.ncells, dtype=bool)
                bnd = b.boundaries[f]
                if bnd.kind == "fixed":
                    nbv = np.where(at, -1, nbv)
                    fixed = at.copy()
                elif bnd.kind == "periodic":
                    q = p.copy()
                    q[:, a] = 0 if up else b.size[a] - 1
                    wrap = o + q[:, 0] + stride[1] * q[:, 1] + stride[2] * q[:, 2]
                    nbv = np.where(at, wrap, nbv)
                elif bnd.kind == "connected":
                    ob = self.blocks[bnd.block]
                    oo = self.offsets[bnd.block]
                    ostride = [1, ob.size[0], ob.size[0] * (ob.size[1] if D > 1 else 1)]
                    q = p.copy()  # computeConnectedPos, extensions/PISO_multiblock_cuda_kernel.cu:326-345
                    ca = bnd.axes[0] >> 1
                    q[:, ca] = ob.size[ca] - 1 if (bnd.axes[0] & 1) else 0
                    if D > 1:
                        ax = (a + 1) % D
                        ca1 = bnd.axes[1] >> 1
                        q[:, ca1] = (ob.size[ca1] - 1 - p[:, ax]) if (bnd.axes[1] & 1) else p[:, ax]
                        if D > 2:
                            ax2 = (a + 2) % D
                            ca2 = bnd.axes[2] >> 1
                            q[:, ca2] = (ob.size[ca2] - 1 - p[:, ax2]) if (bnd.axes[2] & 1) else p[:, ax2]
                    conn = oo + q[:, 0] + ostride[1] * q[:, 1] + ostride[2] * q[:, 2]
                    nbv = np.where(at, conn, nbv)
                    ncomp = np.where(at, ca, ncomp)
                    other_up = bnd.axes[0] & 1
                    flip = np.where(at & (other_up == up), -1.0, 1.0)
                self.nb[f, sl] = nbv
                self.fixed[f, sl] = fixed
                self.ncomp[f, sl] = ncomp
                self.flip[f, sl] = flip
        self._gather_static()
        self.p_result = np.zeros(N)  # Domain::CreatePressureResult, extensions/domain_structs.cpp:2823-2826

    def _gather_static(self):
        D = self.dims
        N = self.N
        self.det = np.ones(N)
        self.Minv = np.zeros((N, D, D))
        for i in range(D):
            self.Minv[:, i, i] = 1.0
        for bi, b in enumerate(self.blocks):
            o = self.offsets[bi]
            sl = slice(o, o + b.ncells)
            if b.transform is not None:
                T = b.transform.reshape(b.ncells, -1)
                self.Minv[sl] = T[:, D * D:2 * D * D].reshape(-1, D, D)
                self.det[sl] = T[:, -1]

    # ---- per-step gathers ----
    def velocity_global(self):
        D = self.dims
        u = np.zeros((D, self.N))
        for bi, b in enumerate(self.blocks):
            o = self.offsets[bi]
            u[:, o:o + b.ncells] = b.velocity.reshape(D, -1)
        return u

    def pressure_global(self):
        p = np.zeros(self.N)
        for bi, b in enumerate(self.blocks):
            o = self.offsets[bi]
            p[o:o + b.ncells] = b.pressure.reshape(-1)
        return p

    def set_velocity_global(self, u):
        D = self.dims
        for bi, b in enumerate(self.blocks):
            o = self.offsets[bi]
            b.velocity = u[:, o:o + b.ncells].reshape(b.velocity.shape).copy()

    def set_pressure_global(self, p):
        for bi, b in enumerate(self.blocks):
            o = self.offsets[bi]
            b.pressure = p[o:o + b.ncells].reshape(b.pressure.shape).copy()

    def viscosity_cells(self):
        """getViscosityBlock, extensions/PISO_multiblock_cuda_kernel.cu:1801-1822."""
        nu = np.full(self.N, self.viscosity)
        for bi, b in enumerate(self.blocks):
            if b.viscosity is None:
                continue
            o = self.offsets[bi]
            v = np.asarray(b.viscosity, dtype=np.float64)
            if v.ndim == 1:  # static
                nu[o:o + b.ncells] = v[0]
            else:
                nu[o:o + b.ncells] = v.reshape(-1)
        return nu

    def source_cells(self):
        """getBlockVelocitySource, extensions/PISO_multiblock_cuda_kernel.cu:2241-2251."""
        D = self.dims
        s = np.zeros((D, self.N))
        for bi, b in enumerate(self.blocks):
            if b.source is None:
                continue
            o = self.offsets[bi]
            v = np.asarray(b.source, dtype=np.float64)
            if v.ndim == 2:  # static [1,D]
                s[:, o:o + b.ncells] = v.reshape(D, 1)
            else:
                s[:, o:o + b.ncells] = v.reshape(D, -1)
        return s

    def boundary_cell_data(self):
        """Per face: boundary velocity [D,N], contravariant normal boundary flux [N] and
        boundary Laplace coefficient [N] at fixed faces (getFixedBoundaryData extensions/PISO_multiblock_cuda_kernel.cu:2374-2433,
        getContravariantComponentBoundaryFixed extensions/PISO_multiblock_cuda_kernel.cu:728-748, getLaplaceCoefficientOrthogonalBoundary
        extensions/PISO_multiblock_cuda_kernel.cu:1434-1447)."""
        D = self.dims
        N = self.N
        K = 2 * D
        bvel = np.zeros((K, D, N))
        bflux = np.zeros((K, N))
        balpha = np.ones((K, N))
        for f in range(K):
            a = f >> 1
            for bi, b in enumerate(self.blocks):
                bnd = b.boundaries[f]
                if bnd.kind != "fixed":
                    continue
                o = self.offsets[bi]
                sl = slice(o, o + b.ncells)
                p = self.pos[sl]
                at = self.fixed[f, sl]
                bsize = list(b.size) + [1] * (3 - D)
                bsize[a] = 1
                bflat = p[:, 0] * (1 if a != 0 else 0) + bsize[0] * (p[:, 1] if a != 1 else 0) \
                    + bsize[0] * bsize[1] * (p[:, 2] if a != 2 else 0)
                vel = np.asarray(bnd.velocity, dtype=np.float64)
                if vel.ndim == 2:
                    v = np.repeat(vel.reshape(D, 1), b.ncells, axis=1)
                else:
                    v = vel.reshape(D, -1)[:, bflat]
                if bnd.transform is not None:
                    T = bnd.transform.reshape(-1, 2 * D * D + 1)[bflat]
                    Minv = T[:, D * D:2 * D * D].reshape(-1, D, D)
                    det = T[:, -1]
                    contra = det * np.einsum("nj,jn->n", Minv[:, a, :], v)
                    alpha = det * np.einsum("nj,nj->n", Minv[:, a, :], Minv[:, a, :])
                else:
                    contra = v[a]
                    alpha = np.ones(b.ncells)
                bvel[f, :, sl] = np.where(at[None], v, 0.0)
                bflux[f, sl] = np.where(at, contra, 0.0)
                balpha[f, sl] = np.where(at, alpha, 1.0)
        return bvel, bflux, balpha

    def clone(self):
        import copy
        return copy.deepcopy(self)


# --------------------------------------------------------------------------
# assembly (kernel.cu)
# --------------------------------------------------------------------------

def contravariant(dom: ODomain, u: np.ndarray, comp: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """det * Minv[comp] . u at cells idx (VelocityToContravariantComponent, extensions/PISO_multiblock_cuda_kernel.cu:479-494)."""
    Mrow = dom.Minv[idx, comp, :]  # [n, D]
    return dom.det[idx] * np.einsum("nj,jn->n", Mrow, u[:, idx])


def laplace_coef(dom: ODomain, comp: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """det * |Minv[comp]|^2 (getLaplaceCoefficientOrthogonal, extensions/PISO_multiblock_cuda_kernel.cu:1209-1224)."""
    Mrow = dom.Minv[idx, comp, :]
    return dom.det[idx] * np.einsum("nj,nj->n", Mrow, Mrow)


def face_fluxes(dom: ODomain, u: np.ndarray, bflux: np.ndarray) -> np.ndarray:
    """computeFluxesNDLoop, extensions/PISO_multiblock_cuda_kernel.cu:1552-1630: per face the (unsigned) contravariant face flux,
    central average of the two cells, or the prescribed boundary flux at fixed faces."""
    D = dom.dims
    N = dom.N
    allc = np.arange(N)
    fl = np.zeros((2 * D, N))
    for f in range(2 * D):
        a = f >> 1
        velC = contravariant(dom, u, np.full(N, a), allc)
        nb = dom.nb[f]
        ok = nb >= 0
        velN = np.zeros(N)
        velN[ok] = contravariant(dom, u, dom.ncomp[f][ok], nb[ok]) * dom.flip[f][ok]
        fl[f] = np.where(dom.fixed[f], bflux[f], 0.5 * (velN + velC))
    return fl


def advection_matrix(dom: ODomain, dt: float, non_ortho_flags: int = 0):
    """PISO_build_matrix, extensions/PISO_multiblock_cuda_kernel.cu:3601-3865 (orthogonal terms, plus the
    non-orthogonal terms of ``nonortho_matrix_terms`` when non_ortho_flags selects them).

    Returns (coef[K,N], A[N]) with coefficients divided by det as the reference does.
    """
    D = dom.dims
    N = dom.N
    K = 2 * D + 1
    u = dom.velocity_global()
    _, bflux, _ = dom.boundary_cell_data()
    fl = face_fluxes(dom, u, bflux)
    nu = dom.viscosity_cells()
    allc = np.arange(N)
    det = dom.det
    diag = det / dt
    coef = np.zeros((K, N))
    alpha_p = [laplace_coef(dom, np.full(N, d), allc) for d in range(D)]
    for f in range(2 * D):
        d = f >> 1
        sign = 2 * (f & 1) - 1
        fixed = dom.fixed[f]
        nb = dom.nb[f]
        ok = ~fixed
        ff = sign * 0.5 * fl[f]
        alpha_n = np.zeros(N)
        nu_n = np.zeros(N)
        alpha_n[ok] = laplace_coef(dom, dom.ncomp[f][ok], nb[ok])
        nu_n[ok] = nu[nb[ok]]
        vc = 0.5 * (alpha_p[d] * nu + alpha_n * nu_n)
        diag = diag + np.where(ok, ff + vc, 2.0 * nu * alpha_p[d])  # slip=0 for Dirichlet walls
        coef[f + 1] = np.where(ok, ff - vc, 0.0)
    coef[0] = diag
    if non_ortho_flags:
        coef = coef + nonortho_matrix_terms(dom, non_ortho_flags, "adv", nu=nu)
    coef = coef / det[None]
    return coef, coef[0].copy()


def advection_rhs(dom: ODomain, dt: float, non_ortho_flags: int = 0, u_result: Optional[np.ndarray] = None):
    """kPISO_build_advection_RHS, extensions/PISO_multiblock_cuda_kernel.cu:4281-4385 (FIXED boundaries, no pressure
    gradient); with non_ortho_flags the explicit non-orthogonal viscous terms of the velocity result
    `u_result` [D,N] are subtracted before the division by det (kernel.cu:4368)."""
    D = dom.dims
    u = dom.velocity_global()
    bvel, bflux, balpha = dom.boundary_cell_data()
    nu = dom.viscosity_cells()
    src = dom.source_cells()
    det = dom.det
    rhs = det[None] * u / dt
    for f in range(2 * D):
        fixed = dom.fixed[f]
        sign = 2 * (f & 1) - 1
        flux = bflux[f] * sign
        for c in range(D):
            vel = bvel[f, c]
            add = -vel * flux + vel * nu * 2.0 * balpha[f]
            rhs[c] = rhs[c] + np.where(fixed, add, 0.0)
    if non_ortho_flags:
        fields = {"vel": u if u_result is None else u_result}
        for c in range(D):
            rhs[c] = rhs[c] - nonortho_rhs(dom, non_ortho_flags, "vel", fields, c, True, False, nu=nu)
    rhs = rhs / det[None] + src
    return rhs


# --------------------------------------------------------------------------
# Smagorinsky sub-grid-scale viscosity
# --------------------------------------------------------------------------

def sgs_smagorinsky(dom: ODomain, coefficient: float) -> np.ndarray:
    """SGSviscosityIncompressibleSmagorinsky, kernel.cu:6896-7019, per cell [N]: coefficient * delta * |S| with
    the velocity gradient of getBlockDataGradient (kernel.cu:2987-3031: neighbour differences along each
    computational axis over 2 cells, 1.5 where one side is a fixed face holding the boundary velocity;
    the same component across a connection) times Minv, |S| = sqrt(2 S:S), and delta the largest
    squared column length of the cell's transform M (1 without a transform)."""
    D = dom.dims
    N = dom.N
    u = dom.velocity_global()
    bvel, _, _ = dom.boundary_cell_data()
    g = np.zeros((N, D, D))
    for k in range(D):
        dist = np.full(N, 2.0)
        vals = []
        for up in (0, 1):
            f = 2 * k + up
            fixed = dom.fixed[f]
            vals.append(np.where(fixed[None], bvel[f], u[:, np.maximum(dom.nb[f], 0)]))
            dist = dist - np.where(fixed, 0.5, 0.0)
        g[:, :, k] = ((vals[1] - vals[0]) / dist[None]).T
    G = np.einsum("nck,nkj->ncj", g, dom.Minv)
    S = 0.5 * (G + np.transpose(G, (0, 2, 1)))
    norm = np.sqrt(2.0 * np.sum(S * S, axis=(1, 2)))
    delta = np.ones(N)
    for bi, b in enumerate(dom.blocks):
        if b.transform is None:
            continue
        o = dom.offsets[bi]
        M = b.transform.reshape(b.ncells, -1)[:, :D * D].reshape(-1, D, D)
        delta[o:o + b.ncells] = np.max(np.sum(M * M, axis=1), axis=1)
    return coefficient * delta * norm


# --------------------------------------------------------------------------
# passive scalars
# --------------------------------------------------------------------------

def scalar_viscosity(dom: ODomain, c: int) -> float:
    """getViscosity with forPassiveScalar, kernel.cu:1788-1799: the scalar viscosity ([1] or per channel),
    else the domain viscosity; block viscosities do not apply to scalars (kernel.cu:1804-1807)."""
    sv = dom.scalar_viscosity
    if sv is None:
        return dom.viscosity
    return float(sv[0] if sv.size == 1 else sv[c])


def scalar_global(dom: ODomain) -> np.ndarray:
    """The blocks' passive scalars as [C, N] (CopyScalarResultFromBlocks)."""
    C = dom.scalar_channels
    return np.concatenate([np.asarray(b.scalar, dtype=np.float64).reshape(C, -1) for b in dom.blocks], axis=1)


def _scalar_face_data(dom: ODomain, c: int):
    """Per face: boundary scalar of channel c [N] and Neumann mask [N] at cells on fixed faces."""
    D = dom.dims
    N = dom.N
    sb = np.zeros((2 * D, N))
    neu = np.zeros((2 * D, N), dtype=bool)
    for g in range(N):
        bi = int(dom.blk[g])
        p = [int(v) for v in dom.pos[g]]
        for f in range(2 * D):
            if dom.fixed[f, g]:
                sb[f, g] = _fixed_data(dom, bi, f, p, c, "sc")
                neu[f, g] = _scalar_type(dom, bi, f, c) == "neumann"
    return sb, neu


def scalar_matrix(dom: ODomain, dt: float, channel: int, non_ortho_flags: int = 0):
    """PISO_build_matrix with forPassiveScalar, kernel.cu:3601-3865: the advection-diffusion matrix with the
    scalar viscosity of `channel`; a fixed face adds 2 nu alpha to the diagonal only where the channel's
    boundary type is Dirichlet (slip = 1 for Neumann, kernel.cu:3817-3832).  Returns (coef[K,N], A[N])."""
    D = dom.dims
    N = dom.N
    K = 2 * D + 1
    u = dom.velocity_global()
    _, bflux, _ = dom.boundary_cell_data()
    fl = face_fluxes(dom, u, bflux)
    nu = scalar_viscosity(dom, channel)
    _, neu = _scalar_face_data(dom, channel)
    allc = np.arange(N)
    det = dom.det
    diag = det / dt
    coef = np.zeros((K, N))
    alpha_p = [laplace_coef(dom, np.full(N, d), allc) for d in range(D)]
    for f in range(2 * D):
        d = f >> 1
        sign = 2 * (f & 1) - 1
        ok = ~dom.fixed[f]
        nb = dom.nb[f]
        ff = sign * 0.5 * fl[f]
        alpha_n = np.zeros(N)
        alpha_n[ok] = laplace_coef(dom, dom.ncomp[f][ok], nb[ok])
        vc = 0.5 * (alpha_p[d] + alpha_n) * nu
        diag = diag + np.where(ok, ff + vc, np.where(neu[f], 0.0, 2.0 * nu * alpha_p[d]))
        coef[f + 1] = np.where(ok, ff - vc, 0.0)
    coef[0] = diag
    if non_ortho_flags:
        coef = coef + nonortho_matrix_terms(dom, non_ortho_flags, "sc", nu=np.full(N, nu), channel=channel)
    coef = coef / det[None]
    return coef, coef[0].copy()


def scalar_rhs(dom: ODomain, dt: float, non_ortho_flags: int = 0, s_result: Optional[np.ndarray] = None):
    """kPISO_build_scalar_advection_RHS, kernel.cu:4079-4183: per channel det s / dt, at fixed faces minus the
    boundary scalar times the boundary flux plus nu 2 alpha s_b (Dirichlet) or nu s_b (Neumann), minus nu
    times the explicit non-orthogonal terms of `s_result` [C,N] (kernel.cu:4165-4167), over det."""
    D = dom.dims
    N = dom.N
    C = dom.scalar_channels
    s = scalar_global(dom)
    _, bflux, balpha = dom.boundary_cell_data()
    det = dom.det
    rhs = det[None] * s / dt
    for c in range(C):
        nu = scalar_viscosity(dom, c)
        sb, neu = _scalar_face_data(dom, c)
        for f in range(2 * D):
            sign = 2 * (f & 1) - 1
            add = -sb[f] * bflux[f] * sign + np.where(neu[f], sb[f] * nu, sb[f] * nu * 2.0 * balpha[f])
            rhs[c] = rhs[c] + np.where(dom.fixed[f], add, 0.0)
        if non_ortho_flags:
            fields = {"sc": s if s_result is None else s_result}
            rhs[c] = rhs[c] - nonortho_rhs(dom, non_ortho_flags, "sc", fields, c, True, False, nu=np.full(N, nu))
    return rhs / det[None]


def pressure_matrix(dom: ODomain, A: np.ndarray, non_ortho_flags: int = 0):
    """PISO_build_pressure_matrix, extensions/PISO_multiblock_cuda_kernel.cu:4797-4963 (no face transforms; the
    non-orthogonal terms of ``nonortho_matrix_terms`` when non_ortho_flags selects them)."""
    D = dom.dims
    N = dom.N
    K = 2 * D + 1
    allc = np.arange(N)
    raP = 1.0 / A
    coef = np.zeros((K, N))
    for f in range(2 * D):
        d = f >> 1
        ok = ~dom.fixed[f]
        nb = dom.nb[f]
        alphaP = laplace_coef(dom, np.full(N, d), allc)
        alphaN = np.zeros(N)
        raN = np.zeros(N)
        alphaN[ok] = laplace_coef(dom, dom.ncomp[f][ok], nb[ok])
        raN[ok] = 1.0 / A[nb[ok]]
        c = np.where(ok, 0.5 * (alphaP * raP + alphaN * raN), 0.0)
        coef[0] -= c
        coef[f + 1] = c
    if non_ortho_flags:
        coef = coef + nonortho_matrix_terms(dom, non_ortho_flags, "p", A=A)
    return coef


def pressure_rhs(dom: ODomain, dt: float, Ccoef: np.ndarray, A: np.ndarray, u_star: np.ndarray):
    """PISO_build_pressure_rhs, extensions/PISO_multiblock_cuda_kernel.cu:5121-5240 (with boundary sources, the compiled default)."""
    D = dom.dims
    N = dom.N
    u = dom.velocity_global()
    bvel, bflux, balpha = dom.boundary_cell_data()
    nu = dom.viscosity_cells()
    src = dom.source_cells()
    det = dom.det
    allc = np.arange(N)
    h = np.zeros((D, N))
    for c in range(D):
        H = np.zeros(N)
        S = np.zeros(N)
        for f in range(2 * D):
            nb = dom.nb[f]
            ok = (nb >= 0) & (nb != allc)
            H[ok] += Ccoef[f + 1][ok] * u_star[c][nb[ok]]
            fixed = dom.fixed[f]
            sign = 2 * (f & 1) - 1
            vel = bvel[f, c]
            S += np.where(fixed, -vel * bflux[f] * sign + vel * nu * 2.0 * balpha[f], 0.0)
        S = S / det + src[c]
        h[c] = (u[c] / dt - H + S) / A
    return h


def divergence(dom: ODomain, h: np.ndarray):
    """k_computePressureRHSdivergenceFromFlux, extensions/PISO_multiblock_cuda_kernel.cu:5374-5419 (no time-step norm)."""
    D = dom.dims
    _, bflux, _ = dom.boundary_cell_data()
    fl = face_fluxes(dom, h, bflux)
    div = np.zeros(dom.N)
    for d in range(D):
        div += fl[2 * d + 1] - fl[2 * d]
    return div


def pressure_rhs_nonortho(dom: ODomain, non_ortho_flags: int, div: np.ndarray, A: np.ndarray,
                          p_result: np.ndarray) -> np.ndarray:
    """k_pressureRHSaddNonOrthoComponents, extensions/PISO_multiblock_cuda_kernel.cu:5423-5453: div plus the explicit
    non-orthogonal terms of the pressure result (with 1/A, no viscosity)."""
    return div + nonortho_rhs(dom, non_ortho_flags, "p", {"p": p_result}, 0, False, True, A=A)


def pressure_gradient_fd(dom: ODomain, p: np.ndarray):
    """getPressureGradient, extensions/PISO_multiblock_cuda_kernel.cu:801-834 with getPressureAtWithBounds extensions/PISO_multiblock_cuda_kernel.cu:2160-2239."""
    D = dom.dims
    N = dom.N
    g = np.zeros((D, N))
    for d in range(D):
        lo, hi = 2 * d, 2 * d + 1
        fac = np.full(N, 0.5)
        lo_fixed = dom.fixed[lo]
        hi_fixed = dom.fixed[hi]
        nbl = np.where(lo_fixed, np.arange(N), dom.nb[lo])
        nbh = np.where(hi_fixed, np.arange(N), dom.nb[hi])
        fac = np.where(lo_fixed | hi_fixed, 1.0, fac)
        g[d] = (p[nbh] - p[nbl]) * fac
    # matmul(pressureGrad, Minv): g_j = sum_i g_i Minv[i][j]
    return np.einsum("in,nij->jn", g, dom.Minv)


def correct_velocity(dom: ODomain, p_blocks: np.ndarray, A: np.ndarray, h: np.ndarray):
    """PISO_update_velocity (version 1, FD), extensions/PISO_multiblock_cuda_kernel.cu:5947-5980."""
    g = pressure_gradient_fd(dom, p_blocks)
    return h - g / A[None]


def _cells(dom: ODomain, bi: int):
    b = dom.blocks[bi]
    s = list(b.size) + [1] * (3 - dom.dims)
    for z in range(s[2]):
        for y in range(s[1]):
            for x in range(s[0]):
                yield [x, y, z]


def _across(dom: ODomain, bi: int, p, face: int):
    """The cell across a non-prescribed face (resolveNeighborCell without the second layer): (block, pos,
    connected boundary or None)."""
    b = dom.blocks[bi]
    a = face >> 1
    if _at_bound(dom, bi, p, face):
        bnd = b.boundaries[face]
        if bnd.kind == "connected":
            ob, q = _conn_pos(dom, bi, face, p, 0)
            return ob, q, bnd
        q = list(p)
        q[a] = 0 if face & 1 else b.size[a] - 1
        return bi, q, None
    q = list(p)
    q[a] += 1 if face & 1 else -1
    return bi, q, None


def pressure_gradient_fvm(dom: ODomain, p: np.ndarray, interpolation: int):
    """getPressureGradientFVM, extensions/PISO_multiblock_cuda_kernel.cu:991-1123: face pressures times face
    area vectors (rows of det Minv), interpolation 0 = mean of the two cells' fluxes, 3 = the staggered
    face transform times the mean pressure.  A prescribed face extrapolates the pressure from the
    opposite side (half a cell for 0, a full cell for 3) and uses the boundary transform; blocks without
    a transform take the finite-difference gradient."""
    D = dom.dims
    g_fd = pressure_gradient_fd(dom, p)
    out = np.zeros((D, dom.N))
    T = 2 * D * D + 1
    for bi, b in enumerate(dom.blocks):
        for q in _cells(dom, bi):
            gi = _gidx(dom, bi, q)
            if b.transform is None:
                out[:, gi] = g_fd[:, gi]
                continue
            MP, dP, pP = dom.Minv[gi], dom.det[gi], p[gi]
            grad = np.zeros(D)
            for face in range(2 * D):
                a, up = face >> 1, face & 1
                fs = 1.0 if up else -1.0
                fluxP = MP[a] * (dP * pP)
                axisN, tsgn = a, 1.0
                if _at_bound(dom, bi, q, face) and _is_empty(dom, bi, face):
                    bnd = b.boundaries[face]
                    qi = list(q)
                    qi[a] -= 1 if up else -1
                    p_in = p[_gidx(dom, bi, qi)]
                    if interpolation != 3:
                        Tb = bnd.transform.reshape(-1, T)[_bound_flat(dom, bi, face, q)]
                        pb = pP + (pP - p_in) * 0.5
                        grad += Tb[D * D:2 * D * D].reshape(D, D)[a] * (Tb[-1] * pb) * fs
                        continue
                    pn = pP + (pP - p_in)
                    MN, dN = MP, dP
                else:
                    ob, qn, cb = _across(dom, bi, q, face)
                    if cb is not None:
                        axisN = cb.axes[0] >> 1
                        if (cb.axes[0] & 1) == up:
                            tsgn = -1.0
                    gN = _gidx(dom, ob, qn)
                    MN, dN, pn = dom.Minv[gN], dom.det[gN], p[gN]
                if interpolation == 0:
                    grad += (fluxP + MN[axisN] * (dN * pn * tsgn)) * (0.5 * fs)
                elif interpolation == 3:
                    fq = list(q)
                    fq[a] += up
                    if D == 2:
                        F = b.face_transform[0, a, fq[1], fq[0]]
                    else:
                        F = b.face_transform[0, a, fq[2], fq[1], fq[0]]
                    grad += F[D * D:2 * D * D].reshape(D, D)[a] * (F[-1] * (pn + pP) * 0.5 * fs)
            out[:, gi] = grad / dP
    return out


def correct_velocity_fvm(dom: ODomain, p_blocks: np.ndarray, A: np.ndarray, h: np.ndarray, dt: float,
                         version: int, time_step_norm: bool = False):
    """PISO_update_velocity_PressureFVM (versions 5 and 6), extensions/PISO_multiblock_cuda_kernel.cu:6013-6050,
    6180-6191."""
    g = pressure_gradient_fvm(dom, p_blocks, 0 if version == 5 else 3)
    if time_step_norm:
        g = g * dt
    return h - g / A[None]


def correct_velocity_v4(dom: ODomain, p_blocks: np.ndarray, A: np.ndarray, h: np.ndarray, dt: float):
    """PISO_update_velocity_v4_orthogonal (version 4), extensions/PISO_multiblock_cuda_kernel.cu:6053-6160: the mean
    of the two face fluxes (H/A minus the pressure flux through the face, with the orthogonal metrics of
    the two cells), transformed back; a prescribed face contributes nothing.  As in the reference, the
    cell's own metric is Minv[0][0] for every component (it is read at the cell position, whose channel
    is 0), the neighbour's is Minv[d][d] (its aligned axis across a connection)."""
    D = dom.dims
    u = np.zeros((D, dom.N))
    for bi, b in enumerate(dom.blocks):
        for q in _cells(dom, bi):
            gi = _gidx(dom, bi, q)
            ra, pc, det = 1.0 / A[gi], p_blocks[gi], dom.det[gi]
            t = dom.Minv[gi][0, 0]
            for d in range(D):
                cc = det * t
                v = 0.0
                for up in (0, 1):
                    face = 2 * d + up
                    if _at_bound(dom, bi, q, face) and _is_empty(dom, bi, face):
                        continue
                    ob, qn, cb = _across(dom, bi, q, face)
                    comp = (cb.axes[0] >> 1) if cb is not None else d
                    gN = _gidx(dom, ob, qn)
                    tN = dom.Minv[gN][comp, comp]
                    ccN = dom.det[gN] * tN
                    dp = (pc - p_blocks[gN]) if up == 0 else (p_blocks[gN] - pc)
                    v += (cc * h[d, gi] + ccN * h[comp, gN] - (cc * t * ra + ccN * tN / A[gN]) * dp * dt) * 0.25
                u[d, gi] = v / (det * t)
    return u


# --------------------------------------------------------------------------
# non-orthogonal terms (nonOrthoFlags != 0): tangential Laplacian fluxes on skewed grids
# --------------------------------------------------------------------------

# bit flags, extensions/PISO_multiblock_cuda.h:9-13; the driver's default set, sim.py:390-396
NON_ORTHO_DIRECT_MATRIX = 1
NON_ORTHO_DIRECT_RHS = 2
NON_ORTHO_DIAGONAL_MATRIX = 4
NON_ORTHO_DIAGONAL_RHS = 8
NON_ORTHO_CENTER_MATRIX = 16
NON_ORTHO_DEFAULT = NON_ORTHO_CENTER_MATRIX | NON_ORTHO_DIRECT_MATRIX | NON_ORTHO_DIAGONAL_RHS


def _gidx(dom: ODomain, bi: int, p) -> int:
    b = dom.blocks[bi]
    sx = b.size[0]
    sy = b.size[1] if dom.dims > 1 else 1
    return dom.offsets[bi] + p[0] + sx * (p[1] + sy * p[2])


def _at_bound(dom: ODomain, bi: int, p, face: int) -> bool:
    """isAtBound, kernel.cu:228-240."""
    a = face >> 1
    return p[a] == (dom.blocks[bi].size[a] - 1 if face & 1 else 0)


def _is_empty(dom: ODomain, bi: int, face: int) -> bool:
    """isEmptyBound, kernel.cu:188-194: a prescribed (fixed) face, by type only."""
    return dom.blocks[bi].boundaries[face].kind == "fixed"


def _conn_pos(dom: ODomain, bi: int, face: int, p, offset: int):
    """computeConnectedPos, kernel.cu:326-345: the cell `offset` layers into the block across the
    connection of face `face` (offset 0 is the first layer)."""
    D = dom.dims
    bnd = dom.blocks[bi].boundaries[face]
    ob = dom.blocks[bnd.block]
    a = face >> 1
    q = list(p)
    ca = bnd.axes[0] >> 1
    q[ca] = ob.size[ca] - 1 - offset if bnd.axes[0] & 1 else offset
    for k in range(1, D):
        ax = (a + k) % D
        ca = bnd.axes[k] >> 1
        q[ca] = ob.size[ca] - 1 - p[ax] if bnd.axes[k] & 1 else p[ax]
    return bnd.block, q


def _conn_dir(dom: ODomain, bi: int, face: int, d: int) -> int:
    """computeConnectedDir, kernel.cu:314-323 (getAxisRelativeToOther kernel.cu:243-245)."""
    bnd = dom.blocks[bi].boundaries[face]
    rel = ((d >> 1) - (face >> 1)) % dom.dims
    return bnd.axes[rel] ^ (d & 1)


def _lap_full(dom: ODomain, g: int) -> np.ndarray:
    """getLaplaceCoefficientsFull, kernel.cu:1270-1295: alpha[c1][c2] = det Minv[c1].Minv[c2]."""
    M = dom.Minv[g]
    return dom.det[g] * (M @ M.T)


def _bound_flat(dom: ODomain, bi: int, face: int, p) -> int:
    a = face >> 1
    s = list(dom.blocks[bi].size) + [1] * (3 - dom.dims)
    s[a] = 1
    q = list(p)
    q[a] = 0
    return q[0] + s[0] * (q[1] + s[1] * q[2])


def _bound_lap_axis(dom: ODomain, bi: int, face: int, p, axis: int) -> np.ndarray:
    """getLaplaceCoefficientsNeighbourBoundary, kernel.cu:1469-1491 (fixed boundary transform)."""
    D = dom.dims
    bnd = dom.blocks[bi].boundaries[face]
    if bnd.transform is None:
        e = np.zeros(D)
        e[axis] = 1.0
        return e
    T = bnd.transform.reshape(-1, 2 * D * D + 1)[_bound_flat(dom, bi, face, p)]
    Minv = T[D * D:2 * D * D].reshape(D, D)
    return T[-1] * (Minv @ Minv[axis])


def _fixed_data(dom: ODomain, bi: int, face: int, p, comp: int, kind: str) -> float:
    """getFixedBoundaryData, kernel.cu:2379-2447, fixed boundaries: the velocity component or passive scalar
    channel; the fixed boundary pressure is a static zero (domain_structs.cpp:565-576); IS_FIXED_BOUNDARY
    reads 1."""
    if kind == "flag":
        return 1.0
    if kind == "p":
        return 0.0
    if kind == "sc":
        sc = dom.blocks[bi].boundaries[face].scalar
        if sc is None:
            return 0.0
        sc = np.asarray(sc, dtype=np.float64)
        if sc.ndim == 2:
            return float(sc[0, comp])
        return float(sc.reshape(dom.scalar_channels, -1)[comp, _bound_flat(dom, bi, face, p)])
    vel = np.asarray(dom.blocks[bi].boundaries[face].velocity, dtype=np.float64)
    if vel.ndim == 2:
        return float(vel[0, comp])
    return float(vel.reshape(dom.dims, -1)[comp, _bound_flat(dom, bi, face, p)])


def _scalar_type(dom: ODomain, bi: int, face: int, comp: int) -> str:
    types = dom.blocks[bi].boundaries[face].scalar_types or ["dirichlet"]
    return types[comp] if len(types) > 1 else types[0]


def _fixed_type(kind: str, dom: Optional[ODomain] = None, bi: int = 0, face: int = 0, comp: int = 0) -> str:
    """getFixedBoundaryType, kernel.cu:2353-2377: velocity Dirichlet, pressure Neumann, passive scalar per
    face and channel."""
    if kind == "sc":
        return _scalar_type(dom, bi, face, comp)
    return "neumann" if kind == "p" else "dirichlet"


def _block_data(dom: ODomain, bi: int, p, comp: int, kind: str, fields) -> float:
    """getBlockData, kernel.cu:2322-2330, on the global result vectors (kind 'vel' / 'p'); other kinds read 0."""
    if fields is None:
        return 0.0
    g = _gidx(dom, bi, p)
    if kind == "vel":
        return float(fields["vel"][comp, g])
    if kind == "p":
        return float(fields["p"][g])
    if kind == "sc":
        return float(fields["sc"][comp, g])
    return 0.0


def corner_value(dom: ODomain, bi: int, p, comp: int, dir1: int, dir2: int, incl0: bool, incl1: bool,
                 max_depth: int, kind: str, fields=None):
    """getCornerValue, kernel.cu:2742-2860: walk around the corner of cell `p` between faces dir1 and
    dir2 in both directions (depth 1: the face neighbours, depth 2: the diagonal cell) until the walks
    meet, a fixed boundary is hit or max_depth is reached.  Returns (value, cells, boundary type);
    cells == 0 means the value came from a fixed boundary.  Across a block connection the walk lands
    on the second cell layer of the connected block (computeConnectedPos with borderOffset 1,
    kernel.cu:2810), as the reference does."""
    data = 0.0
    n = 0
    btype = "dirichlet"
    if incl0:
        data += _block_data(dom, bi, p, comp, kind, fields)
    n += 1
    walk = [[dir1, dir2, bi, list(p)], [dir2, dir1, bi, list(p)]]
    for depth in range(1, max_depth + 1):
        for d in range(2):
            w = walk[d]
            d1, d2, wb, wp = w
            a = d1 >> 1
            if _at_bound(dom, wb, wp, d1):
                bnd = dom.blocks[wb].boundaries[d1]
                if bnd.kind == "fixed":
                    btype = _fixed_type(kind, dom, wb, d1, comp)
                    if _at_bound(dom, wb, wp, d2):
                        return _fixed_data(dom, wb, d1, wp, comp, kind), 0, btype
                    q = list(wp)
                    q[d2 >> 1] += 1 if d2 & 1 else -1
                    return (_fixed_data(dom, wb, d1, wp, comp, kind) + _fixed_data(dom, wb, d1, q, comp, kind)) * 0.5, 0, btype
                if bnd.kind == "connected":
                    nb_, q = _conn_pos(dom, wb, d1, wp, 1)
                    w[0] = _conn_dir(dom, wb, d1, d2)
                    w[1] = _conn_dir(dom, wb, d1, d1) ^ 1
                    w[2], w[3] = nb_, q
                else:  # periodic
                    q = list(wp)
                    q[a] = 0 if d1 & 1 else dom.blocks[wb].size[a] - 1
                    w[0], w[1], w[3] = d2, d1 ^ 1, q
            else:
                q = list(wp)
                q[a] += 1 if d1 & 1 else -1
                w[0], w[1], w[3] = d2, d1 ^ 1, q
            o = walk[d ^ 1]
            if w[2] == o[2] and w[3] == o[3]:
                return data / n, n, btype
            if depth > 1 or incl1:
                data += _block_data(dom, w[2], w[3], comp, kind, fields)
            n += 1
    return data / n, n, btype


def _neighbor_info(dom: ODomain, bi: int, p, face: int):
    """resolveNeighborCell, kernel.cu:432-477, for a face that is not prescribed: the neighbour's block,
    position and the axis mapping (faces of the neighbour's block for +x, +y, +z of this block)."""
    D = dom.dims
    a = face >> 1
    mapping = [0, 2, 4]
    if _at_bound(dom, bi, p, face):
        bnd = dom.blocks[bi].boundaries[face]
        if bnd.kind == "connected":
            nb_, q = _conn_pos(dom, bi, face, p, 0)
            mapping = [_conn_dir(dom, bi, face, mapping[k]) if k < D else mapping[k] for k in range(3)]
            return nb_, q, mapping
        q = list(p)
        q[a] = 0 if face & 1 else dom.blocks[bi].size[a] - 1
        return bi, q, mapping
    q = list(p)
    q[a] += 1 if face & 1 else -1
    return bi, q, mapping


def _neighbor_data(dom: ODomain, bi: int, p, face: int, comp: int, kind: str, fields) -> float:
    """getBlockDataNeighbor, kernel.cu:2519-2560 (zeroBound false; second layer across connections)."""
    a = face >> 1
    if _at_bound(dom, bi, p, face):
        bnd = dom.blocks[bi].boundaries[face]
        if bnd.kind == "fixed":
            return _fixed_data(dom, bi, face, p, comp, kind)
        if bnd.kind == "connected":
            nb_, q = _conn_pos(dom, bi, face, p, 1)
            return _block_data(dom, nb_, q, comp, kind, fields)
        q = list(p)
        q[a] = 0 if face & 1 else dom.blocks[bi].size[a] - 1
        return _block_data(dom, bi, q, comp, kind, fields)
    q = list(p)
    q[a] += 1 if face & 1 else -1
    return _block_data(dom, bi, q, comp, kind, fields)


def _diagonal_data(dom: ODomain, bi: int, p, dir1: int, dir2: int, comp: int, kind: str, fields) -> float:
    """getBlockDataNeighborDiagonal, kernel.cu:2615-2660: two steps (dir2 first if dir1's face is a
    prescribed type); a fixed face on the way returns its data; no direction remapping across a
    connection; second layer across connections."""
    first_empty = _is_empty(dom, bi, dir1)
    dirs = [dir2, dir1] if first_empty else [dir1, dir2]
    cb, q = bi, list(p)
    for bound in dirs:
        a = bound >> 1
        if _at_bound(dom, cb, q, bound):
            bnd = dom.blocks[cb].boundaries[bound]
            if bnd.kind == "fixed":
                return _fixed_data(dom, cb, bound, q, comp, kind)
            if bnd.kind == "connected":
                cb, q = _conn_pos(dom, cb, bound, q, 1)
            else:
                q = list(q)
                q[a] = 0 if bound & 1 else dom.blocks[cb].size[a] - 1
        else:
            q = list(q)
            q[a] += 1 if bound & 1 else -1
    return _block_data(dom, cb, q, comp, kind, fields)


def nonortho_alpha_interp(dom: ODomain, bi: int, p, with_visc: bool, with_A: bool, A=None, nu=None) -> np.ndarray:
    """interpolateNonOrthoLaplaceComponents, kernel.cu:1911-1987: per face and tangent axis
    (axis + i) % D the face-averaged off-diagonal Laplace coefficient, [2D][D-1].  A face counts as
    prescribed unless the cell is strictly inside along its axis or the face is not a prescribed type
    (so a cell on one wall also drops the opposite face, as in the reference)."""
    D = dom.dims
    g = _gidx(dom, bi, p)
    aP = _lap_full(dom, g)
    raP = (1.0 / A[g] if with_A else 1.0) * (nu[g] if with_visc else 1.0)
    out = np.zeros((2 * D, max(D - 1, 1)))
    for face in range(2 * D):
        axis = face >> 1
        s = dom.blocks[bi].size[axis]
        if not ((0 < p[axis] < s - 1) or not _is_empty(dom, bi, face)):
            continue
        if _at_bound(dom, bi, p, face) and dom.blocks[bi].boundaries[face].kind == "connected":
            nb_, q = _conn_pos(dom, bi, face, p, 0)
        else:
            nb_, q = bi, list(p)
            if _at_bound(dom, bi, p, face) and dom.blocks[bi].boundaries[face].kind == "periodic":
                q[axis] = 0 if face & 1 else s - 1
            else:
                q[axis] += 1 if face & 1 else -1
        gN = _gidx(dom, nb_, q)
        M = dom.Minv[gN]
        aN = dom.det[gN] * (M @ M[axis])  # getLaplaceCoefficientsSingleAxis, kernel.cu:1298-1320 (no axis mapping)
        raN = (1.0 / A[gN] if with_A else 1.0) * (nu[gN] if with_visc else 1.0)
        for i in range(1, D):
            t = (axis + i) % D
            out[face, i - 1] = (aP[axis, t] * raP + aN[t] * raN) * 0.5
    return out


def nonortho_matrix_terms(dom: ODomain, flags: int, which: str, A=None, nu=None, channel: int = 0) -> np.ndarray:
    """Non-orthogonal stencil terms [K, N]: which='adv' as PISO_build_matrix, kernel.cu:3736-3800 (with
    viscosity; the caller divides by det afterwards), which='p' as PISO_build_pressure_matrix,
    kernel.cu:4877-4934 (with 1/A).  A corner interpolated from n cells contributes
    faceSign * tFaceSign * alpha / n to the diagonal, the face neighbour and the tangential neighbour;
    a corner on a gradient boundary is replaced by a one-sided difference (3/4, 1/4)."""
    D = dom.dims
    N = dom.N
    add = np.zeros((2 * D + 1, N))
    incl_nb = bool(flags & NON_ORTHO_DIRECT_MATRIX)
    incl_diag = bool(flags & NON_ORTHO_CENTER_MATRIX)
    if D < 2 or not (incl_nb or incl_diag):
        return add
    sgn = 1.0 if which == "p" else -1.0
    kind = {"adv": "vel", "p": "flag", "sc": "sc"}[which]
    for g in range(N):
        bi = int(dom.blk[g])
        p = [int(v) for v in dom.pos[g]]
        ai = nonortho_alpha_interp(dom, bi, p, which != "p", which == "p", A, nu)
        for face in range(2 * D):
            if _at_bound(dom, bi, p, face) and _is_empty(dom, bi, face):
                continue
            fs = 1.0 if face & 1 else -1.0
            axis = face >> 1
            for i in range(1, D):
                t = (axis + i) % D
                alpha = ai[face, i - 1]
                if alpha == 0:
                    continue
                for tup in range(2):
                    tface = 2 * t + tup
                    ts = 1.0 if tup else -1.0
                    _, n, btype = corner_value(dom, bi, p, channel, face, tface, False, False, 2, kind, None)
                    grad = (btype == "neumann") if which != "p" else True
                    if n < 1:
                        if grad:
                            v = fs * ts * alpha * 0.25
                            if incl_diag:
                                add[0, g] += sgn * 3 * v
                            if incl_nb:
                                add[face + 1, g] += sgn * 3 * v
                                add[(tface ^ 1) + 1, g] -= sgn * v
                    else:
                        v = fs * ts * alpha / n
                        if incl_diag:
                            add[0, g] += sgn * v
                        if incl_nb:
                            add[face + 1, g] += sgn * v
                            add[tface + 1, g] += sgn * v
    return add


def nonortho_rhs(dom: ODomain, flags: int, kind: str, fields, comp: int, with_visc: bool, with_A: bool,
                 A=None, nu=None) -> np.ndarray:
    """getNonOrthoLaplaceRHS_v2, kernel.cu:3033-3187, for component `comp` of every cell: the explicit
    part of the tangential fluxes (corner values of the data in `fields`: kind 'vel' the velocity
    result, 'p' the pressure result), and for the velocity the tangential gradient of the fixed
    boundary data on prescribed faces.  The sign assumes the Laplacian on the left-hand side."""
    D = dom.dims
    N = dom.N
    S = np.zeros(N)
    if not (flags & (NON_ORTHO_DIRECT_RHS | NON_ORTHO_DIAGONAL_RHS)) or D < 2:
        return S
    incl1 = bool(flags & NON_ORTHO_DIRECT_RHS)
    for g in range(N):
        bi = int(dom.blk[g])
        p = [int(v) for v in dom.pos[g]]
        aP = _lap_full(dom, g)
        raP = (1.0 / A[g] if with_A else 1.0) * (nu[g] if with_visc else 1.0)
        s = 0.0
        for face in range(2 * D):
            axis = face >> 1
            fs = 1.0 if face & 1 else -1.0
            if _at_bound(dom, bi, p, face) and _is_empty(dom, bi, face):
                if kind == "p" or _fixed_type(kind, dom, bi, face, comp) == "neumann":
                    continue
                balpha = _bound_lap_axis(dom, bi, face, p, axis)
                for i in range(1, D):
                    t = (axis + i) % D
                    tlo = p[t] == 0
                    thi = p[t] == dom.blocks[bi].size[t] - 1
                    lo, hi = list(p), list(p)
                    if not tlo:
                        lo[t] -= 1
                    if not thi:
                        hi[t] += 1
                    df = 1.0 if (tlo or thi) else 0.5
                    tg = df * (_fixed_data(dom, bi, face, hi, comp, kind) - _fixed_data(dom, bi, face, lo, comp, kind))
                    bv = nu[g] if with_visc else 1.0
                    s -= fs * balpha[t] * tg * bv
                continue
            nb_, q, mapping = _neighbor_info(dom, bi, p, face)
            gN = _gidx(dom, nb_, q)
            M = dom.Minv[gN]
            am = mapping[axis] >> 1
            aN = np.array([dom.det[gN] * np.dot(M[mapping[c] >> 1], M[am]) for c in range(D)])
            raN = (1.0 / A[gN] if with_A else 1.0) * (nu[gN] if with_visc else 1.0)
            for i in range(1, D):
                t = (axis + i) % D
                fa = (aP[axis, t] * raP + aN[t] * raN) * 0.5
                tg = 0.0
                for tup in range(2):
                    tface = 2 * t + tup
                    ts = 1.0 if tup else -1.0
                    val, n, btype = corner_value(dom, bi, p, comp, face, tface, False, incl1, 2, kind, fields)
                    if n == 0 and (btype == "neumann" or kind == "p"):
                        tother = tface ^ 1
                        if flags & NON_ORTHO_DIRECT_RHS:
                            tg += ts * _neighbor_data(dom, bi, p, face, comp, kind, fields) * 0.75
                            tg += -ts * _neighbor_data(dom, bi, p, tother, comp, kind, fields) * 0.25
                        if flags & NON_ORTHO_DIAGONAL_RHS:
                            tg += -ts * _diagonal_data(dom, bi, p, face, tother, comp, kind, fields) * 0.25
                    else:
                        tg += ts * val
                s -= fs * fa * tg
        S[g] = s
    return S


# --------------------------------------------------------------------------
# CSR export in the reference ordering
# --------------------------------------------------------------------------

def stencil_to_csr(dom: ODomain, coef: np.ndarray):
    """CSR (value, index, row) with each row sorted by column like extensions/PISO_multiblock_cuda_kernel.cu:3846-3860."""
    D = dom.dims
    N = dom.N
    cols = [np.arange(N)] + [dom.nb[f] for f in range(2 * D)]
    rows_v, rows_i, row_ptr = [], [], [0]
    C = np.stack(cols, 0)
    V = coef
    for i in range(N):
        c = C[:, i]
        v = V[:, i]
        m = c >= 0
        order = np.argsort(c[m], kind="stable")
        rows_i.append(c[m][order])
        rows_v.append(v[m][order])
        row_ptr.append(row_ptr[-1] + int(m.sum()))
    return np.concatenate(rows_v), np.concatenate(rows_i), np.array(row_ptr)


def stencil_to_scipy(dom: ODomain, coef: np.ndarray) -> sp.csr_matrix:
    D = dom.dims
    N = dom.N
    rows, cols, vals = [np.arange(N)], [np.arange(N)], [coef[0]]
    for f in range(2 * D):
        ok = dom.nb[f] >= 0
        rows.append(np.arange(N)[ok])
        cols.append(dom.nb[f][ok])
        vals.append(coef[f + 1][ok])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))


# --------------------------------------------------------------------------
# Krylov solvers with the reference's iteration semantics
# --------------------------------------------------------------------------

@dataclass
class SolveInfo:
    finalResidual: float
    usedIterations: int
    converged: bool
    isFiniteResidual: bool


def _crit(r):
    """NORM2_NORMALIZED: ||r||_2 / sqrt(n) (extensions/cg_solver_kernel.cu:85-90)."""
    return float(np.sqrt(np.dot(r, r)) / math.sqrt(r.shape[0]))


def criterion(r, conv="NORM2_NORMALIZED"):
    """ComputeConvergenceCriterion, extensions/cg_solver_kernel.cu:77-110."""
    n = r.size
    if conv == "NORM2":
        return float(np.linalg.norm(r))
    if conv == "NORM2_NORMALIZED":
        return float(np.linalg.norm(r)) / math.sqrt(n)
    if conv == "ABS_SUM":
        return float(np.abs(r).sum())
    if conv == "ABS_MEAN":
        return float(np.abs(r).sum()) / n
    if conv == "ABS_MAX":
        return float(np.abs(r).max())
    raise KeyError(conv)


def cg(A, b, x0=None, tol=1e-5, maxit=5000, dtype=np.float64, reset=0, return_best=False, conv="NORM2_NORMALIZED",
       rank_deficient=False):
    """cgSolveGPU, extensions/cg_solver_kernel.cu:236-427; `reset` > 0 restarts the iteration
    (r = b - A x, p = r) before every iteration i with (i+1) % reset == 0 (:266-286); `return_best` keeps the
    iterate of the lowest criterion and returns it, with its iteration and criterion, when the solve stops
    unconverged at maxit or after 100 iterations of a non-falling criterion (:330-413); `conv` names the
    convergence criterion (:77-110).  `rank_deficient` uses the reference's operator for singular Laplacians
    (:240-298): with s = sum |diag A| / n^3, A p is replaced by A p + s |p|_1 e and the (re)started residual
    is b - A x + s |x|_1 e (that sign, as the reference computes it)."""
    b = np.asarray(b, dtype=dtype)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=dtype)
    A = A.astype(dtype)
    n = b.size
    s = float(np.abs(A.diagonal()).sum()) / n / n / n if rank_deficient else 0.0

    def residual(x):
        r = b - A @ x
        if rank_deficient:
            r = r + s * float(np.abs(x).sum())
        return r

    r = residual(x)
    p = r.copy()
    rho = float(np.dot(r, r))
    info = SolveInfo(0.0, -1, False, True)
    best, best_it, best_x, last, rising = 0.0, -1, x, 0.0, 0
    for i in range(maxit):
        if reset > 0 and (i + 1) % reset == 0:
            r = residual(x)
            p = r.copy()
            rho = float(np.dot(r, r))
        q = A @ p
        if rank_deficient:
            q = q + s * float(np.abs(p).sum())
        with np.errstate(divide="ignore", invalid="ignore"):  # a vanishing p.q gives inf / nan, as on the device
            alpha = np.float64(rho) / np.float64(np.dot(p, q))
        x = x + alpha * p
        r = r - alpha * q
        crit = criterion(r, conv)
        if not math.isfinite(crit):
            return x, SolveInfo(crit, i, False, False)
        if return_best:
            if i == 0 or crit < best:
                best, best_it, best_x = crit, i, x.copy()
            rising = rising + 1 if (i > 0 and crit >= last) else 0
            last = crit
        info = SolveInfo(crit, i, False, True)
        if crit < tol:
            info.converged = True
            break
        if return_best and (i == maxit - 1 or rising >= 100):
            return best_x, SolveInfo(best, best_it, False, True)
        rhop = rho
        rho = float(np.dot(r, r))
        with np.errstate(divide="ignore", invalid="ignore"):
            beta = np.float64(rho) / np.float64(rhop)
        p = beta * p + r
    return x, info


def bicgstab(A, b, x0=None, tol=1e-5, maxit=5000, dtype=np.float64, conv="NORM2_NORMALIZED"):
    """bicgstabSolveGPU without preconditioner, extensions/bicgstab_solver_kernel.cu:240-360; `conv` names the
    convergence criterion (ComputeConvergenceCriterion, extensions/cg_solver_kernel.cu:77-110)."""
    b = np.asarray(b, dtype=dtype)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=dtype)
    A = A.astype(dtype)
    r = b - A @ x
    rw = r.copy()
    p = r.copy()
    v = np.zeros_like(b)
    nrmr0 = criterion(r, conv)
    if nrmr0 < tol:
        return x, SolveInfo(nrmr0, -1, True, True)
    rho = 0.0
    alpha = omega = 0.0
    info = SolveInfo(0.0, -1, False, True)
    f64 = np.float64
    for i in range(maxit):
        rhop = rho
        rho = float(np.dot(rw, r))
        with np.errstate(divide="ignore", invalid="ignore"):  # breakdowns give inf / nan, as on the device
            if i > 0:
                beta = (f64(rho) / f64(rhop)) * (f64(alpha) / f64(omega))
                p = r + beta * (p - omega * v)
            v = A @ p
            alpha = f64(rho) / f64(np.dot(rw, v))
        r = r - alpha * v
        x = x + alpha * p
        nrmr = criterion(r, conv)
        if not math.isfinite(nrmr):
            return x, SolveInfo(nrmr, i, False, False)
        info = SolveInfo(nrmr, i, False, True)
        if nrmr < tol:
            info.converged = True
            break
        s = r
        t = A @ s
        with np.errstate(divide="ignore", invalid="ignore"):
            omega = f64(np.dot(t, r)) / f64(np.dot(t, t))
        x = x + omega * s
        r = r - omega * t
        nrmr = criterion(r, conv)
        info.finalResidual = nrmr
        if nrmr < tol:
            info = SolveInfo(nrmr, i + 1, True, True)
            break
    return x, info


def ilu0(val, index, row):
    """Incomplete LU factorisation with zero fill (csrilu02, extensions/bicgstab_solver_kernel.cu:196-208):
    the IKJ elimination restricted to the sparsity pattern of the CSR matrix (rows sorted by column).  Returns
    the factor values on the same pattern: L strictly below the diagonal (unit diagonal implied), U on and
    above it."""
    f = np.array(val, dtype=np.float64 if np.asarray(val).dtype == np.float64 else np.asarray(val).dtype)
    n = len(row) - 1
    pos = [dict((int(index[k]), k) for k in range(row[i], row[i + 1])) for i in range(n)]
    diag = [pos[i][i] for i in range(n)]
    for i in range(n):
        for k in range(row[i], row[i + 1]):
            c = int(index[k])
            if c >= i:
                break
            f[k] = f[k] / f[diag[c]]
            for j in range(k + 1, row[i + 1]):
                m = pos[c].get(int(index[j]))
                if m is not None:
                    f[j] -= f[k] * f[m]
    return f


def _precond_apply(kind, A, L, U, y, transpose):
    """One application of the BiCGStab preconditioner, z = M^-1 y (or M^-T y; transposed triangular solves
    at extensions/bicgstab_solver_kernel.cu:270-276, 313-319).  kind "as_reference": the operator the
    reference's build applies, M = T T with T = tril(A) including the diagonal (the matrix values; the
    csrilu02 factors of :196-208 are not what its solves read), reproducing its iterations, residuals and
    solutions; kind "ilu0": M = L U of ilu0()."""
    if kind == "as_reference":
        T = sp.tril(A, 0, format="csr")
        if transpose:
            Tt = T.T.tocsr()
            return spla.spsolve_triangular(Tt, spla.spsolve_triangular(Tt, y, lower=False), lower=False)
        return spla.spsolve_triangular(T, spla.spsolve_triangular(T, y, lower=True), lower=True)
    if not transpose:
        return spla.spsolve_triangular(U, spla.spsolve_triangular(L, y, lower=True, unit_diagonal=True), lower=False)
    return spla.spsolve_triangular(L.T.tocsr(), spla.spsolve_triangular(U.T.tocsr(), y, lower=True), lower=False,
                                   unit_diagonal=True)


def bicgstab_ilu(val, index, row, b, tol=1e-5, maxit=5000, transpose=False, conv="NORM2_NORMALIZED",
                 preconditioner="as_reference"):
    """bicgstabSolveGPU with its preconditioner (extensions/bicgstab_solver_kernel.cu:240-360): right
    preconditioning, p^ = M^-1 p and s^ = M^-1 s (M per _precond_apply), from x = 0; `transpose` solves with
    A^T and M^T.  Iteration bookkeeping as bicgstab()."""
    val = np.asarray(val, dtype=np.float64)
    n = len(row) - 1
    A0 = sp.csr_matrix((val, np.asarray(index), np.asarray(row)), shape=(n, n))
    L = U = None
    if preconditioner == "ilu0":
        f = ilu0(val, index, row)
        F = sp.csr_matrix((f, np.asarray(index), np.asarray(row)), shape=(n, n))
        L = sp.tril(F, -1, format="csr")
        U = sp.triu(F, 0, format="csr")
    elif preconditioner != "as_reference":
        raise KeyError(preconditioner)
    A = A0.T.tocsr() if transpose else A0
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    r = b.copy()
    rw = r.copy()
    p = r.copy()
    v = np.zeros_like(b)
    nrmr0 = criterion(r, conv)
    if nrmr0 < tol:
        return x, SolveInfo(nrmr0, -1, True, True)
    rho = alpha = omega = 0.0
    info = SolveInfo(0.0, -1, False, True)
    for i in range(maxit):
        rhop = rho
        rho = float(np.dot(rw, r))
        if i > 0:
            beta = (rho / rhop) * (alpha / omega)
            p = r + beta * (p - omega * v)
        pw = _precond_apply(preconditioner, A0, L, U, p, transpose)
        v = A @ pw
        alpha = rho / float(np.dot(rw, v))
        r = r - alpha * v
        x = x + alpha * pw
        nrmr = criterion(r, conv)
        if not math.isfinite(nrmr):
            return x, SolveInfo(nrmr, i, False, False)
        info = SolveInfo(nrmr, i, False, True)
        if nrmr < tol:
            info.converged = True
            break
        s = _precond_apply(preconditioner, A0, L, U, r, transpose)
        t = A @ s
        omega = float(np.dot(t, r)) / float(np.dot(t, t))
        x = x + omega * s
        r = r - omega * t
        nrmr = criterion(r, conv)
        info.finalResidual = nrmr
        if nrmr < tol:
            info = SolveInfo(nrmr, i + 1, True, True)
            break
    return x, info


def solve(A, b, use_bicg: bool, tol: float, maxit: int = 5000, method: str = "iterative"):
    """Linear solve as the simulation driver issues it (PISOtorch_diff.py:245-293): an all-zero RHS gives x=0."""
    if not np.any(b != 0):
        return np.zeros_like(b), SolveInfo(0.0, 0, True, True)
    if method == "direct":
        import scipy.sparse.linalg as spla
        x = spla.spsolve(A.tocsc(), b)
        return x, SolveInfo(0.0, 0, True, True)
    if use_bicg:
        return bicgstab(A, b, tol=tol, maxit=maxit)
    return cg(A, b, tol=tol, maxit=maxit)


# --------------------------------------------------------------------------
# PISO step (PISOtorch_simulation.py:1054-1327, orthogonal branch)
# --------------------------------------------------------------------------

@dataclass
class StepResult:
    C: np.ndarray
    A: np.ndarray
    velocityRHS: np.ndarray
    u_star: np.ndarray
    P: np.ndarray
    pressureRHS: np.ndarray
    pressureRHSdiv: np.ndarray
    pressure: np.ndarray
    velocity: np.ndarray
    infos: list


def piso_step(dom: ODomain, dt: float, corrector_steps: int = 2, adv_tol: float = 1e-5,
              p_tol: float = 1e-5, method: str = "iterative", maxit: int = 5000,
              normalize_pressure: bool = True, non_ortho_flags: int = 0, advect_non_ortho_steps: int = 1,
              pressure_non_ortho_steps: int = 1) -> StepResult:
    """One PISO step, Simulation._PISO_split_step, PISOtorch_simulation.py:1054-1327: the orthogonal branch, or
    with non_ortho_flags the non-orthogonal branch (PISOtorch_simulation.py:1194-1296).

    Updates the block velocity and pressure of ``dom`` in place and returns the intermediate fields
    of the last corrector for inspection.
    """
    if non_ortho_flags:
        return _piso_step_nonortho(dom, dt, corrector_steps, adv_tol, p_tol, method, maxit, normalize_pressure,
                                   non_ortho_flags, advect_non_ortho_steps, pressure_non_ortho_steps)
    D = dom.dims
    N = dom.N
    infos = []
    Ccoef, A = advection_matrix(dom, dt)
    rhs = advection_rhs(dom, dt)
    Cm = stencil_to_scipy(dom, Ccoef)
    u_star = np.zeros((D, N))
    for c in range(D):  # nBatches = D, solved one after another (extensions/bicgstab_solver_kernel.cu:221)
        u_star[c], info = solve(Cm, rhs[c], True, adv_tol, maxit, method)
        infos.append(("adv", c, info))
    u_cur = u_star
    P = h = div = p = None
    for _ in range(corrector_steps):
        P = pressure_matrix(dom, A)
        h = pressure_rhs(dom, dt, Ccoef, A, u_cur)
        div = divergence(dom, h)
        Pm = stencil_to_scipy(dom, P)
        p, info = solve(Pm, div, False, p_tol, maxit, method)
        infos.append(("p", 0, info))
        if normalize_pressure:
            p = p - p.mean()  # PISOtorch_simulation.py:1243-1244
        dom.set_pressure_global(p)  # CopyPressureResultToBlocks
        u_cur = correct_velocity(dom, p, A, h)
    dom.set_velocity_global(u_cur)  # CopyVelocityResultToBlocks
    return StepResult(Ccoef, A, rhs, u_star, P, h, div, p, u_cur, infos)


def _piso_step_nonortho(dom, dt, corrector_steps, adv_tol, p_tol, method, maxit, normalize_pressure, flags,
                        advect_steps, pressure_steps):
    """The non-orthogonal branch of Simulation._PISO_split_step, PISOtorch_simulation.py:1194-1296: the velocity
    result is copied from the blocks and feeds the explicit terms of the velocity RHS; every corrector
    builds P with the non-orthogonal terms, h and div h plus the explicit terms of the current pressure
    result, solves from zero (each further non-orthogonal pressure step reuses h), subtracts the mean
    and corrects the velocity."""
    D = dom.dims
    N = dom.N
    infos = []
    Ccoef, A = advection_matrix(dom, dt, flags)
    Cm = stencil_to_scipy(dom, Ccoef)
    u_res = dom.velocity_global()  # CopyVelocityResultFromBlocks
    rhs = None
    for _ in range(advect_steps):
        rhs = advection_rhs(dom, dt, flags, u_res)
        u_new = np.zeros((D, N))
        for c in range(D):
            u_new[c], info = solve(Cm, rhs[c], True, adv_tol, maxit, method)
            infos.append(("adv", c, info))
        u_res = u_new
    u_star = u_res
    u_cur = u_star
    P = h = div = p = None
    for _ in range(corrector_steps):
        P = pressure_matrix(dom, A, flags)
        Pm = stencil_to_scipy(dom, P)
        h = pressure_rhs(dom, dt, Ccoef, A, u_cur)
        div0 = divergence(dom, h)
        for _ in range(pressure_steps):
            div = pressure_rhs_nonortho(dom, flags, div0, A, dom.p_result)
            p, info = solve(Pm, div, False, p_tol, maxit, method)
            infos.append(("p", 0, info))
            if normalize_pressure:
                p = p - p.mean()
            dom.p_result = p
        dom.set_pressure_global(p)  # CopyPressureResultToBlocks
        u_cur = correct_velocity(dom, p, A, h)
    dom.set_velocity_global(u_cur)
    return StepResult(Ccoef, A, rhs, u_star, P, h, div, p, u_cur, infos)


def _face_broadcast(dom: ODomain, bi: int, face: int, v: np.ndarray) -> np.ndarray:
    """A boundary tensor [1,C] (static) or [1,C,face zyx] as [1,C,face zyx]."""
    b = dom.blocks[bi]
    D = dom.dims
    shape = list(b.velocity.shape[2:])
    shape[D - 1 - (face >> 1)] = 1
    v = np.asarray(v, dtype=np.float64)
    if v.ndim == 2:
        v = v.reshape(v.shape + (1,) * D)
    return np.broadcast_to(v, v.shape[:2] + tuple(shape)).copy()


def boundary_fluxes(dom: ODomain, bi: int, face: int) -> np.ndarray:
    """FixedBoundary::GetFluxes (extensions/domain_structs.cpp:527-542): per face cell the face-normal
    flux det * (M^-1 u)_axis of the boundary velocity, or u_axis without a boundary transform."""
    D = dom.dims
    axis = face >> 1
    bnd = dom.blocks[bi].boundaries[face]
    u = _face_broadcast(dom, bi, face, bnd.velocity)  # [1,D,zyx]
    if bnd.transform is None:
        return u[:, axis]
    T = bnd.transform  # [1, zyx, T]
    row = T[..., D * D + axis * D: D * D + (axis + 1) * D]
    return T[..., -1] * np.einsum("...c,...c->...", row, np.moveaxis(u, 1, -1))


def advective_outflow(dom: ODomain, faces, velm, dt: float, tol: Optional[float] = None):
    """update_advective_boundaries with a static characteristic velocity, then balance_boundary_fluxes
    (sim.py:145-312).  Every (block, face) of `faces` holds a varying Dirichlet velocity; it moves
    towards the adjacent cell layer by t = 1 - 1/(1 + 2 dt c), c the face-normal component of `velm`
    (in computational coordinates with a boundary transform: row `axis` of M^-1 times velm).  Then,
    unless the net outward flux of all fixed faces is within 1% of the tolerance (default 1e-8, the
    FP64 solver default of PISOtorch_diff.py:183-189) of zero, the free faces' velocities are scaled by
    -(flux of the other fixed faces) / (flux of the free faces)."""
    D = dom.dims
    velm = np.asarray(velm, dtype=np.float64).reshape(1, D)
    faces = [(int(b), int(f)) for b, f in faces]
    for bi, face in faces:
        b = dom.blocks[bi]
        bnd = b.boundaries[face]
        assert bnd.kind == "fixed" and np.asarray(bnd.velocity).ndim == D + 2, "outflow faces must be varying"
        axis = face >> 1
        ax = 2 + (D - 1 - axis)
        layer = np.take(b.velocity, [b.velocity.shape[ax] - 1 if (face & 1) else 0], axis=ax)
        if bnd.transform is not None:
            row = bnd.transform[..., D * D + axis * D: D * D + (axis + 1) * D]  # [1, zyx, D]
            c = np.einsum("...c,c->...", row, velm[0])[:, None]  # [1,1,zyx]
        else:
            c = velm[:, axis].reshape((1, 1) + (1,) * D)
        t = 1.0 - 1.0 / (1.0 + 2.0 * dt * c)
        vb = bnd.velocity
        bnd.velocity = vb - t * (vb - layer)
    fixed = free = 0.0
    for bi, b in enumerate(dom.blocks):
        for f, bnd in enumerate(b.boundaries):
            if bnd.kind != "fixed":
                continue
            flux = float(np.sum(boundary_fluxes(dom, bi, f)))
            flux = flux if (f & 1) else -flux
            if (bi, f) in faces:
                free += flux
            else:
                fixed += flux
    tol = 1e-8 if tol is None else tol
    if abs(fixed + free) > tol * 0.01:
        scale = -fixed / free
        for bi, face in faces:
            bnd = dom.blocks[bi].boundaries[face]
            bnd.velocity = bnd.velocity * scale


def run_steps(dom: ODomain, steps: int, dt: float, **kw):
    res = None
    for _ in range(steps):
        res = piso_step(dom, dt, **kw)
    return res
