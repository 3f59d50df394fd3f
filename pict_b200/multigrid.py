"""Multigrid hierarchy of a (batched) domain for the multigrid-preconditioned CG of ``libpict_b200``.

Eligible domains: every system is one block whose faces are fixed or periodic (no connections).
Level l+1 halves every block of level l along its strongly coupled axes (ceil(n/2) cells; all axes
on isotropic grids, the stretched axis first on stretched ones) until every block has at most 4
cells along each axis.  The block tables and cell-to-block maps
are built once on the host; the coarse stencils are recomputed on the device (Galerkin product)
whenever the finest matrix changes.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._lib import MgLevel, check

MAX_LEVELS = 16
TILE_CELLS = 512           # cells per work tile of the coarse levels
STAGE_CELLS = 4096         # cells per array of the shared-memory stage of the 2D restriction / prolongation
SUB_MAX_CELLS = 2048       # the V-cycle runs in one CTA per block from the first level whose blocks have at
SUB_MAX_SMEM = 160 * 1024  # most this many cells and whose sub-cycle fits this much shared memory


def eligible(host_blocks, num_blocks, dims, sim_of_block) -> Optional[str]:
    """None if a multigrid hierarchy can be built, else the reason."""
    seen = set()
    for b in range(num_blocks):
        B = host_blocks[b]
        if B.sim in seen:
            return "a system has more than one block"
        seen.add(B.sim)
        for f in range(2 * dims):
            if B.face[f].type == _lib.PICT_FACE_CONNECTED:
                return "connected block faces"
    return None


def axis_strengths(domain) -> np.ndarray:
    """Mean orthogonal Laplace coefficient det |Minv row a|^2 per block and axis (the coupling strength
    of the pressure operator along each axis; 1 without transforms): [num_blocks, 3]."""
    D = domain.getSpatialDims()
    out = np.ones((len(domain.getBlocks()), 3))
    for k, b in enumerate(domain.getBlocks()):
        tr = getattr(b, "transform", None)
        if tr is None or tr.numel() == 0:
            continue
        t = tr.reshape(-1, 2 * D * D + 1).double()
        det = t[:, -1]
        minv = t[:, D * D:2 * D * D].reshape(-1, D, D)
        alpha = det[:, None] * (minv ** 2).sum(dim=2)
        out[k, :D] = alpha.mean(dim=0).cpu().numpy()
    return out


def two_sweep_fits(fine_sizes, fine_per, coarse_offs, coarse_sizes, coarse_shifts, coarse_tiles, fine_tiles,
                   dims: int) -> bool:
    """True if the tile kernels can smooth level l with two Jacobi sweeps: 2D, no y-periodic block, every
    coarse tile's fine rows plus two halo rows on each side fit the restriction's stage, and every tile of
    level l plus three halo rows on each side fits the four-array stage of the prolongation (fine_tiles None:
    the domain's tiles, checked at launch)."""
    if dims != 2 or bool(fine_per[:, 1].any()):
        return False
    t = coarse_tiles.reshape(-1, 4)
    for sim, b, s0, cnt in t:
        sxc = int(coarse_sizes[b, 0])
        lc0 = int(s0) - int(coarse_offs[b])
        lc1 = lc0 + int(cnt) - 1
        shy = int(coarse_shifts[b, 1])
        ylo = max(0, ((lc0 // sxc) << shy) - 2)
        yhi = min(int(fine_sizes[b, 1]) - 1, ((lc1 // sxc + 1) << shy) + 1)
        if (yhi - ylo + 1) * int(fine_sizes[b, 0]) > STAGE_CELLS:
            return False
    if fine_tiles is not None:
        for sim, b, s0, cnt in fine_tiles.reshape(-1, 4):
            if int(cnt) + 6 * int(fine_sizes[b, 0]) > (3 * STAGE_CELLS) // 4:
                return False
    return True


def level_tiles(offs, counts, sims, tile: int = TILE_CELLS) -> np.ndarray:
    """Work tiles of a coarse level, [num_tiles * 4]: system, block, first cell, cell count (each
    block split into runs of at most `tile` cells)."""
    out = []
    for b, (o, n) in enumerate(zip(offs, counts)):
        for s0 in range(0, int(n), tile):
            out.append((int(sims[b]), b, int(o) + s0, min(tile, int(n) - s0)))
    return np.array(out, dtype=np.int32).reshape(-1)


class MGHierarchy:
    """Levels of the multigrid preconditioner.  At every level an axis of a block is halved if its
    coupling strength is at least `theta` times the strongest of the block (semi-coarsening on stretched
    grids); strengths of the coarse Galerkin operator grow with the number of fine faces a coarse face
    sums (the product of the factors of the other axes)."""

    def __init__(self, host_blocks, num_blocks: int, dims: int, dtype, device, cell_block_dev: torch.Tensor,
                 strengths: Optional[np.ndarray] = None, min_size: int = 4, theta: float = 0.5):
        why = eligible(host_blocks, num_blocks, dims, None)
        if why is not None:
            raise ValueError("multigrid not applicable: " + why)
        self.dims = dims
        self.K = 2 * dims + 1
        self.dtype = dtype
        self.device = device
        code = _lib.PICT_F64 if dtype == torch.float64 else _lib.PICT_F32
        sizes = np.array([[host_blocks[b].size[a] for a in range(3)] for b in range(num_blocks)], dtype=np.int64)
        per = np.array([[1 if (host_blocks[b].face[2 * a].type == _lib.PICT_FACE_PERIODIC) else 0 for a in range(3)]
                        for b in range(num_blocks)], dtype=np.int64)
        per[:, dims:] = 0
        sims = np.array([host_blocks[b].sim for b in range(num_blocks)], dtype=np.int64)
        strength = np.ones((num_blocks, 3)) if strengths is None else np.array(strengths, dtype=np.float64)
        strength[:, dims:] = 0.0
        shifts = np.zeros((num_blocks, 3), dtype=np.int64)
        self.levels_py = []   # keep tensors alive
        self.shifts = []
        levels = []
        host_geo = []         # per level: sizes, periodic flags, offsets, shifts, tiles (host copies)
        for lvl in range(MAX_LEVELS):
            n = sizes.prod(axis=1)
            offs = np.concatenate([[0], np.cumsum(n)[:-1]])
            table = np.zeros((num_blocks, 12), dtype=np.int32)
            table[:, 0] = offs
            table[:, 1:4] = sizes
            table[:, 4:7] = per
            table[:, 7] = sims
            table[:, 8:11] = shifts
            blocks_t = torch.tensor(table.reshape(-1), dtype=torch.int32, device=device)
            if lvl == 0:
                cb = cell_block_dev
                coef = None
            else:
                cb = torch.tensor(np.repeat(np.arange(num_blocks, dtype=np.int32), n), dtype=torch.int32, device=device)
                coef = torch.zeros(self.K * int(n.sum()), dtype=dtype, device=device)
            L = MgLevel()
            L.num_cells = int(n.sum())
            L.num_blocks = num_blocks
            L.dims = dims
            L.dtype = code
            L.blocks = blocks_t.data_ptr()
            L.cell_block = cb.data_ptr()
            L.coef = coef.data_ptr() if coef is not None else None
            L.max_block_cells = int(n.max())
            L.max_block_sx = int(sizes[:, 0].max())
            tiles_t = None
            if lvl > 0:
                tiles_t = torch.tensor(level_tiles(offs, n, sims), dtype=torch.int32, device=device)
                L.num_tiles = tiles_t.numel() // 4
                L.tiles = tiles_t.data_ptr()
            levels.append(L)
            self.levels_py.append((blocks_t, cb, coef, tiles_t))
            self.shifts.append(shifts.copy())
            host_geo.append((sizes.copy(), per.copy(), offs.copy(), shifts.copy(),
                             level_tiles(offs, n, sims) if lvl > 0 else None))
            if (sizes[:, :dims] <= min_size).all():
                break
            # choose the axes to halve per block
            can = sizes > 1
            can[:, dims:] = False
            s_can = np.where(can, strength, 0.0)
            smax = s_can.max(axis=1, keepdims=True)
            shifts = ((s_can >= theta * smax) & can).astype(np.int64)
            none = shifts.sum(axis=1) == 0
            shifts[none] = can[none].astype(np.int64)  # degenerate: halve what can be halved
            fac = 1 << shifts
            prod = fac[:, :dims].prod(axis=1, keepdims=True)
            strength[:, :dims] = strength[:, :dims] * prod / fac[:, :dims]
            sizes = np.where(shifts == 1, (sizes + 1) // 2, sizes)
        if int(sizes[:, :dims].prod(axis=1).max()) > 256:
            raise ValueError("multigrid not applicable: coarsest blocks too large")
        for l in range(len(levels) - 1):
            fs, fp, _, _, ft = host_geo[l]
            cs, _, co, csh, ct = host_geo[l + 1]
            levels[l].sweeps = 2 if two_sweep_fits(fs, fp, co, cs, csh, ct, ft, dims) else 1
        levels[-1].sweeps = 1
        self.num_levels = len(levels)
        self.levels = (MgLevel * self.num_levels)(*levels)
        self.cells = [int(L.num_cells) for L in levels]

    def sub_level(self) -> int:
        """First level of the part of the V-cycle that runs in one launch (one CTA per block)."""
        if self.num_levels == 1:
            return 0
        esz = 8 if self.dtype == torch.float64 else 4
        for l in range(1, self.num_levels):
            cells = [int(self.levels[k].max_block_cells) for k in range(l, self.num_levels)]
            smem = esz * (cells[0] + (2 + self.K) * sum(cells))
            if cells[0] <= SUB_MAX_CELLS and smem <= SUB_MAX_SMEM:
                return l
        return self.num_levels - 1

    def launches_per_vcycle(self) -> int:
        lc = self.sub_level()
        return 2 * lc + 1 if lc > 0 else 3

    def setup(self, fine_coef: torch.Tensor, stream):
        """Point level 0 at the finest stencil and recompute every coarse stencil."""
        self.levels[0].coef = fine_coef.data_ptr()
        lib = _lib.load()
        for l in range(self.num_levels - 1):
            check(lib.pict_mg_galerkin(ctypes.byref(self.levels[l]), ctypes.byref(self.levels[l + 1]), stream),
                  "mg galerkin")

    def workspace_bytes(self, desc) -> int:
        return int(_lib.load().pict_pcg_mg_workspace_bytes(ctypes.byref(desc), self.levels, self.num_levels))

    def solve(self, desc, rhs: torch.Tensor, x: torch.Tensor, iterations: int, tol: float, info: torch.Tensor,
              ws: torch.Tensor, stream, omega: float = 0.8, prolong_scale: float = 2.0, coarse_sweeps: int = 8):
        check(_lib.load().pict_pcg_mg(ctypes.byref(desc), self.levels, self.num_levels, ctypes.c_void_p(rhs.data_ptr()),
                                      ctypes.c_void_p(x.data_ptr()), int(iterations), float(tol),
                                      _lib.PICT_CONV_NORM2_NORMALIZED, ctypes.c_void_p(info.data_ptr()),
                                      ctypes.c_void_p(ws.data_ptr()), ws.numel(), float(omega), float(prolong_scale),
                                      int(coarse_sweeps), stream), "pcg mg")


def hierarchy_for(domain) -> MGHierarchy:
    """Build the hierarchy of a prepared Domain or BatchDomain (raises ValueError if not eligible)."""
    host = domain._host_blocks if hasattr(domain, "_host_blocks") and not callable(domain._host_blocks) else None
    if host is None:
        host = domain._pack_blocks()
    nb = len(domain.getBlocks())
    return MGHierarchy(host, nb, domain.getSpatialDims(), domain.getDtype(), domain.getDevice(), domain._cell_block,
                       strengths=axis_strengths(domain))
