"""Batched simulation: many independent prepared ``PISOtorch.Domain`` objects in one launch per stage.

``BatchDomain`` packs the blocks of several single-simulation domains into one
block table with a system index per block, concatenates their global vectors
and keeps a per-system viscosity and time step on the device.  Every kernel of
the step then covers all simulations in one launch; the Krylov kernels pull
systems from a device work queue (largest first), so uneven sizes and
iteration counts balance across the SMs.

The fields stay in the member domains' own block tensors (velocity, pressure),
so each ``Domain`` remains usable on its own before and after batched steps.
This has no counterpart in the reference, which runs one domain per call; the
per-simulation numerics are those of the plain step.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence

import torch

from . import _lib
from ._lib import BlockDesc, DomainDesc, check
from . import PISOtorch as P


class _Coef:
    def __init__(self, coef):
        self.coef = coef


class BatchDomain:
    def __init__(self, domains: Sequence["P.Domain"], time_steps=None, order="largest_first", tile_cells=None):
        _ok = P._check
        _ok(len(domains) > 0, "BatchDomain needs at least one domain")
        d0 = domains[0]
        self._dims = d0.getSpatialDims()
        self._dtype = d0.getDtype()
        self._device = d0.getDevice()
        for d in domains:
            _ok(d.getSpatialDims() == self._dims and d.getDtype() == self._dtype and d.getDevice() == self._device,
                "all batched domains must share dims, dtype and device")
            _ok(d.IsInitialized(), "batched domains must be prepared (PrepareSolve)")
        self.domains = list(domains)
        n = len(domains)
        sizes = [d.getTotalSize() for d in domains]
        if order == "largest_first":
            self.order = sorted(range(n), key=lambda i: -sizes[i])
        else:
            self.order = list(range(n))
        self.num_sims = n
        self.tile_cells = P.TILE_CELLS if tile_cells is None else int(tile_cells)
        self._pack(time_steps)

    # -- Domain-like accessors used by the step engine --
    def getSpatialDims(self):
        return self._dims

    def getDtype(self):
        return self._dtype

    def getDevice(self):
        return self._device

    def getBlocks(self):
        return [b for i in self.order for b in self.domains[i].getBlocks()]

    def getTotalSize(self):
        return self._N

    def IsTensorChanged(self):
        return any(d.IsTensorChanged() for d in self.domains)

    def _check_ready(self):
        if self.IsTensorChanged():
            self.UpdateDomainData()

    def sim_slice(self, i):
        """Cell range [start, end) of member domain i in the batched global vectors."""
        return self._sim_range[i]

    def _pack(self, time_steps):
        D = self._dims
        host = []
        sim_cells = [0]
        sim_blocks = [0]
        self._sim_range = {}
        offset = 0
        for si, di in enumerate(self.order):
            d = self.domains[di]
            arr = d._pack_blocks()
            base = len(host)
            start = offset
            for k in range(len(arr)):
                b = BlockDesc()
                ctypes.memmove(ctypes.byref(b), ctypes.byref(arr[k]), ctypes.sizeof(BlockDesc))
                b.offset = arr[k].offset + offset
                b.sim = si
                for f in range(2 * D):
                    if b.face[f].type == _lib.PICT_FACE_CONNECTED:
                        b.face[f].conn_block += base
                host.append(b)
            offset += d.getTotalSize()
            self._sim_range[di] = (start, offset)
            sim_cells.append(offset)
            sim_blocks.append(len(host))
        self._N = offset
        N = offset
        self._host_blocks = (BlockDesc * len(host))(*host)
        nbr = torch.empty((2 * D, N), dtype=torch.int32)
        cb = torch.empty(N, dtype=torch.int32)
        check(_lib.load().pict_build_topology(self._host_blocks, len(host), D, N, nbr.data_ptr(), cb.data_ptr()),
              "build_topology")
        dev = self._device
        self._nbr = nbr.to(dev)
        self._cell_block = cb.to(dev)
        self._sim_cells = torch.tensor(sim_cells, dtype=torch.int32, device=dev)
        self._sim_blocks = torch.tensor(sim_blocks, dtype=torch.int32, device=dev)
        self._n_host_blocks = len(host)
        self._tiles, self._sim_tiles, self._num_tiles = P.build_tiles(self._host_blocks, len(host), self.num_sims, dev,
                                                                      self.tile_cells)
        self._sim_visc = torch.tensor([float(self.domains[i].viscosity.item()) for i in self.order],
                                      dtype=self._dtype, device=dev)
        self.max_sim_cells = max(sim_cells[k + 1] - sim_cells[k] for k in range(self.num_sims))
        opts = dict(dtype=self._dtype, device=dev)
        K = 2 * D + 1
        self.C = _Coef(torch.zeros((K, N), **opts))
        self.P = _Coef(torch.zeros((K, N), **opts))
        self.A = torch.zeros(N, **opts)
        self.velocityRHS = torch.zeros(D * N, **opts)
        self.velocityResult = torch.zeros(D * N, **opts)
        self.pressureRHS = torch.zeros(D * N, **opts)
        self.pressureRHSdiv = torch.zeros(N, **opts)
        self.pressureResult = torch.zeros(N, **opts)
        raw = bytes(self._host_blocks)
        self._blocks_dev = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
        self.set_time_steps(time_steps)

    def set_time_steps(self, time_steps):
        """Per-simulation time steps (in member order); None keeps the scalar passed to each step."""
        if time_steps is None:
            self._sim_dt = None
        else:
            ts = [float(t) for t in time_steps]
            P._check(len(ts) == self.num_sims, "one time step per batched domain")
            self._sim_dt = torch.tensor([ts[i] for i in self.order], dtype=self._dtype, device=self._device)
        self._desc = self._make_desc()

    def set_tile_cells(self, tile_cells):
        """Cells per Krylov work tile (1..2048): rebuilds the tile table.  Steppers created before the
        change must be re-created (their workspace depends on the tile count)."""
        tile_cells = int(tile_cells)
        P._check(1 <= tile_cells <= 2048, "tile_cells must be in [1, 2048]")
        self.tile_cells = tile_cells
        self._tiles, self._sim_tiles, self._num_tiles = P.build_tiles(self._host_blocks, self._n_host_blocks,
                                                                      self.num_sims, self._device, tile_cells)
        self._desc = self._make_desc()

    def set_viscosities(self, nus):
        P._check(len(nus) == self.num_sims, "one viscosity per batched domain")
        self._sim_visc.copy_(torch.tensor([float(nus[i]) for i in self.order], dtype=self._dtype))

    def pack_state(self):
        """Place the velocity and the pressure of every block of the batch in one contiguous device tensor
        each (batch block order, each block's field contiguous inside), and make the blocks' fields views
        of them.  The member domains stay usable on their own; the whole batch state then moves between
        host and device in one copy per field and direction instead of one per block.  Returns
        (velocity_arena, pressure_arena)."""
        blocks = self.getBlocks()
        opts = dict(dtype=self._dtype, device=self._device)
        va = torch.empty(sum(b.velocity.numel() for b in blocks), **opts)
        pa = torch.empty(sum(b.pressure.numel() for b in blocks), **opts)
        ov = op = 0
        for b in blocks:
            n = b.velocity.numel()
            v = va[ov:ov + n].view(b.velocity.shape)
            v.copy_(b.velocity)
            b.setVelocity(v)
            ov += n
            n = b.pressure.numel()
            p = pa[op:op + n].view(b.pressure.shape)
            p.copy_(b.pressure)
            b.setPressure(p)
            op += n
        self.velocity_arena, self.pressure_arena = va, pa
        self.UpdateDomainData()
        return va, pa

    def UpdateDomainData(self):
        """Re-pack after member tensors were replaced (pointers change)."""
        for d in self.domains:
            if d.IsTensorChanged():
                d.UpdateDomainData()
        dt = None if self._sim_dt is None else self._sim_dt
        self._pack(None)
        self._sim_dt = dt
        self._desc = self._make_desc()

    def _make_desc(self):
        d = DomainDesc()
        d.dims = self._dims
        d.num_blocks = len(self._host_blocks)
        d.num_cells = self._N
        d.num_sims = self.num_sims
        d.dtype = P._dtype_code(self._dtype)
        d.max_sim_cells = self.max_sim_cells
        d.blocks = self._blocks_dev.data_ptr()
        d.nbr = self._nbr.data_ptr()
        d.cell_block = self._cell_block.data_ptr()
        d.sim_cells = self._sim_cells.data_ptr()
        d.sim_blocks = self._sim_blocks.data_ptr()
        d.tiles = self._tiles.data_ptr()
        d.sim_tiles = self._sim_tiles.data_ptr()
        d.num_tiles = self._num_tiles
        d.tile_cells = self.tile_cells
        d.sim_viscosity = self._sim_visc.data_ptr()
        d.sim_dt = None if self._sim_dt is None else self._sim_dt.data_ptr()
        d.C = self.C.coef.data_ptr()
        d.A = self.A.data_ptr()
        d.P = self.P.coef.data_ptr()
        d.velocity_rhs = self.velocityRHS.data_ptr()
        d.velocity_result = self.velocityResult.data_ptr()
        d.pressure_rhs = self.pressureRHS.data_ptr()
        d.pressure_rhs_div = self.pressureRHSdiv.data_ptr()
        d.pressure_result = self.pressureResult.data_ptr()
        return d
