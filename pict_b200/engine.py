"""Fused PISO step engine: the whole time step as a short, host-sync-free launch sequence.

``PISOStepper`` advances a prepared ``PISOtorch.Domain`` (one simulation, or a
batch of independent simulations packed into one domain by
``pict_b200.batch``) by full PISO steps with the same sequence as the
reference driver's orthogonal branch (``Simulation._PISO_split_step``,
PISOtorch_simulation.py:1054-1327):

1. advection matrix C, diagonal A and velocity RHS in one pass
   (SetupAdvectionMatrix + SetupAdvectionVelocity);
2. one persistent BiCGStab launch for all D velocity components;
3. per corrector: pressure matrix (first corrector only: it depends on A and
   the metrics alone, so rebuilding it is redundant) + H/A RHS + divergence,
   one persistent CG launch that also removes the mean pressure and writes the
   blocks' pressure (CopyPressureResultToBlocks), then the velocity
   correction, which on the last corrector also stores the blocks' velocity
   (CopyVelocityResultToBlocks).

No host synchronisation happens inside a step; solver reports land in a device
buffer and are checked by :meth:`check` (raising ``LinsolveError`` like the
reference's wrapper, PISOtorch_diff.py:199-243).  The sequence is CUDA-graph
capturable (:meth:`capture`).
"""
from __future__ import annotations

import ctypes
import warnings
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import check
from . import PISOtorch as P


class LinsolveError(RuntimeError):
    pass


def default_tolerance(dtype):
    """_get_solver_tolerance, PISOtorch_diff.py:183-189."""
    return 1e-8 if dtype == torch.float64 else 1e-5


class PISOStepper:
    def __init__(self, domain, time_step=None, corrector_steps: int = 2, advection_tol: Optional[float] = None,
                 pressure_tol: Optional[float] = None, max_iterations: int = 5000, adv_group_size: int = 0,
                 p_group_size: int = 0, threads: int = 0, normalize_pressure: bool = True, cg_variant: int = 1,
                 pressure_refine: int = 0, refine_tol: Optional[float] = None, warm_start_pressure: bool = False,
                 refine_solver: str = "cg", mg_iterations: int = 0, pressure_first_solve: bool = True,
                 warm_start_advection: bool = False, outflow=None, outflow_velocity=None,
                 outflow_tol: Optional[float] = None):
        self.domain = domain
        self.dims = domain.getSpatialDims()
        self.corrector_steps = int(corrector_steps)
        dt = domain.getDtype()
        self.adv_tol = default_tolerance(dt) if advection_tol is None else float(advection_tol)
        self.p_tol = default_tolerance(dt) if pressure_tol is None else float(pressure_tol)
        self.max_iterations = int(max_iterations)
        self.normalize_pressure = normalize_pressure
        self.time_step = time_step
        # warm start of the advection solve from the blocks' velocity (advect_use_prev_result of
        # PISOtorch_simulation.py:1189): the same solution to the tolerance, fewer BiCGStab iterations.
        # "increment": from the blocks' velocity plus the advection increment u* - u extrapolated from the two
        # previous steps (the increment changes slowly; on viscous-dominated cavities 6-7 instead of 11-12
        # iterations)
        self.advection_increment = warm_start_advection == "increment"
        self.warm_start_advection = bool(warm_start_advection)
        self._adv_incr = None
        self.adv_params = P._solve_params(self.dims, self.max_iterations, self.adv_tol, _lib.PICT_CONV_NORM2_NORMALIZED,
                                          True, False, x_zero=not self.warm_start_advection, group_size=adv_group_size,
                                          threads=threads)
        # mixed precision: `pressure_refine` FP64 refinement sweeps after the first pressure solve, each
        # solving the correction of the FP64 residual to `refine_tol`
        self.pressure_refine = int(pressure_refine)
        self.refine_tol = (1e-9 if refine_tol is None else float(refine_tol))
        refine = self.pressure_refine > 0
        # warm start: every pressure solve starts from pressureResult (the previous corrector's or step's
        # mean-free pressure) instead of zero; same solution, fewer iterations
        self.warm_start_pressure = bool(warm_start_pressure)
        # "increment": corrector k >= 1 of the refined solve starts from corrector k-1's pressure plus the previous
        # step's difference between the two, and the first corrector from the linear extrapolation of the first
        # correctors' pressures of the two previous steps (the pressure changes smoothly from step to step; on
        # cavities the initial residuals fall 10-180x)
        self.pressure_increment = warm_start_pressure == "increment"
        self._p_delta = None
        self._p0_hist = None
        self._p0_count = 0
        self.p_params = P._solve_params(1, self.max_iterations, self.p_tol, _lib.PICT_CONV_NORM2_NORMALIZED, False,
                                        False, x_zero=not self.warm_start_pressure,
                                        subtract_mean=normalize_pressure and not refine,
                                        write_block_pressure=not refine, group_size=p_group_size, threads=threads,
                                        variant=cg_variant)
        # correction solves of the refinement: "cg" (persistent CG), "mg" (multigrid-preconditioned CG,
        # single-block systems only; falls back to "cg" otherwise) or "auto" (multigrid on near-isotropic
        # grids, CG on strongly stretched ones)
        self.refine_solver = refine_solver
        # with refinement, the first FP32 pressure solve can be left out: the refinement sweeps then start
        # from the warm-start pressure (needs warm_start_pressure)
        self.pressure_first_solve = bool(pressure_first_solve) or not (self.pressure_refine > 0 and self.warm_start_pressure)
        self.mg_iterations = int(mg_iterations)
        self._mg = None
        self.r_params = P._solve_params(1, self.max_iterations, self.refine_tol, _lib.PICT_CONV_NORM2_NORMALIZED, False,
                                        False, x_zero=True, group_size=p_group_size, threads=threads,
                                        variant=cg_variant)
        # advective outflow faces, updated on the device at the start of every step like the reference
        # samples' prep_fn (update_advective_boundaries, PISOtorch_simulation.py:210-312): (block, face)
        # pairs of varying Dirichlet faces, the static characteristic velocity [D] and the flux-balance
        # tolerance (default: the solver default of the dtype, whose 1% is the balance threshold)
        self.outflow = [(int(b), int(f)) for b, f in (outflow or [])]
        if self.outflow:
            for b, f in self.outflow:
                bnd = domain.getBlock(b).getBoundary(f)
                if not isinstance(bnd, P.FixedBoundary) or bnd.isVelocityStatic:
                    raise ValueError("outflow face (%d, %d) must be a FixedBoundary with varying velocity" % (b, f))
            vel = [1.0] + [0.0] * (self.dims - 1) if outflow_velocity is None else \
                [float(v) for v in torch.as_tensor(outflow_velocity).reshape(-1).tolist()]
            if len(vel) != self.dims:
                raise ValueError("outflow_velocity must have %d components" % self.dims)
            self._of_faces = (ctypes.c_int32 * (2 * len(self.outflow)))(*[v for bf in self.outflow for v in bf])
            self._of_vel = (ctypes.c_double * self.dims)(*vel)
            self._of_atol = 0.01 * (default_tolerance(dt) if outflow_tol is None else float(outflow_tol))
        self._graph = None
        self._graph_steps = 0
        self._prepare()

    def _prepare(self):
        d = self.domain
        d._check_ready()
        self.desc = d._desc
        lib = _lib.load()
        ns = self.desc.num_sims
        dev = d.getDevice()
        self.info_bytes = _lib.SOLVE_INFO_BYTES
        # per step: adv (ns*D) + corrector_steps pressure solves (ns each)
        self.n_adv_info = ns * self.dims
        self.n_p_info = ns
        nbytes_adv = self.n_adv_info * self.info_bytes
        nbytes_p = self.n_p_info * self.info_bytes
        nr = self.pressure_refine
        self.info = torch.zeros(nbytes_adv + self.corrector_steps * (1 + nr) * nbytes_p, dtype=torch.uint8, device=dev)
        self.info_adv = self.info[:nbytes_adv]
        self.info_p = [self.info[nbytes_adv + k * nbytes_p: nbytes_adv + (k + 1) * nbytes_p]
                       for k in range(self.corrector_steps)]
        base = nbytes_adv + self.corrector_steps * nbytes_p
        self.info_r = [[self.info[base + (k * nr + m) * nbytes_p: base + (k * nr + m + 1) * nbytes_p]
                        for m in range(nr)] for k in range(self.corrector_steps)]
        if nr > 0:
            N = d.getTotalSize()
            self._x64 = torch.zeros(N, dtype=torch.float64, device=dev)
            self._res = torch.zeros(N, dtype=d.getDtype(), device=dev)
            self._corr = torch.zeros(N, dtype=d.getDtype(), device=dev)
            self._tile_scratch = torch.zeros(max(1, self.desc.num_tiles), dtype=torch.float64, device=dev)
            if self.refine_solver in ("mg", "auto"):
                from .multigrid import hierarchy_for, axis_strengths
                try:
                    if self.refine_solver == "auto":
                        # point-smoothed multigrid is robust on near-isotropic grids only
                        st_ = axis_strengths(d)[:, :self.dims]
                        if float((st_.max(axis=1) / np.maximum(st_.min(axis=1), 1e-300)).max()) > 4.0:
                            raise ValueError("strongly anisotropic grid")
                    self._mg = hierarchy_for(d)
                    self._mg_ws = torch.empty(self._mg.workspace_bytes(self.desc), dtype=torch.uint8, device=dev)
                    if self.mg_iterations <= 0:
                        # cap of the PCG iterations (each system stops at the target): a correction takes at
                        # most ~5 with two smoothing sweeps on the finest level, ~9 with one
                        from .multigrid import STAGE_CELLS
                        L0 = self._mg.levels[0]
                        two = int(L0.sweeps) >= 2 and \
                            int(self.desc.tile_cells) + 6 * int(L0.max_block_sx) <= (3 * STAGE_CELLS) // 4
                        self.mg_iterations = 8 if two else 12
                except ValueError as e:
                    if self.refine_solver == "mg":
                        warnings.warn("multigrid refinement not available (%s); using CG" % e)
                    self._mg = None
        ws = max(lib.pict_solve_workspace_bytes(ctypes.byref(self.desc), ctypes.byref(self.adv_params)),
                 lib.pict_solve_workspace_bytes(ctypes.byref(self.desc), ctypes.byref(self.p_params)),
                 lib.pict_solve_workspace_bytes(ctypes.byref(self.desc), ctypes.byref(self.r_params)))
        self.ws = torch.empty(int(ws), dtype=torch.uint8, device=dev)
        self.ws_bytes = int(ws)
        self.lib = lib

    def _dt(self, time_step):
        ts = self.time_step if time_step is None else time_step
        if isinstance(ts, torch.Tensor):
            ts = float(ts.item())
        return float(ts)

    def _pressure_solve(self, k, desc, st):
        """Pressure solve of corrector k (plus FP64 refinement sweeps); leaves the mean-free solution in
        pressureResult and the blocks' pressure."""
        d = self.domain
        lib = self.lib
        if self.pressure_first_solve:
            check(lib.pict_solve(desc, P._ptr(d.P.coef), P._ptr(d.pressureRHSdiv), P._ptr(d.pressureResult),
                                 ctypes.byref(self.p_params), P._ptr(self.info_p[k]), P._ptr(self.ws), self.ws_bytes,
                                 st), "pressure solve")
        if self.pressure_refine > 0:
            self._refine_warm(k, desc, st)

    def _axpby(self, a, x, b, y, out, st):
        d = self.domain
        code = _lib.PICT_F64 if d.getDtype() == torch.float64 else _lib.PICT_F32
        check(self.lib.pict_vector_axpby(d.getTotalSize(), code, float(a), P._ptr(x), float(b), P._ptr(y), P._ptr(out),
                                         st), "pressure warm start")

    def _refine_warm(self, k, desc, st, events=None, ev=None):
        """Refinement of corrector k, started (in "increment" mode) from the extrapolated first-corrector
        pressure (k = 0, once two steps are known) or from corrector k-1's pressure plus the previous step's
        corrector increment (k >= 1)."""
        if not self.pressure_increment or self.pressure_first_solve:
            self._refine_only(k, desc, st, events=events, ev=ev)
            return
        d = self.domain
        n = d.getTotalSize()
        if self._p_delta is None:
            z = lambda *shape: torch.zeros(*shape, dtype=d.getDtype(), device=d.getDevice())
            self._p_delta = z(max(self.corrector_steps - 1, 1), n)
            self._p_prev, self._p_guess, self._p0_hist = z(n), z(n), z(2, n)
        pr = d.pressureResult
        if k == 0:
            x_init = None
            if self._p0_count >= 2:
                self._axpby(2.0, self._p0_hist[0], -1.0, self._p0_hist[1], self._p_guess, st)
                x_init = self._p_guess
            self._refine_only(k, desc, st, events=events, ev=ev, x_init=x_init)
            self._axpby(1.0, self._p0_hist[0], 0.0, self._p0_hist[0], self._p0_hist[1], st)
            self._axpby(1.0, pr, 0.0, pr, self._p0_hist[0], st)
            self._p0_count += 1
        else:
            self._axpby(1.0, pr, 0.0, pr, self._p_prev, st)
            self._axpby(1.0, pr, 1.0, self._p_delta[k - 1], self._p_guess, st)
            self._refine_only(k, desc, st, events=events, ev=ev, x_init=self._p_guess)
            self._axpby(1.0, pr, -1.0, self._p_prev, self._p_delta[k - 1], st)

    def step(self, time_step=None, stream=None):
        """Launch one PISO step (no host synchronisation)."""
        d = self.domain
        lib = self.lib
        desc = ctypes.byref(self.desc)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
        dt = self._dt(time_step)
        D = self.dims
        self._outflow(desc, dt, st)
        check(lib.pict_setup_advection(desc, dt, st), "advection setup")
        self._advection_guess(desc, st)
        check(lib.pict_solve(desc, P._ptr(d.C.coef), P._ptr(d.velocityRHS), P._ptr(d.velocityResult),
                             ctypes.byref(self.adv_params), P._ptr(self.info_adv), P._ptr(self.ws), self.ws_bytes, st),
              "advection solve")
        self._advection_increment(desc, st)
        for k in range(self.corrector_steps):
            if k == 0:
                check(lib.pict_setup_pressure_correction(desc, dt, 0, 0, st), "pressure setup")
            else:
                check(lib.pict_setup_pressure_rhs(desc, dt, 0, 0, st), "pressure rhs")
            self._pressure_solve(k, desc, st)
            last = k == self.corrector_steps - 1
            check(lib.pict_correct_velocity(desc, dt, 1, 0, 1 if last else 0, st), "velocity correction")
        if self.corrector_steps == 0:
            check(lib.pict_copy_velocity_result_to_blocks(desc, st), "copy velocity")

    def _advection_guess(self, desc, st):
        """Advection initial guess: the blocks' velocity plus the extrapolated advection increment
        2 d_n - d_{n-1} (d_n - d_{n-1} ... the first steps: d_n, or none), or the blocks' velocity."""
        if self.advection_increment:
            d = self.domain
            n = self.dims * d.getTotalSize()
            if self._adv_incr is None:
                self._adv_incr = torch.zeros(3, n, dtype=d.getDtype(), device=d.getDevice())  # d_n, d_{n-1}, guess
                self._adv_count = 0
            inc = self._adv_incr
            code = _lib.PICT_F64 if d.getDtype() == torch.float64 else _lib.PICT_F32
            if self._adv_count >= 2:
                check(self.lib.pict_vector_axpby(n, code, 2.0, P._ptr(inc[0]), -1.0, P._ptr(inc[1]), P._ptr(inc[2]),
                                                 st), "advection increment extrapolation")
                g = inc[2]
            else:
                g = inc[0]
            check(self.lib.pict_advection_guess(desc, P._ptr(g), 0, st), "advection initial guess")
        elif self.warm_start_advection:
            check(self.lib.pict_copy_velocity_result_from_blocks(desc, st), "advection initial guess")

    def _advection_increment(self, desc, st):
        if self.advection_increment:
            d = self.domain
            n = self.dims * d.getTotalSize()
            inc = self._adv_incr
            code = _lib.PICT_F64 if d.getDtype() == torch.float64 else _lib.PICT_F32
            check(self.lib.pict_vector_axpby(n, code, 1.0, P._ptr(inc[0]), 0.0, P._ptr(inc[0]), P._ptr(inc[1]), st),
                  "advection increment history")
            check(self.lib.pict_advection_guess(desc, P._ptr(inc[0]), 1, st), "advection increment")
            self._adv_count += 1

    def _outflow(self, desc, dt, st):
        if self.outflow:
            check(self.lib.pict_advective_outflow(desc, self._of_faces, len(self.outflow), self._of_vel, dt,
                                                  self._of_atol, st), "advective outflow")

    def _refine_only(self, k, desc, st, events=None, ev=None, x_init=None):
        """FP64 refinement sweeps after the first pressure solve of corrector k: residual of the FP64
        accumulator, FP32 correction solve, accumulation; then the mean-free result into
        pressureResult and the blocks' pressure."""
        d = self.domain
        lib = self.lib
        x64 = ctypes.c_void_p(self._x64.data_ptr())
        for m in range(self.pressure_refine):
            start = (d.pressureResult if x_init is None else x_init) if m == 0 else None
            check(lib.pict_refine_residual(desc, P._ptr(d.P.coef), P._ptr(d.pressureRHSdiv),
                                           P._ptr(start), x64, P._ptr(self._res),
                                           int(self.normalize_pressure), ctypes.c_void_p(self._tile_scratch.data_ptr()),
                                           st), "refine residual")
            a = ev() if ev else None
            if self._mg is not None:
                if k == 0 and m == 0:  # the pressure matrix is assembled once per step
                    self._mg.setup(d.P.coef, st)
                self._mg.solve(self.desc, self._res, self._corr, self.mg_iterations, self.refine_tol, self.info_r[k][m],
                               self._mg_ws, st)
            else:
                check(lib.pict_solve(desc, P._ptr(d.P.coef), P._ptr(self._res), P._ptr(self._corr),
                                     ctypes.byref(self.r_params), P._ptr(self.info_r[k][m]), P._ptr(self.ws),
                                     self.ws_bytes, st), "refinement solve")
            if events is not None:
                events.append((a, ev(), self.info_r[k][m].clone()))
            check(lib.pict_refine_update(desc, x64, P._ptr(self._corr), st), "refine update")
        check(lib.pict_refine_finish(desc, x64, P._ptr(d.pressureResult), int(self.normalize_pressure), 1,
                                     ctypes.c_void_p(self._tile_scratch.data_ptr()), st), "refine finish")

    def kernels_per_step(self):
        """Kernels of this library launched per step: advection setup 1; per solve init-info, solver and
        finish-info 3; per corrector pressure setup 2 (matrix/RHS, divergence), correction 1, and the
        refinement sweeps when enabled; the copy of the initial guess of a warm-started advection solve 1;
        the advective outflow update 1."""
        n = 1 + 3 + (1 if self.warm_start_advection else 0) + (3 if self.advection_increment else 0) + \
            (1 if self.outflow else 0)
        n += self.corrector_steps * (2 + (3 if self.pressure_first_solve else 0) + 1)
        if self.pressure_refine > 0:  # per sweep: residual (+2 projection), solve, update; partials + finish
            if self._mg is not None:
                nl, it = self._mg.num_levels, self.mg_iterations
                v = self._mg.launches_per_vcycle()   # with the PCG update / dot partials fused in
                if nl == 1:  # separate update, sub-cycle, dot
                    solve = (v - 1) + 1 + it * 3 + max(it - 1, 0) * v + (1 if it > 0 else 0) + 1
                else:
                    solve = v + 1 + it * 3 + max(it - 1, 0) * v + (1 if it > 0 else 0) + 1
                n += nl - 1  # Galerkin coarse operators once per step
            else:
                solve = 3
            per = 2 + solve + (2 if self.normalize_pressure else 0)
            n += self.corrector_steps * (per * self.pressure_refine + (2 if self.normalize_pressure else 1))
        if self.corrector_steps == 0:
            n += 1
        return n

    def step_with_events(self, time_step=None):
        """Eager step with CUDA events around each Krylov launch (timing of the dominant kernels).

        Returns {"bicg": [(start, end, info)], "cg": [...], "mg": [...]} (persistent BiCGStab, persistent CG
        and multigrid-preconditioned CG solves) with copies of the solver reports of each launch.
        """
        d = self.domain
        lib = self.lib
        desc = ctypes.byref(self.desc)
        cs = torch.cuda.current_stream()
        st = ctypes.c_void_p(cs.cuda_stream)
        dt = self._dt(time_step)
        out = {"bicg": [], "cg": [], "mg": []}
        self._outflow(desc, dt, st)

        def ev():
            e = torch.cuda.Event(enable_timing=True)
            e.record(cs)
            return e

        check(lib.pict_setup_advection(desc, dt, st), "advection setup")
        self._advection_guess(desc, st)
        a = ev()
        check(lib.pict_solve(desc, P._ptr(d.C.coef), P._ptr(d.velocityRHS), P._ptr(d.velocityResult),
                             ctypes.byref(self.adv_params), P._ptr(self.info_adv), P._ptr(self.ws), self.ws_bytes, st),
              "advection solve")
        b = ev()
        self._advection_increment(desc, st)
        out["bicg"].append((a, b, self.info_adv.clone()))
        for k in range(self.corrector_steps):
            if k == 0:
                check(lib.pict_setup_pressure_correction(desc, dt, 0, 0, st), "pressure setup")
            else:
                check(lib.pict_setup_pressure_rhs(desc, dt, 0, 0, st), "pressure rhs")
            if self.pressure_first_solve:
                a = ev()
                check(lib.pict_solve(desc, P._ptr(d.P.coef), P._ptr(d.pressureRHSdiv), P._ptr(d.pressureResult),
                                     ctypes.byref(self.p_params), P._ptr(self.info_p[k]), P._ptr(self.ws),
                                     self.ws_bytes, st), "pressure solve")
                b = ev()
                out["cg"].append((a, b, self.info_p[k].clone()))
            if self.pressure_refine > 0:
                self._refine_warm(k, desc, st, events=out["mg" if self._mg is not None else "cg"], ev=ev)
            last = k == self.corrector_steps - 1
            check(lib.pict_correct_velocity(desc, dt, 1, 0, 1 if last else 0, st), "velocity correction")
        return out

    def infos(self):
        """Decode the solver reports of the last step: (advection [ns*D], [pressure [ns]] per corrector)."""
        all_infos = P.decode_infos(self.info)
        adv = all_infos[:self.n_adv_info]
        ps = [all_infos[self.n_adv_info + k * self.n_p_info: self.n_adv_info + (k + 1) * self.n_p_info]
              for k in range(self.corrector_steps)]
        return adv, ps

    def refine_infos(self):
        """Reports of the refinement solves of the last step: [corrector][sweep] -> [ns]."""
        return [[P.decode_infos(t) for t in row] for row in self.info_r]

    def check(self):
        """Raise LinsolveError if any solve of the last step failed (synchronises)."""
        adv, ps = self.infos()
        extra = [("pressure %d refinement %d" % (k, m), r) for k, row in enumerate(self.refine_infos())
                 for m, r in enumerate(row)]
        first = [("pressure %d" % k, p) for k, p in enumerate(ps)] if self.pressure_first_solve else []
        for name, lst in [("advection", adv)] + first + extra:
            for i, inf in enumerate(lst):
                if getattr(inf, "status", 0) == 1:
                    raise LinsolveError("%s solve: inter-CTA barrier timed out (system %d)" % (name, i))
                if not inf.isFiniteResidual:
                    raise LinsolveError("%s solve reported non-finite residual for RHS %d: %s" % (name, i, inf))
                if not inf.converged:
                    raise LinsolveError("%s solve RHS %d did not converge: %s" % (name, i, inf))
        return adv, ps

    # ---------------- CUDA graph ----------------
    def capture(self, steps: int = 1, time_step=None):
        """Capture `steps` PISO steps into a CUDA graph (replay with :meth:`replay`).

        One eager step runs first (module loading, allocator warm-up); the blocks' velocity and
        pressure are restored afterwards, so capturing does not advance the simulation.
        """
        d = self.domain
        saved = [(b.velocity.clone(), b.pressure.clone()) for b in d.getBlocks()]
        saved_out = [d.getBlock(b).getBoundary(f).velocity.clone() for b, f in self.outflow]
        saved_incr = None if self._adv_incr is None else (self._adv_incr.clone(), self._adv_count)
        saved_pd = None if self._p_delta is None else (self._p_delta.clone(), self._p0_hist.clone(), self._p0_count)
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.step(time_step)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        for b, (v, p) in zip(d.getBlocks(), saved):
            b.velocity.copy_(v)
            b.pressure.copy_(p)
        for (b, f), v in zip(self.outflow, saved_out):
            d.getBlock(b).getBoundary(f).velocity.copy_(v)
        if self._adv_incr is not None:
            if saved_incr is None:
                self._adv_incr.zero_()
                self._adv_count = 0
            else:
                self._adv_incr.copy_(saved_incr[0])
                self._adv_count = saved_incr[1]
        if self._p_delta is not None:
            if saved_pd is None:
                self._p_delta.zero_()
                self._p0_hist.zero_()
                self._p0_count = 0
            else:
                self._p_delta.copy_(saved_pd[0])
                self._p0_hist.copy_(saved_pd[1])
                self._p0_count = saved_pd[2]
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for _ in range(steps):
                self.step(time_step)
        self._graph = g
        self._graph_steps = steps
        return g

    def replay(self):
        self._graph.replay()
