"""Reverse mode of the fused PISO step: taped forward steps, the adjoint step, and a checkpointed
rollout behind ``torch.autograd.Function``.

The reference differentiates a step operator by operator through ``PISOtorch_diff`` (autograd
Functions around every Setup*/SolveLinear/CorrectVelocity call, PISOtorch_diff.py:295-1236).  Here
one forward step records a small tape of global vectors and the reverse step runs the adjoint
operators of ``libpict_b200`` (adjoint.cu) plus two transposed Krylov solves:

    per corrector k = K-1 .. 0:
        CorrectVelocity^T      -> h_bar, A_bar, p_bar
        mean removal^T         -> p_bar - mean(p_bar)
        CG on P^T lambda = p_bar (P is symmetric: multigrid-preconditioned on the stepper's hierarchy,
            from the previous adjoint step's lambda with one FP64 refinement sweep)
        divergence^T, H/A^T, P(A)^T (with -lambda x^T)  -> A_bar, C_bar, U_bar, parameter gradients
    BiCGStab on C^T rhs_bar = u*_bar (all components in one launch)
    advection^T (with -rhs_bar u*^T)   -> gradient of the step's input velocity and parameters

Gradients with respect to the simulation parameters accumulate over all steps: per-cell viscosity
(reduced to the system / block viscosity), velocity source, boundary velocity of fixed faces.

``rollout()`` keeps only every ``checkpoint_every``-th velocity during the forward pass, tapes the last
window as it runs and, in the backward pass, reverses that window directly and recomputes each earlier
window from its checkpoint with taping before reversing it.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence

import torch

from . import _lib
from ._lib import check
from . import PISOtorch as P
from .engine import PISOStepper, LinsolveError

FIELD_VELOCITY, FIELD_PRESSURE, FIELD_SOURCE, FIELD_VELOCITY_GRAD, FIELD_PRESSURE_GRAD, FIELD_SOURCE_GRAD = range(6)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class StepTape:
    """Forward quantities of one PISO step needed by its adjoint (global layouts)."""

    def __init__(self, N, D, K, correctors, dtype, device):
        z = lambda *s: torch.empty(*s, dtype=dtype, device=device)
        self.un = z(D * N)         # velocity at the start of the step
        self.C = z(K * N)          # advection matrix (stencil)
        self.A = z(N)              # its diagonal
        self.ustar = z(D * N)      # advection solve result
        self.h = [z(D * N) for _ in range(correctors)]   # H/A per corrector
        self.p = [z(N) for _ in range(correctors)]       # pressure solution per corrector
        self.U = [None] + [z(D * N) for _ in range(correctors - 1)]  # velocity used in H/A (k >= 1)


class PISOAdjoint:
    """Taped forward steps and adjoint steps of a :class:`PISOStepper` (same domain and settings).

    ``adjoint_advection_tol`` / ``adjoint_pressure_tol`` default to the forward tolerances.  With
    ``use_graph = True`` the untaped forward steps of :func:`rollout` replay the stepper's captured
    one-step CUDA graph, and its backward pass replays CUDA graphs of the taped step into each slot of
    the checkpoint window and of the adjoint step from it, captured on first use (like the stepper's
    graph they hold the time step and the tolerances of their capture).  ``adjoint_pressure_solver``:
    the transposed pressure solves run as multigrid-preconditioned CG on the stepper's hierarchy where it
    has one ("auto", the default, or "mg"), or as the persistent CG ("cg").
    """

    def __init__(self, stepper: PISOStepper, adjoint_advection_tol: Optional[float] = None,
                 adjoint_pressure_tol: Optional[float] = None, relative_tolerance: bool = False,
                 adjoint_pressure_solver: str = "auto", adjoint_mg_iterations: int = 24):
        self.st = stepper
        # relative_tolerance: every transposed solve first scales its right-hand side to unit RMS per
        # system (on the device) and scales the solution back, so that the (absolute, RMS) tolerance acts
        # relative to the adjoint's own magnitude; without it the adjoint solves stop at the absolute
        # tolerance, as the reference's backward solves do (PISOtorch_diff.py:331-372), which for a
        # small loss gradient is a loose relative tolerance
        self.relative = bool(relative_tolerance)
        d = stepper.domain
        P._check(stepper.normalize_pressure, "the adjoint needs normalize_pressure=True (mean-free pressure)")
        self.dom = d
        self.lib = stepper.lib
        self.D = stepper.dims
        self.K = 2 * self.D + 1
        self.N = d.getTotalSize()
        self.dtype = d.getDtype()
        self.dev = d.getDevice()
        self.ns = stepper.desc.num_sims
        self.nc = stepper.corrector_steps
        P._check(self.nc >= 1, "the adjoint needs at least one corrector")
        atol = stepper.adv_tol if adjoint_advection_tol is None else float(adjoint_advection_tol)
        ptol = stepper.p_tol if adjoint_pressure_tol is None else float(adjoint_pressure_tol)
        ap, pp = stepper.adv_params, stepper.p_params
        self.adv_params = P._solve_params(self.D, stepper.max_iterations, atol, _lib.PICT_CONV_NORM2_NORMALIZED, True,
                                          True, x_zero=False, group_size=ap.group_size)
        self.p_params = P._solve_params(1, stepper.max_iterations, ptol, _lib.PICT_CONV_NORM2_NORMALIZED, False, True,
                                        x_zero=True, group_size=pp.group_size, variant=pp.variant)
        # adjoint pressure solves: the pressure matrix is symmetric, so the transposed solve is the forward
        # operator and the stepper's multigrid hierarchy preconditions it ("auto": where the stepper has one,
        # "mg": required, "cg": the persistent CG); each system stops at the same RMS criterion, within
        # adjoint_mg_iterations iterations (under graph capture only the iterations still needed run)
        P._check(adjoint_pressure_solver in ("auto", "mg", "cg"), "adjoint_pressure_solver: auto, mg or cg")
        P._check(adjoint_pressure_solver != "mg" or stepper._mg is not None,
                 "adjoint_pressure_solver='mg' needs a stepper with a multigrid hierarchy (refine_solver='auto'/'mg')")
        self.p_mg = stepper._mg is not None and adjoint_pressure_solver != "cg"
        self.p_tol = ptol
        self.p_mg_iterations = int(adjoint_mg_iterations)
        N, D, K = self.N, self.D, self.K
        z = lambda n: torch.zeros(n, dtype=self.dtype, device=self.dev)
        # per-step work
        self.Abar, self.Cbar, self.hbar, self.pbar, self.lam = z(N), z(K * N), z(D * N), z(N), z(N)
        self.Ubar, self.rhsbar, self.unbar = z(D * N), z(D * N), z(D * N)
        self.Pwork = z(K * N)
        # parameter accumulators (whole rollout)
        self.nubar = z(N)
        self.srcbar = z(D * N)
        self.vbbar = z(2 * D * D * N)
        self.info = torch.zeros((D + 1) * self.ns * _lib.SOLVE_INFO_BYTES, dtype=torch.uint8, device=self.dev)
        self.block_scratch = torch.zeros(max(1, len(d.getBlocks())), dtype=torch.float64, device=self.dev)
        self.sim_nu_bar = z(self.ns)
        # warm starts of the transposed solves: the solutions of the previous adjoint step (the next time
        # step), which the adjoint variables follow smoothly; zero at the start of every backward pass
        self._rhs_prev = z(D * N)
        self._lam_prev = [z(N) for _ in range(self.nc)]
        if self.p_mg:
            # the multigrid pressure solve from the warm start: one FP64 refinement sweep (FP64 residual,
            # FP32 correction solve, FP64 accumulation), so the residual can fall below the FP32 level
            self._lam64 = torch.zeros(N, dtype=torch.float64, device=self.dev)
            self._pres, self._pcorr = z(N), z(N)
            self._tile_scratch = torch.zeros(max(1, int(stepper.desc.num_tiles)), dtype=torch.float64, device=self.dev)
        sc = d._sim_cells.long().to(self.dev)
        self._sim_start, self._sim_end = sc[:-1], sc[1:]
        self._sim_n = (sc[1:] - sc[:-1]).double()
        self._cell_sim = torch.repeat_interleave(torch.arange(self.ns, device=self.dev), sc[1:] - sc[:-1])

    # ------------------------------------------------------------------ state helpers
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _desc(self, A=None, C=None, Pm=None):
        """A copy of the stepper's descriptor with matrix pointers replaced."""
        src = self.st.domain._desc
        dsc = _lib.DomainDesc()
        ctypes.memmove(ctypes.byref(dsc), ctypes.byref(src), ctypes.sizeof(dsc))
        if A is not None:
            dsc.A = A.data_ptr()
        if C is not None:
            dsc.C = C.data_ptr()
        if Pm is not None:
            dsc.P = Pm.data_ptr()
        return dsc

    def velocity(self, out=None):
        """The blocks' velocity as a global [D*N] vector."""
        out = torch.empty(self.D * self.N, dtype=self.dtype, device=self.dev) if out is None else out
        check(self.lib.pict_copy_field(ctypes.byref(self.st.domain._desc), FIELD_VELOCITY, 0, _p(out), 0,
                                       self._stream()), "copy velocity")
        return out

    def set_velocity(self, u):
        u = u.contiguous()
        check(self.lib.pict_copy_field(ctypes.byref(self.st.domain._desc), FIELD_VELOCITY, 1, _p(u), 0,
                                       self._stream()), "set velocity")

    def pressure(self, out=None):
        """The blocks' pressure as a global [N] vector."""
        out = torch.empty(self.N, dtype=self.dtype, device=self.dev) if out is None else out
        check(self.lib.pict_copy_field(ctypes.byref(self.st.domain._desc), FIELD_PRESSURE, 0, _p(out), 0,
                                       self._stream()), "copy pressure")
        return out

    def set_pressure(self, p):
        p = p.contiguous()
        check(self.lib.pict_copy_field(ctypes.byref(self.st.domain._desc), FIELD_PRESSURE, 1, _p(p), 0,
                                       self._stream()), "set pressure")

    def set_source(self, src):
        src = src.contiguous()
        check(self.lib.pict_copy_field(ctypes.byref(self.st.domain._desc), FIELD_SOURCE, 1, _p(src), 0,
                                       self._stream()), "set source")

    def reset_warm_starts(self):
        """Start the transposed solves of the next adjoint step from zero (the first step of a backward pass)."""
        self._rhs_prev.zero_()
        for v in self._lam_prev:
            v.zero_()

    def zero_parameter_grads(self):
        self.nubar.zero_()
        self.srcbar.zero_()
        self.vbbar.zero_()

    # ------------------------------------------------------------------ forward with tape
    def new_tape(self):
        return StepTape(self.N, self.D, self.K, self.nc, self.dtype, self.dev)

    def tapes(self, n):
        """The adjoint's own tapes for a checkpoint window of n steps (kept, so that the graphs captured
        for a window slot keep their buffers)."""
        pool = self.__dict__.setdefault("_tape_pool", [])
        while len(pool) < n:
            pool.append(self.new_tape())
        return pool[:n]

    # ------------------------------------------------------------------ graphed steps of the backward pass
    def _capture(self, fn):
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            out = fn()
        return g, out

    def step_taped_graphed(self, slot: int, tape: StepTape):
        """step_taped(tape) as a CUDA graph replay (captured on the first call for this slot).  Capturing
        launches nothing, so the first call captures and then replays."""
        graphs = self.__dict__.setdefault("_taped_graphs", {})
        if slot not in graphs or graphs[slot][1] is not tape:
            graphs[slot] = (self._capture(lambda: self.step_taped(tape))[0], tape)
        graphs[slot][0].replay()

    def backward_step_graphed(self, slot: int, tape: StepTape, ubar):
        """backward_step(tape, ubar) as a CUDA graph replay with a fixed input buffer per slot; returns
        dL/du^n in the graph's output buffer (valid until the next replay of this slot)."""
        graphs = self.__dict__.setdefault("_back_graphs", {})
        if slot not in graphs or graphs[slot][2] is not tape:
            ub = torch.empty(self.D * self.N, dtype=self.dtype, device=self.dev)
            ub.copy_(ubar)
            g, out = self._capture(lambda: self.backward_step(tape, ub))
            graphs[slot] = (g, ub, tape, out)
        g, ub, _, out = graphs[slot]
        ub.copy_(ubar)
        g.replay()
        return out

    def step_taped(self, tape: StepTape, time_step=None):
        st = self.st
        d = st.domain
        lib = self.lib
        desc = ctypes.byref(d._desc)
        s = self._stream()
        dt = st._dt(time_step)
        self.velocity(tape.un)
        check(lib.pict_setup_advection(desc, dt, s), "advection setup")
        tape.C.copy_(d.C.coef.reshape(-1))
        tape.A.copy_(d.A)
        st._advection_guess(desc, s)  # the stepper's initial guess (its solves converge to the same tolerance)
        check(lib.pict_solve(desc, P._ptr(d.C.coef), P._ptr(d.velocityRHS), P._ptr(d.velocityResult),
                             ctypes.byref(st.adv_params), P._ptr(st.info_adv), P._ptr(st.ws), st.ws_bytes, s),
              "advection solve")
        st._advection_increment(desc, s)
        tape.ustar.copy_(d.velocityResult)
        for k in range(self.nc):
            if k > 0:
                tape.U[k].copy_(d.velocityResult)
            if k == 0:
                check(lib.pict_setup_pressure_correction(desc, dt, 0, 0, s), "pressure setup")
            else:
                check(lib.pict_setup_pressure_rhs(desc, dt, 0, 0, s), "pressure rhs")
            tape.h[k].copy_(d.pressureRHS)
            st._pressure_solve(k, desc, s)
            tape.p[k].copy_(d.pressureResult)
            last = k == self.nc - 1
            check(lib.pict_correct_velocity(desc, dt, 1, 0, 1 if last else 0, s), "velocity correction")

    # ------------------------------------------------------------------ adjoint step
    def backward_step(self, tape: StepTape, ubar, pbar_out=None, time_step=None):
        """Reverse one step: ubar = dL/du^{n+1} [D*N] (and dL/dp^{n+1} [N]); returns dL/du^n [D*N].
        Parameter gradients accumulate into nubar / srcbar / vbbar."""
        st = self.st
        lib = self.lib
        s = self._stream()
        dt = st._dt(time_step)
        dsc = self._desc(A=tape.A, C=tape.C, Pm=self.Pwork)
        desc = ctypes.byref(dsc)
        self.Abar.zero_()
        self.Cbar.zero_()
        self.unbar.zero_()
        check(lib.pict_setup_pressure_matrix(desc, 0, s), "adjoint pressure matrix")
        if self.p_mg:
            st._mg.setup(self.Pwork, s)  # coarse operators of this step's pressure matrix
        ucur = ubar.contiguous()
        info_p = self.info[self.D * self.ns * _lib.SOLVE_INFO_BYTES:]
        info_a = self.info[:self.D * self.ns * _lib.SOLVE_INFO_BYTES]
        src = _p(self.srcbar)
        for k in reversed(range(self.nc)):
            check(lib.pict_correct_velocity_grad(desc, _p(tape.A), _p(tape.p[k]), _p(ucur), _p(self.Abar),
                                                 _p(self.pbar), _p(self.hbar), s), "correct velocity grad")
            if k == self.nc - 1 and pbar_out is not None:
                self.pbar.add_(pbar_out)
            check(lib.pict_sim_mean_project(desc, _p(self.pbar), s), "mean projection")
            if self.relative:
                scale = self._rms_scale(self.pbar, 1)
                self.pbar.div_(scale)
            if self.p_mg:
                guess = self._lam_prev[k] / scale if self.relative else self._lam_prev[k]
                x64 = ctypes.c_void_p(self._lam64.data_ptr())
                scratch = ctypes.c_void_p(self._tile_scratch.data_ptr())
                check(lib.pict_refine_residual(desc, _p(self.Pwork), _p(self.pbar), _p(guess), x64, _p(self._pres), 1,
                                               scratch, s), "adjoint pressure residual")
                st._mg.solve(dsc, self._pres, self._pcorr, self.p_mg_iterations, self.p_tol, info_p, st._mg_ws, s)
                check(lib.pict_refine_update(desc, x64, _p(self._pcorr), s), "adjoint pressure update")
                check(lib.pict_refine_finish(desc, x64, _p(self.lam), 1, 0, scratch, s), "adjoint pressure finish")
            else:
                self.lam.zero_()
                check(lib.pict_solve(desc, _p(self.Pwork), _p(self.pbar), _p(self.lam), ctypes.byref(self.p_params),
                                     _p(info_p), P._ptr(st.ws), st.ws_bytes, s), "adjoint pressure solve")
            if self.relative:
                self.lam.mul_(scale)
            if self.p_mg:
                self._lam_prev[k].copy_(self.lam)
            self._check_info(info_p, "adjoint pressure")
            check(lib.pict_divergence_grad(desc, _p(self.lam), _p(self.hbar), _p(self.vbbar), s), "divergence grad")
            U = tape.ustar if k == 0 else tape.U[k]
            check(lib.pict_pressure_rhs_grad(desc, dt, _p(self.hbar), _p(tape.h[k]), _p(tape.A), _p(tape.C), _p(U),
                                             _p(self.lam), _p(tape.p[k]), _p(self.Abar), _p(self.Cbar),
                                             _p(self.Ubar), _p(self.unbar), src, _p(self.nubar), _p(self.vbbar), s),
                  "pressure rhs grad")
            ucur = self.Ubar.clone() if k > 0 else self.Ubar
        # advection solve (transposed, all components) and assembly
        if self.relative:
            scale = self._rms_scale(self.Ubar, self.D)
            self.Ubar.div_(scale)
            torch.div(self._rhs_prev, scale, out=self.rhsbar)
        else:
            self.rhsbar.copy_(self._rhs_prev)
        check(lib.pict_solve(desc, _p(tape.C), _p(self.Ubar), _p(self.rhsbar), ctypes.byref(self.adv_params),
                             _p(info_a), P._ptr(st.ws), st.ws_bytes, s), "adjoint advection solve")
        if self.relative:
            self.rhsbar.mul_(scale)
        self._rhs_prev.copy_(self.rhsbar)
        self._check_info(info_a, "adjoint advection")
        check(lib.pict_advection_grad(desc, dt, _p(tape.ustar), _p(self.rhsbar), _p(self.Cbar), _p(self.Abar),
                                      _p(self.unbar), _p(self.nubar), _p(self.vbbar), src, s), "advection grad")
        return self.unbar.clone()

    def _rms_scale(self, v, ncomp):
        """Per-system RMS of v [ncomp*N] spread to every entry [ncomp*N] (FP64 sums, no host sync; the
        cumulative sum keeps the per-system sums in a fixed order)."""
        sq = (v.double().reshape(ncomp, self.N) ** 2).sum(0)
        c = torch.cat([sq.new_zeros(1), torch.cumsum(sq, 0)])
        rms = torch.sqrt((c[self._sim_end] - c[self._sim_start]) / (self._sim_n * ncomp))
        rms = rms.clamp_min(float(torch.finfo(self.dtype).tiny) * 1e6).to(self.dtype)
        return rms[self._cell_sim].repeat(ncomp)

    def _check_info(self, info, what):
        if not getattr(self, "check_solves", False):
            return
        for i, inf in enumerate(P.decode_infos(info)):
            if getattr(inf, "status", 0) == 1 or not inf.isFiniteResidual or not inf.converged:
                raise LinsolveError("%s solve %d failed: %s" % (what, i, inf))

    def parameter_grads_to_blocks(self):
        """Add the accumulated parameter gradients to the blocks' / boundaries' gradient tensors (those
        that are set) and return the gradient of the system viscosities [num_sims]."""
        self.sim_nu_bar.zero_()
        check(self.lib.pict_adjoint_to_blocks(ctypes.byref(self.st.domain._desc), None, _p(self.nubar), _p(self.srcbar),
                                              _p(self.vbbar), _p(self.sim_nu_bar), _p(self.block_scratch),
                                              self._stream()), "adjoint to blocks")
        return self.sim_nu_bar


# ---------------------------------------------------------------------------------------------
# checkpointed rollout
# ---------------------------------------------------------------------------------------------

class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, adj, steps, record, checkpoint_every, u0, nu, src):
        st = adj.st
        dom = st.domain
        if nu is not None:
            dom._sim_visc.copy_(nu.detach())
        if src is not None:
            adj.set_source(src.detach())
        adj.set_velocity(u0.detach())
        ckpt = {0: u0.detach().clone()}
        outs = []
        rec = sorted(set(int(r) for r in record))
        use_graph = getattr(adj, "use_graph", False) and st._graph is not None
        one_step = st.replay if (use_graph and st._graph_steps == 1) else st.step
        # the last checkpoint window is taped as it runs, so the backward pass reverses it without
        # recomputing it (the taped step is the stepper's step plus the tape copies; domains with an
        # advective outflow update, which the taped step leaves out, keep the recomputation)
        w_last = ((steps - 1) // checkpoint_every) * checkpoint_every
        tape_last = not st.outflow
        graphed = use_graph and not getattr(adj, "check_solves", False)
        tapes = adj.tapes(steps - w_last) if tape_last else None
        for t in range(1, steps + 1):
            if tape_last and t - 1 >= w_last:
                slot = t - 1 - w_last
                if graphed:
                    adj.step_taped_graphed(slot, tapes[slot])
                else:
                    adj.step_taped(tapes[slot])
            else:
                one_step()
            if t % checkpoint_every == 0 and t < steps:
                ckpt[t] = adj.velocity()
            if t in rec:
                outs.append(adj.velocity())
        if getattr(adj, "check_solves", False):
            st.check()
        ctx.final = (adj.velocity(), adj.pressure())
        ctx.adj = adj
        ctx.steps = steps
        ctx.rec = rec
        ctx.K = checkpoint_every
        ctx.ckpt = ckpt
        ctx.has_nu = nu is not None
        ctx.has_src = src is not None
        # the tapes hold this pass's last window until another pass (or a recomputation) reuses them
        ctx.tape_token = object() if tape_last else None
        adj._tape_owner = ctx.tape_token
        return tuple(outs)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, *grads):
        adj = ctx.adj
        steps, K, rec = ctx.steps, ctx.K, ctx.rec
        gmap = {t: g for t, g in zip(rec, grads)}
        adj.zero_parameter_grads()
        adj.reset_warm_starts()
        ubar = torch.zeros(adj.D * adj.N, dtype=adj.dtype, device=adj.dev)
        tapes = adj.tapes(min(K, steps))
        # graphed: the taped and adjoint steps replay per-slot CUDA graphs (the solves' reports are then
        # not read back between steps, so check_solves keeps the eager path)
        graphed = (getattr(adj, "use_graph", False) and adj.st._graph is not None
                   and not getattr(adj, "check_solves", False))
        starts = list(range(0, steps, K))
        for w0 in reversed(starts):
            w1 = min(w0 + K, steps)
            taped = (w0 == starts[-1] and ctx.tape_token is not None
                     and getattr(adj, "_tape_owner", None) is ctx.tape_token)
            adj._tape_owner = None
            if not taped:
                adj.set_velocity(ctx.ckpt[w0])
                for t in range(w0, w1):
                    if graphed:
                        adj.step_taped_graphed(t - w0, tapes[t - w0])
                    else:
                        adj.step_taped(tapes[t - w0])
            for t in reversed(range(w0, w1)):
                g = gmap.get(t + 1)
                if g is not None:
                    ubar = ubar + g.reshape(-1)
                if graphed:
                    ubar = adj.backward_step_graphed(t - w0, tapes[t - w0], ubar)
                else:
                    ubar = adj.backward_step(tapes[t - w0], ubar)
        if graphed:
            ubar = ubar.clone()  # the last replay's output buffer is reused by the next backward pass
        # the recomputation moved the domain state; restore the end of the forward pass
        adj.set_velocity(ctx.final[0])
        adj.set_pressure(ctx.final[1])
        nu_sim = adj.parameter_grads_to_blocks()
        nu_bar = nu_sim.clone() if ctx.has_nu else None
        src_bar = adj.srcbar.clone() if ctx.has_src else None
        return None, None, None, None, ubar, nu_bar, src_bar


def rollout(adj: PISOAdjoint, u0, steps: int, record: Sequence[int], checkpoint_every: int = 10, nu=None, src=None):
    """Run `steps` PISO steps from the global velocity u0 [D*N] and return the velocities after the
    steps listed in `record` (tuple of [D*N] tensors), differentiable with respect to u0, the system
    viscosities nu [num_sims] (descriptor order) and a per-cell velocity source src [D*N].
    The forward keeps every `checkpoint_every`-th velocity and tapes the last window; the backward
    recomputes each earlier window.
    The backward also adds the parameter gradients to the gradient tensors that are allocated on the
    domain (block viscosityGrad / velocitySourceGrad, boundary velocityGrad), and leaves the domain in
    the state at the end of the forward pass."""
    P._check(steps >= 1 and checkpoint_every >= 1, "steps and checkpoint_every must be >= 1")
    P._check(all(1 <= int(r) <= steps for r in record) and len(record) > 0, "record steps must be in [1, steps]")
    return _Rollout.apply(adj, int(steps), tuple(record), int(checkpoint_every), u0, nu, src)
