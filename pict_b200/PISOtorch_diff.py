"""Differentiable operators of the PISO step: drop-in for the reference's ``PISOtorch_diff`` module.

Same function names, arguments and behaviour as PISOtorch_diff.py: every operator is a
``torch.autograd.Function`` whose forward runs the ``libpict_b200`` kernel on freshly created output
tensors of the domain (so every step owns its tensors in the autograd graph) and whose backward
restores the forward tensors on the domain and runs the hand-written adjoint kernels (adjoint.cu).
Tracked inputs, as in the reference (flatten_domain, PISOtorch_diff.py:44-118): block velocity,
pressure, velocity source and viscosity, boundary velocity of fixed faces, domain viscosity and the
domain vectors A, C, P, velocityResult, pressureRHS, pressureResult.

Matrices are the stencil coefficient tensors ``C.coef`` / ``P.coef`` (the reference tracks the CSR
``value`` arrays); ``linear_solve_GPU`` differentiates with respect to them with the transposed
solve and the stencil outer product -b_grad x^T (PISOtorch_diff.py:295-375).

Passive scalars (matrix per channel, scalar RHS, result copies) and the non-orthogonal terms
(nonOrthoFlags of the matrix and RHS operators) are differentiable through their adjoint kernels
(scalar.cu, nonortho.cu), and so are the ``timeStepNorm`` forms of the pressure operators and of the
corrector.  ``SetupAdvectionVelocity(apply_pressure_gradient=True)`` also returns the gradient with respect
to the blocks' pressure, which the reference's wrapper does not track.  Not differentiable here
(NotImplementedError): face transforms (``useFaceTransform``), whose forward operators the reference marks
experimental.
"""
from __future__ import annotations

import ctypes
import logging
from typing import Dict, List, Tuple

import torch

from . import _lib
from ._lib import check
from . import PISOtorch
from .engine import LinsolveError

_LOG = logging.getLogger("Diff")

_EXCLUDED_GRADIENTS: Dict[str, Tuple[set, set]] = {}


def exclude_gradient(function_name: str, grad_name: str, is_gradient_input: bool):
    """PISOtorch_diff.py:14-20: skip an input (is_gradient_input) or output gradient of an operator."""
    if function_name not in _EXCLUDED_GRADIENTS:
        raise KeyError("Unknown function '%s'" % function_name)
    _EXCLUDED_GRADIENTS[function_name][0 if is_gradient_input else 1].add(grad_name)


def clear_excluded_gradients():
    for v in _EXCLUDED_GRADIENTS.values():
        v[0].clear()
        v[1].clear()


def _get_solver_tolerance(tol=None, dtype=torch.float32):
    """PISOtorch_diff.py:183-189."""
    if tol is None:
        tol = 1e-8 if dtype == torch.float64 else 1e-5
    return tol


def _get_solver_tolerance_torch(tol=None, dtype=torch.float32):
    return torch.tensor([_get_solver_tolerance(tol, dtype)], dtype=dtype)


def check_non_ortho_rhs(non_ortho_flags):
    """True if the flags add explicit non-orthogonal right-hand-side terms, which read the velocity or
    pressure result (PISOtorch_diff.py:34-42); those results are then tracked inputs of the operator."""
    return bool(int(non_ortho_flags) & (PISOtorch.NON_ORTHO_DIRECT_RHS | PISOtorch.NON_ORTHO_DIAGONAL_RHS))


def _nonortho_grad(domain, flags, what, out_bar, A_bar=None, data_bar=None, coef_bar=None, vb=None):
    """Add the gradient of the non-orthogonal terms of one operator (pict_nonortho_grad)."""
    if int(flags) == 0:
        return
    check(_lib.load().pict_nonortho_grad(ctypes.byref(domain._desc), int(flags), what, _p(out_bar), _p(A_bar),
                                         _p(data_bar), _p(coef_bar), _p(vb), _stream()), "non-orthogonal grad")


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _dt(time_step):
    return float(time_step.item()) if isinstance(time_step, torch.Tensor) else float(time_step)


# ------------------------------------------------------------------------------------------ domain state

def _fixed(b, f):
    return isinstance(b.boundaries[f], PISOtorch.FixedBoundary)


def flatten_domain(domain, tensor_filter: List[str], empty: bool = False, exclusion_list=()):
    """(keys, tensors) of the domain tensors named in `tensor_filter` (PISOtorch_diff.py:44-118)."""
    keys, ts = [], []

    def add(key, t):
        keys.append(key)
        ts.append(None if (empty or key[0] in exclusion_list) else t)

    for name in tensor_filter:
        if name == "A":
            add(("A",), domain.A)
        elif name == "C":
            add(("C",), domain.C.coef)
        elif name == "P":
            add(("P",), domain.P.coef)
        elif name == "VISCOSITY":
            add(("VISCOSITY",), domain.viscosity)
        elif name == "VELOCITY_RESULT":
            add(("VELOCITY_RESULT",), domain.velocityResult)
        elif name == "PRESSURE_RHS":
            add(("PRESSURE_RHS",), domain.pressureRHS)
        elif name == "PRESSURE_RESULT":
            add(("PRESSURE_RESULT",), domain.pressureResult)
        elif name == "VELOCITY_RHS":
            add(("VELOCITY_RHS",), domain.velocityRHS)
        elif name == "PRESSURE_RHS_DIV":
            add(("PRESSURE_RHS_DIV",), domain.pressureRHSdiv)
        elif name == "PASSIVE_SCALAR_RESULT":
            add(("PASSIVE_SCALAR_RESULT",), domain.scalarResult)
        elif name == "PASSIVE_SCALAR_VISCOSITY":
            if domain.passiveScalarViscosity is not None:
                add(("PASSIVE_SCALAR_VISCOSITY",), domain.passiveScalarViscosity)
        else:
            for bi, b in enumerate(domain.getBlocks()):
                if name == "VELOCITY":
                    add(("VELOCITY", bi), b.velocity)
                elif name == "PRESSURE":
                    add(("PRESSURE", bi), b.pressure)
                elif name == "VELOCITY_SOURCE" and b.velocitySource is not None:
                    add(("VELOCITY_SOURCE", bi), b.velocitySource)
                elif name == "VISCOSITY_BLOCK" and b.viscosity is not None:
                    add(("VISCOSITY_BLOCK", bi), b.viscosity)
                elif name == "BOUNDARY_VELOCITY":
                    for f in range(2 * domain.getSpatialDims()):
                        if _fixed(b, f):
                            add(("BOUNDARY_VELOCITY", bi, f), b.boundaries[f].velocity)
                elif name == "PASSIVE_SCALAR" and b.passiveScalar is not None:
                    add(("PASSIVE_SCALAR", bi), b.passiveScalar)
                elif name == "BOUNDARY_PASSIVE_SCALAR":
                    for f in range(2 * domain.getSpatialDims()):
                        if _fixed(b, f) and b.boundaries[f].passiveScalar is not None:
                            add(("BOUNDARY_PASSIVE_SCALAR", bi, f), b.boundaries[f].passiveScalar)
    return keys, ts


def set_domain_tensors_from_flat(domain, keys, tensors):
    """Put saved forward tensors back on the domain (PISOtorch_diff.py:120-181)."""
    blocks = domain.getBlocks()
    for key, t in zip(keys, tensors):
        if t is None:
            continue
        k = key[0]
        if k == "A":
            domain.setA(t)
        elif k == "C":
            domain.C.setCoef(t)
        elif k == "P":
            domain.P.setCoef(t)
        elif k == "VISCOSITY":
            domain.setViscosity(t.detach())
        elif k == "VELOCITY_RESULT":
            domain.setVelocityResult(t)
        elif k == "PRESSURE_RHS":
            domain.setPressureRHS(t)
        elif k == "PRESSURE_RESULT":
            domain.setPressureResult(t)
        elif k == "VELOCITY":
            blocks[key[1]].setVelocity(t)
        elif k == "PRESSURE":
            blocks[key[1]].setPressure(t)
        elif k == "VELOCITY_SOURCE":
            blocks[key[1]].setVelocitySource(t)
        elif k == "VISCOSITY_BLOCK":
            blocks[key[1]].setViscosity(t)
        elif k == "BOUNDARY_VELOCITY":
            blocks[key[1]].boundaries[key[2]].setVelocity(t)
        elif k == "PASSIVE_SCALAR_RESULT":
            domain.setScalarResult(t)
        elif k == "PASSIVE_SCALAR_VISCOSITY":
            domain.setScalarViscosity(t)
        elif k == "PASSIVE_SCALAR":
            blocks[key[1]].setPassiveScalar(t)
        elif k == "BOUNDARY_PASSIVE_SCALAR":
            blocks[key[1]].boundaries[key[2]].setPassiveScalar(t)


class _Grads:
    """Per-call gradient accumulators and the mapping onto the tracked inputs."""

    def __init__(self, domain):
        self.d = domain
        self.D = domain.getSpatialDims()
        self.N = domain.getTotalSize()
        z = lambda n: torch.zeros(n, dtype=domain.getDtype(), device=domain.getDevice())
        self.z = z
        self.un = z(self.D * self.N)
        self.nu = z(self.N)
        self.src = z(self.D * self.N)
        self.vb = z(2 * self.D * self.D * self.N)

    def to_inputs(self, keys):
        """Write the accumulators into fresh gradient tensors of the blocks / boundaries and return the
        gradients aligned with `keys`."""
        d = self.d
        blocks = d.getBlocks()
        for b in blocks:
            b.setVelocityGrad(torch.zeros_like(b.velocity))
            if b.velocitySource is not None:
                b.setVelocitySourceGrad(torch.zeros_like(b.velocitySource))
            if b.viscosity is not None:
                b.setViscosityGrad(torch.zeros_like(b.viscosity))
            for f in range(2 * self.D):
                if _fixed(b, f):
                    b.boundaries[f].setVelocityGrad(torch.zeros_like(b.boundaries[f].velocity))
        d.UpdateDomainData()
        sim_nu = self.z(1)
        scratch = torch.zeros(max(1, len(blocks)), dtype=torch.float64, device=d.getDevice())
        check(_lib.load().pict_adjoint_to_blocks(ctypes.byref(d._desc), _p(self.un), _p(self.nu), _p(self.src),
                                                 _p(self.vb), _p(sim_nu), _p(scratch), _stream()), "adjoint_to_blocks")
        out = []
        for key in keys:
            k = key[0]
            if k == "VELOCITY":
                out.append(blocks[key[1]].velocityGrad)
            elif k == "VELOCITY_SOURCE":
                out.append(blocks[key[1]].velocitySourceGrad)
            elif k == "VISCOSITY_BLOCK":
                out.append(blocks[key[1]].viscosityGrad)
            elif k == "BOUNDARY_VELOCITY":
                out.append(blocks[key[1]].boundaries[key[2]].velocityGrad)
            elif k == "VISCOSITY":
                out.append(sim_nu.reshape(d.viscosity.shape).to(d.viscosity.device, d.viscosity.dtype))
            else:
                out.append(None)
        return out


def _zero_or(t, like):
    return torch.zeros_like(like) if t is None else t.contiguous()


def _apply_exclusions(name, keys, grads):
    excl = _EXCLUDED_GRADIENTS.get(name, (set(), set()))[1]
    return [None if (g is not None and k[0] + "_GRAD" in excl) else g for k, g in zip(keys, grads)]


# ------------------------------------------------------------------------------------------ linear solve

class LinsolveFailed(LinsolveError):
    pass


def _linear_solve_wrapper(csrMat, rhs, result, maxit_torch, tol_torch, convergence_criterion, use_BiCG,
                          matrix_rank_deficient, residual_reset_step, transpose, print_residual, return_best_result,
                          is_FWD=None, debug_out=False, double_fallback=False, BiCG_with_preconditioner=True,
                          BiCG_precondition_fallback=False):
    """Solve and check the reports (PISOtorch_diff.py:245-293).  An all-zero right-hand side gives x = 0.
    BiCGStab runs with the ILU(0) preconditioner when BiCG_with_preconditioner is set; with
    BiCG_precondition_fallback an unpreconditioned BiCGStab solve that did not succeed is repeated from zero
    with the preconditioner (PISOtorch_diff.py:276-286)."""
    if bool(rhs.eq(0).all()):
        result.zero_()
        return []
    use_pre = bool(use_BiCG and BiCG_with_preconditioner)
    infos = PISOtorch.SolveLinear(csrMat, rhs, result, maxit_torch, tol_torch, convergence_criterion, use_BiCG,
                                  matrix_rank_deficient, residual_reset_step, transpose, print_residual,
                                  return_best_result, BiCGwithPreconditioner=use_pre)

    def not_solved(sinfos):
        return (not return_best_result and any(not i.converged for i in sinfos)) or \
            (return_best_result and any(not i.isFiniteResidual for i in sinfos))

    if BiCG_precondition_fallback and use_BiCG and not use_pre and not_solved(infos):
        _LOG.warning("Not preconditioned BiCG solve failed, trying preconditioned.")
        result.zero_()
        infos = PISOtorch.SolveLinear(csrMat, rhs, result, maxit_torch, tol_torch, convergence_criterion, use_BiCG,
                                      matrix_rank_deficient, residual_reset_step, transpose, print_residual,
                                      return_best_result, BiCGwithPreconditioner=True)
    _check_solver_return_infos(infos, transpose, use_BiCG, float(tol_torch.reshape(-1)[0]) if isinstance(tol_torch, torch.Tensor) else tol_torch,
                               int(maxit_torch.reshape(-1)[0]) if isinstance(maxit_torch, torch.Tensor) else maxit_torch,
                               return_best_result, is_FWD)
    return infos


def _check_solver_return_infos(solver_infos, transpose, use_BiCG, tol, max_iter, return_best_result, is_FWD=None,
                               debug_out=False):
    """PISOtorch_diff.py:199-243: raise LinsolveError on non-convergence or a non-finite residual."""
    for i, info in enumerate(solver_infos):
        if not info.isFiniteResidual or (not info.converged and not return_best_result):
            raise LinsolveError("%s%s solve (%s) failed for RHS %d: %s (tol %g, max_iter %d)" % (
                "Bi" if use_BiCG else "", "CG", "transposed" if transpose else "forward", i, info, tol, max_iter))


def linear_solve_GPU(csrMat, rhs, transpose=False, use_BiCG=False, tol=None, max_iter=5000, return_best_result=False,
                     double_fallback: bool = False, BiCG_with_preconditioner: bool = True,
                     BiCG_precondition_fallback: bool = False):
    """x = A^-1 rhs, differentiable with respect to the matrix coefficients and rhs (PISOtorch_diff.py:295-375)."""
    conv = PISOtorch.ConvergenceCriterion.NORM2_NORMALIZED
    tol_torch = _get_solver_tolerance_torch(tol, rhs.dtype)
    maxit_torch = torch.IntTensor([max_iter])
    A = csrMat

    class LinearSolveFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, A_coef, b):
            x = torch.zeros_like(b)
            _linear_solve_wrapper(A, b.detach(), x, maxit_torch, tol_torch, conv, use_BiCG, False, 0, transpose, False,
                                  return_best_result, is_FWD=True, BiCG_with_preconditioner=BiCG_with_preconditioner,
                                  BiCG_precondition_fallback=BiCG_precondition_fallback)
            ctx.save_for_backward(A_coef, x)
            return x

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, grad_x):
            A_coef, x = ctx.saved_tensors
            grad_b = grad_A = None
            if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
                grad_b = torch.zeros_like(grad_x)
                Aw = PISOtorch.StencilMatrix(A._domain(), A_coef)
                _linear_solve_wrapper(Aw, grad_x.contiguous(), grad_b, maxit_torch, tol_torch, conv, use_BiCG, False, 0,
                                      not transpose, False, return_best_result, is_FWD=False,
                                      BiCG_with_preconditioner=BiCG_with_preconditioner,
                                      BiCG_precondition_fallback=BiCG_precondition_fallback)
                if ctx.needs_input_grad[0]:
                    d = A._domain()
                    grad_A = torch.zeros_like(A_coef)
                    nrhs = grad_b.numel() // d.getTotalSize()
                    # -grad_b x^T (transposed solve: -x grad_b^T)
                    a, bb = (grad_b, x) if not transpose else (x, grad_b)
                    check(_lib.load().pict_stencil_outer_product(ctypes.byref(d._desc), _p(a.contiguous()),
                                                                 _p(bb.contiguous()), nrhs, _p(grad_A), -1.0, _stream()),
                          "stencil outer product")
            return grad_A, grad_b

    return LinearSolveFunction.apply(A.coef, rhs)


# ------------------------------------------------------------------------------------------ assembly

_EXCLUDED_GRADIENTS["SetupAdvectionMatrix"] = (set(), set())


def SetupAdvectionMatrix(domain, time_step, non_ortho_flags, forPassiveScalar=False, passiveScalarChannel=0):
    """A, C = advection matrix (PISOtorch_diff.py:377-441); differentiable w.r.t. velocity, boundary
    velocity and viscosity; with ``forPassiveScalar`` the matrix of a passive scalar channel, differentiable
    w.r.t. velocity and the scalar viscosity (or the domain viscosity when there is none)."""
    if forPassiveScalar:
        return _scalar_matrix_function(domain, time_step, non_ortho_flags, int(passiveScalarChannel))
    keys, tracked = flatten_domain(domain, ["VELOCITY", "BOUNDARY_VELOCITY", "VISCOSITY", "VISCOSITY_BLOCK"])
    dt = _dt(time_step)

    class SetupAdvectionMatrixFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.CreateA()
            domain.C.CreateValue()
            domain.UpdateDomainData()
            PISOtorch.SetupAdvectionMatrix(domain, time_step, non_ortho_flags)
            ctx.saved = tracked_tensors
            return domain.A, domain.C.coef

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, A_grad, C_grad):
            if not any(ctx.needs_input_grad):
                return (None,) * len(keys)
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.UpdateDomainData()
            g = _Grads(domain)
            Ab = _zero_or(A_grad, domain.A)
            Cb = _zero_or(C_grad, domain.C.coef)
            zD = g.z(g.D * g.N)
            check(_lib.load().pict_advection_grad(ctypes.byref(domain._desc), dt, _p(zD), _p(zD), _p(Cb), _p(Ab),
                                                  _p(g.un), _p(g.nu), _p(g.vb), None, _stream()), "advection grad")
            _nonortho_grad(domain, non_ortho_flags, 0, Cb, A_bar=Ab, coef_bar=g.nu)
            return tuple(_apply_exclusions("SetupAdvectionMatrix", keys, g.to_inputs(keys)))

    return SetupAdvectionMatrixFunction.apply(*tracked)


def _scalar_viscosity_grads(domain, keys, grads, per_channel):
    """Put the per-channel scalar viscosity adjoint on the PASSIVE_SCALAR_VISCOSITY key, else on VISCOSITY."""
    for i, key in enumerate(keys):
        if key[0] == "PASSIVE_SCALAR_VISCOSITY":
            sv = domain.passiveScalarViscosity
            add = per_channel.sum() if sv.numel() == 1 else per_channel
            grads[i] = add.reshape(sv.shape).to(sv.device, sv.dtype)
            return grads
    for i, key in enumerate(keys):
        if key[0] == "VISCOSITY":
            v = domain.viscosity
            grads[i] = per_channel.sum().reshape(v.shape).to(v.device, v.dtype)
    return grads


def _scalar_matrix_function(domain, time_step, non_ortho_flags, channel):
    """C, A of passive scalar channel `channel` (PISOtorch_diff.py:377-441 with forPassiveScalar)."""
    keys, tracked = flatten_domain(domain, ["VELOCITY", "BOUNDARY_VELOCITY", "VISCOSITY", "PASSIVE_SCALAR_VISCOSITY"])
    dt = _dt(time_step)

    class SetupScalarMatrixFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.CreateA()
            domain.C.CreateValue()
            domain.UpdateDomainData()
            PISOtorch.SetupAdvectionMatrix(domain, time_step, non_ortho_flags, forPassiveScalar=True,
                                           passiveScalarChannel=channel)
            ctx.saved = tracked_tensors
            return domain.A, domain.C.coef

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, A_grad, C_grad):
            if not any(ctx.needs_input_grad):
                return (None,) * len(keys)
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.UpdateDomainData()
            g = _Grads(domain)
            nu = g.z(g.N)
            check(_lib.load().pict_scalar_grad(ctypes.byref(domain._desc), dt, int(non_ortho_flags), 0, channel,
                                               _p(_zero_or(C_grad, domain.C.coef)), _p(_zero_or(A_grad, domain.A)),
                                               _p(g.un), None, None, None, None, _p(nu), _stream()), "scalar matrix grad")
            grads = g.to_inputs(keys)
            per = torch.zeros(domain.getPassiveScalarChannels(), dtype=nu.dtype, device=nu.device)
            per[channel] = nu.sum()
            grads = _scalar_viscosity_grads(domain, keys, grads, per)
            return tuple(_apply_exclusions("SetupAdvectionMatrix", keys, grads))

    return SetupScalarMatrixFunction.apply(*tracked)


_EXCLUDED_GRADIENTS["SetupAdvectionScalar"] = (set(), set())


def SetupAdvectionScalar(domain, time_step, non_ortho_flags):
    """scalarRHS (PISOtorch_diff.py:444-529); differentiable w.r.t. the blocks' and boundaries' passive scalar,
    the boundary velocity, the scalar viscosity (or the domain viscosity) and, with non-orthogonal RHS
    flags, the scalar result."""
    is_non_ortho = check_non_ortho_rhs(non_ortho_flags)
    keys, tracked = flatten_domain(domain, ["PASSIVE_SCALAR", "BOUNDARY_PASSIVE_SCALAR", "BOUNDARY_VELOCITY", "VISCOSITY",
                                            "PASSIVE_SCALAR_VISCOSITY"]
                                   + (["PASSIVE_SCALAR_RESULT"] if is_non_ortho else []))
    dt = _dt(time_step)

    class SetupAdvectionScalarFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.CreateScalarRHS()
            domain.UpdateDomainData()
            PISOtorch.SetupAdvectionScalar(domain, time_step, non_ortho_flags)
            ctx.saved = tracked_tensors
            return domain.scalarRHS

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, grad_rhs):
            if not any(ctx.needs_input_grad):
                return (None,) * len(keys)
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.UpdateDomainData()
            g = _Grads(domain)
            C, N, D = domain.getPassiveScalarChannels(), g.N, g.D
            s_bar, sres, sb, nu = g.z(C * N), g.z(C * N), g.z(2 * D * C * N), g.z(C * N)
            check(_lib.load().pict_scalar_grad(ctypes.byref(domain._desc), dt, int(non_ortho_flags), 1, 0,
                                               _p(grad_rhs.contiguous()), None, None, _p(s_bar), _p(sres), _p(sb),
                                               _p(g.vb), _p(nu), _stream()), "scalar rhs grad")
            grads = g.to_inputs(keys)
            blocks = domain.getBlocks()
            s_bar, sb = s_bar.reshape(C, N), sb.reshape(2 * D, C, N)
            for i, key in enumerate(keys):
                if key[0] == "PASSIVE_SCALAR":
                    b = blocks[key[1]]
                    grads[i] = s_bar[:, b.globalOffset:b.globalOffset + b.pressure.numel()].reshape(b.passiveScalar.shape)
                elif key[0] == "BOUNDARY_PASSIVE_SCALAR":
                    b = blocks[key[1]]
                    bnd = b.boundaries[key[2]]
                    vals = sb[key[2]][:, PISOtorch._face_cells(b, key[2])]
                    grads[i] = vals.sum(dim=1).reshape(bnd.passiveScalar.shape) if bnd.passiveScalar.dim() == 2 \
                        else vals.reshape(bnd.passiveScalar.shape)
                elif key[0] == "PASSIVE_SCALAR_RESULT":
                    grads[i] = sres
            grads = _scalar_viscosity_grads(domain, keys, grads, nu.reshape(C, N).sum(dim=1))
            return tuple(_apply_exclusions("SetupAdvectionScalar", keys, grads))

    return SetupAdvectionScalarFunction.apply(*tracked)


_EXCLUDED_GRADIENTS["SetupAdvectionVelocity"] = (set(), set())


def SetupAdvectionVelocity(domain, time_step, non_ortho_flags, apply_pressure_gradient=False):
    """velocityRHS (PISOtorch_diff.py:531-613); differentiable w.r.t. velocity, source, boundary velocity
    and viscosity, with non-orthogonal RHS flags w.r.t. the velocity result, and with
    apply_pressure_gradient (velocityRHS -= dt grad p) w.r.t. the blocks' pressure (the reference's
    wrapper does not track the pressure there, so it gets no gradient from this operator)."""
    is_non_ortho = check_non_ortho_rhs(non_ortho_flags)
    keys, tracked = flatten_domain(domain, ["VELOCITY", "VELOCITY_SOURCE", "BOUNDARY_VELOCITY", "VISCOSITY",
                                            "VISCOSITY_BLOCK"] + (["VELOCITY_RESULT"] if is_non_ortho else [])
                                   + (["PRESSURE"] if apply_pressure_gradient else []))
    dt = _dt(time_step)

    class SetupAdvectionVelocityFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.CreateVelocityRHS()
            domain.UpdateDomainData()
            PISOtorch.SetupAdvectionVelocity(domain, time_step, non_ortho_flags, apply_pressure_gradient)
            ctx.saved = tracked_tensors
            return domain.velocityRHS

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, grad_rhs):
            if not any(ctx.needs_input_grad):
                return (None,) * len(keys)
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.UpdateDomainData()
            g = _Grads(domain)
            zD = g.z(g.D * g.N)
            zC = g.z((2 * g.D + 1) * g.N)
            zA = g.z(g.N)
            rb = grad_rhs.contiguous()
            check(_lib.load().pict_advection_grad(ctypes.byref(domain._desc), dt, _p(zD), _p(rb),
                                                  _p(zC), _p(zA), _p(g.un), _p(g.nu), _p(g.vb), _p(g.src), _stream()),
                  "advection rhs grad")
            Ub = g.z(g.D * g.N)
            if is_non_ortho:
                _nonortho_grad(domain, non_ortho_flags, 1, rb, data_bar=Ub, coef_bar=g.nu, vb=g.vb)
            grads = g.to_inputs(keys)
            if apply_pressure_gradient:
                # velocityRHS -= dt G p: the adjoint of the corrector's pressure term -G p / A with A = 1 / dt
                p_bar = _pressure_term_adjoint(domain, rb, torch.full_like(zA, 1.0 / dt))
            for i, key in enumerate(keys):
                if key[0] == "VELOCITY_RESULT":
                    grads[i] = Ub
                elif key[0] == "PRESSURE":
                    grads[i] = p_bar[key[1]]
            return tuple(_apply_exclusions("SetupAdvectionVelocity", keys, grads))

    return SetupAdvectionVelocityFunction.apply(*tracked)


def _pressure_term_adjoint(domain, u_bar, A):
    """Gradient with respect to the blocks' pressure of -G p / A (G the corrector's finite-difference
    pressure gradient) for the output gradient u_bar [D][N]: one tensor per block."""
    lib = _lib.load()
    N, D = domain.getTotalSize(), domain.getSpatialDims()
    z = lambda n: torch.zeros(n, dtype=domain.getDtype(), device=domain.getDevice())
    Ab, pb, hb = z(N), z(N), z(D * N)
    check(lib.pict_correct_velocity_grad(ctypes.byref(domain._desc), _p(A.contiguous()), _p(z(N)),
                                         _p(u_bar.contiguous()), _p(Ab), _p(pb), _p(hb), _stream()),
          "pressure term grad")
    saved = [b.pressureGrad for b in domain.getBlocks()]
    for b in domain.getBlocks():
        b.setPressureGrad(torch.zeros_like(b.pressure))
    domain.UpdateDomainData()
    check(lib.pict_copy_field(ctypes.byref(domain._desc), 4, 1, _p(pb), 0, _stream()), "scatter pressure grad")
    out = [b.pressureGrad.clone() for b in domain.getBlocks()]
    for b, g in zip(domain.getBlocks(), saved):
        if isinstance(g, torch.Tensor) and g.is_cuda and g.shape == b.pressure.shape:
            b.setPressureGrad(g)
    domain.UpdateDomainData()
    return out


def _pressure_rhs_backward(domain, dt, keys, h_grad, div_grad, P_grad, want_A, want_C, want_U, flags=0,
                           time_step_norm=False):
    """Shared backward of SetupPressureCorrection / Matrix / RHS / RHSdiv.  With non-orthogonal flags the
    matrix terms add to the A gradient and the explicit RHS terms (read from the pressure result saved by
    the forward pass) to the pressure result and A gradients."""
    lib = _lib.load()
    g = _Grads(domain)
    N, D = g.N, g.D
    desc = ctypes.byref(domain._desc)
    s = _stream()
    hb = g.z(D * N) if h_grad is None else h_grad.detach().clone().contiguous()
    Ab = g.z(N)
    Cb = g.z((2 * D + 1) * N)
    Ub = g.z(D * N)
    Pr = g.z(N)
    if div_grad is not None:
        db = div_grad.contiguous()
        # timeStepNorm divides the divergence by the time step, not the non-orthogonal terms added after it
        dbd = (db / dt).contiguous() if time_step_norm else db
        check(lib.pict_divergence_grad(desc, _p(dbd), _p(hb), _p(g.vb), s), "divergence grad")
        if check_non_ortho_rhs(flags):
            _nonortho_grad(domain, flags, 3, db, data_bar=Pr, coef_bar=Ab)
    if P_grad is not None:
        Pb = P_grad.contiguous()
        check(lib.pict_pressure_matrix_grad(desc, _p(domain.A), _p(Pb), _p(Ab), s), "pressure matrix grad")
        _nonortho_grad(domain, flags, 2, Pb, coef_bar=Ab)
    if h_grad is not None or div_grad is not None:
        zN = g.z(N)
        check(lib.pict_pressure_rhs_grad(desc, dt, _p(hb), _p(domain.pressureRHS), _p(domain.A), _p(domain.C.coef),
                                         _p(domain.velocityResult), _p(zN), _p(zN), _p(Ab), _p(Cb), _p(Ub), _p(g.un),
                                         _p(g.src), _p(g.nu), _p(g.vb), s), "pressure rhs grad")
    grads = g.to_inputs(keys)
    for i, key in enumerate(keys):
        if key[0] == "A":
            grads[i] = Ab
        elif key[0] == "C":
            grads[i] = Cb.reshape(domain.C.coef.shape)
        elif key[0] == "VELOCITY_RESULT":
            grads[i] = Ub
        elif key[0] == "PRESSURE_RHS":
            grads[i] = hb
        elif key[0] == "PRESSURE_RESULT":
            grads[i] = Pr
    return grads


_EXCLUDED_GRADIENTS["SetupPressureCorrection"] = (set(), set())


def SetupPressureCorrection(domain, time_step, non_ortho_flags, use_face_transform=False, timeStepNorm=False):
    """P, pressureRHS (H/A) and pressureRHSdiv (PISOtorch_diff.py:802-895)."""
    is_non_ortho = check_non_ortho_rhs(non_ortho_flags)
    keys, tracked = flatten_domain(domain, ["VELOCITY", "VELOCITY_SOURCE", "VELOCITY_RESULT", "BOUNDARY_VELOCITY",
                                            "VISCOSITY", "VISCOSITY_BLOCK", "A", "C"]
                                   + (["PRESSURE_RESULT"] if is_non_ortho else []))
    dt = _dt(time_step)

    class SetupPressureCorrectionFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.CreatePressureRHS()
            domain.CreatePressureRHSdiv()
            domain.P.CreateValue()
            domain.UpdateDomainData()
            PISOtorch.SetupPressureCorrection(domain, time_step, non_ortho_flags, use_face_transform, timeStepNorm=timeStepNorm)
            ctx.saved = tracked_tensors
            ctx.h = domain.pressureRHS
            return domain.P.coef, domain.pressureRHS, domain.pressureRHSdiv

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, P_grad, rhs_grad, div_grad):
            if not any(ctx.needs_input_grad):
                return (None,) * len(keys)
            if use_face_transform:
                raise NotImplementedError("SetupPressureCorrection: no gradient with face transforms")
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.setPressureRHS(ctx.h)
            domain.UpdateDomainData()
            grads = _pressure_rhs_backward(domain, dt, keys, rhs_grad, div_grad, P_grad, True, True, True,
                                           non_ortho_flags, timeStepNorm)
            return tuple(_apply_exclusions("SetupPressureCorrection", keys, grads))

    return SetupPressureCorrectionFunction.apply(*tracked)


_EXCLUDED_GRADIENTS["SetupPressureMatrix"] = (set(), set())


def SetupPressureMatrix(domain, time_step, non_ortho_flags, use_face_transform=False):
    """P from A (PISOtorch_diff.py:897-965)."""
    keys, tracked = flatten_domain(domain, ["A"])
    dt = _dt(time_step)

    class SetupPressureMatrixFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.P.CreateValue()
            domain.UpdateDomainData()
            PISOtorch.SetupPressureMatrix(domain, time_step, non_ortho_flags, use_face_transform)
            ctx.saved = tracked_tensors
            return domain.P.coef

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, P_grad):
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.UpdateDomainData()
            grads = _pressure_rhs_backward(domain, dt, keys, None, None, P_grad, True, False, False, non_ortho_flags)
            return tuple(_apply_exclusions("SetupPressureMatrix", keys, grads))

    return SetupPressureMatrixFunction.apply(*tracked)


_EXCLUDED_GRADIENTS["SetupPressureRHS"] = (set(), set())


def SetupPressureRHS(domain, time_step, non_ortho_flags, use_face_transform=False, timeStepNorm=False):
    """pressureRHS (H/A) and pressureRHSdiv (PISOtorch_diff.py:967-1065)."""
    is_non_ortho = check_non_ortho_rhs(non_ortho_flags)
    keys, tracked = flatten_domain(domain, ["VELOCITY", "VELOCITY_SOURCE", "VELOCITY_RESULT", "BOUNDARY_VELOCITY",
                                            "VISCOSITY", "VISCOSITY_BLOCK", "A", "C"]
                                   + (["PRESSURE_RESULT"] if is_non_ortho else []))
    dt = _dt(time_step)

    class SetupPressureRHSFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.CreatePressureRHS()
            domain.CreatePressureRHSdiv()
            domain.UpdateDomainData()
            PISOtorch.SetupPressureRHS(domain, time_step, non_ortho_flags, use_face_transform, timeStepNorm=timeStepNorm)
            ctx.saved = tracked_tensors
            ctx.h = domain.pressureRHS
            return domain.pressureRHS, domain.pressureRHSdiv

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, rhs_grad, div_grad):
            if use_face_transform:
                raise NotImplementedError("SetupPressureRHS: no gradient with face transforms")
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.setPressureRHS(ctx.h)
            domain.UpdateDomainData()
            grads = _pressure_rhs_backward(domain, dt, keys, rhs_grad, div_grad, None, True, True, True,
                                           non_ortho_flags, timeStepNorm)
            return tuple(_apply_exclusions("SetupPressureRHS", keys, grads))

    return SetupPressureRHSFunction.apply(*tracked)


_EXCLUDED_GRADIENTS["SetupPressureRHSdiv"] = (set(), set())


def SetupPressureRHSdiv(domain, time_step, non_ortho_flags, use_face_transform=False, timeStepNorm=False):
    """pressureRHSdiv from pressureRHS (PISOtorch_diff.py:1067-1158); with non-orthogonal RHS flags also
    from the pressure result and A."""
    is_non_ortho = check_non_ortho_rhs(non_ortho_flags)
    keys, tracked = flatten_domain(domain, ["PRESSURE_RHS", "BOUNDARY_VELOCITY"]
                                   + (["PRESSURE_RESULT", "A"] if is_non_ortho else []))
    dt = _dt(time_step)

    class SetupPressureRHSdivFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.CreatePressureRHSdiv()
            domain.UpdateDomainData()
            PISOtorch.SetupPressureRHSdiv(domain, time_step, non_ortho_flags, use_face_transform, timeStepNorm=timeStepNorm)
            ctx.saved = tracked_tensors
            return domain.pressureRHSdiv

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, div_grad):
            if use_face_transform:
                raise NotImplementedError("SetupPressureRHSdiv: no gradient with face transforms")
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.UpdateDomainData()
            g = _Grads(domain)
            hb = g.z(g.D * g.N)
            db = div_grad.contiguous()
            dbd = (db / dt).contiguous() if timeStepNorm else db
            check(_lib.load().pict_divergence_grad(ctypes.byref(domain._desc), _p(dbd), _p(hb),
                                                   _p(g.vb), _stream()), "divergence grad")
            Pr, Ab = g.z(g.N), g.z(g.N)
            if is_non_ortho:
                _nonortho_grad(domain, non_ortho_flags, 3, db, data_bar=Pr, coef_bar=Ab)
            grads = g.to_inputs(keys)
            for i, key in enumerate(keys):
                if key[0] == "PRESSURE_RHS":
                    grads[i] = hb
                elif key[0] == "PRESSURE_RESULT":
                    grads[i] = Pr
                elif key[0] == "A":
                    grads[i] = Ab
            return tuple(_apply_exclusions("SetupPressureRHSdiv", keys, grads))

    return SetupPressureRHSdivFunction.apply(*tracked)


# ------------------------------------------------------------------------------------------ correction

_EXCLUDED_GRADIENTS["CorrectVelocity"] = (set(), set())


def CorrectVelocity(domain, time_step, version, timeStepNorm=False):
    """velocityResult = pressureRHS - grad(p)/A (PISOtorch_diff.py:1160-1236).  The backward pass is the adjoint
    of the finite-difference corrector for versions 0/1 and, as in the reference (whose CorrectVelocityGrad
    has no version argument), also for the finite-volume versions 5 and 6, where it is exact on
    orthogonal grids; version 4 has no gradient."""
    keys, tracked = flatten_domain(domain, ["A", "PRESSURE", "PRESSURE_RHS"])

    class CorrectVelocityFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *tracked_tensors):
            domain.CreateVelocityResult()
            domain.UpdateDomainData()
            PISOtorch.CorrectVelocity(domain, time_step, version, timeStepNorm=timeStepNorm)
            ctx.saved = tracked_tensors
            return domain.velocityResult

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, u_grad):
            if not any(ctx.needs_input_grad):
                return (None,) * len(keys)
            if version not in (0, 1, 5, 6):
                raise NotImplementedError("CorrectVelocity: no gradient for version %d" % version)
            set_domain_tensors_from_flat(domain, keys, ctx.saved)
            domain.UpdateDomainData()
            lib = _lib.load()
            N, D = domain.getTotalSize(), domain.getSpatialDims()
            z = lambda n: torch.zeros(n, dtype=domain.getDtype(), device=domain.getDevice())
            p_glob = z(N)
            check(lib.pict_copy_field(ctypes.byref(domain._desc), 1, 0, _p(p_glob), 0, _stream()), "gather pressure")
            Ab, pb, hb = z(N), z(N), z(D * N)
            ug = u_grad.contiguous()
            # timeStepNorm multiplies the pressure update (not pressureRHS) by the time step
            ug_update = (ug * _dt(time_step)).contiguous() if timeStepNorm else ug
            check(lib.pict_correct_velocity_grad(ctypes.byref(domain._desc), _p(domain.A), _p(p_glob),
                                                 _p(ug_update), _p(Ab), _p(pb), _p(hb), _stream()),
                  "correct velocity grad")
            if timeStepNorm:
                hb = ug.clone()
            for b in domain.getBlocks():
                b.setPressureGrad(torch.zeros_like(b.pressure))
            domain.UpdateDomainData()
            check(lib.pict_copy_field(ctypes.byref(domain._desc), 4, 1, _p(pb), 0, _stream()), "scatter pressure grad")
            blocks = domain.getBlocks()
            grads = []
            for key in keys:
                if key[0] == "A":
                    grads.append(Ab)
                elif key[0] == "PRESSURE_RHS":
                    grads.append(hb)
                else:
                    grads.append(blocks[key[1]].pressureGrad)
            return tuple(_apply_exclusions("CorrectVelocity", keys, grads))

    CorrectVelocityFunction.apply(*tracked)


# ------------------------------------------------------------------------------------------ copies

def _copy_fn(to_blocks, vector):
    which_val = 0 if vector else 1        # FIELD_VELOCITY / FIELD_PRESSURE
    which_grad = 3 if vector else 4       # FIELD_VELOCITY_GRAD / FIELD_PRESSURE_GRAD
    return which_val, which_grad


def CopyVelocityResultToBlocks(domain):
    """Blocks' velocity = velocityResult (PISOtorch_diff.py:697-729)."""

    class CopyVelocityResultToBlocksFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, velocity_result):
            domain.CreateVelocityOnBlocks()
            domain.UpdateDomainData()
            PISOtorch.CopyVelocityResultToBlocks(domain)
            return tuple(b.velocity for b in domain.getBlocks())

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, *blocks_velocity_grad):
            for b, gv in zip(domain.getBlocks(), blocks_velocity_grad):
                b.setVelocityGrad(torch.zeros_like(b.velocity) if gv is None else gv.contiguous())
            domain.UpdateDomainData()
            out = torch.zeros(domain.getTotalSize() * domain.getSpatialDims(), dtype=domain.getDtype(),
                              device=domain.getDevice())
            check(_lib.load().pict_copy_field(ctypes.byref(domain._desc), 3, 0, _p(out), 0, _stream()), "copy grad")
            return out

    CopyVelocityResultToBlocksFunction.apply(domain.velocityResult)


def CopyVelocityResultFromBlocks(domain):
    """velocityResult = blocks' velocity (PISOtorch_diff.py:731-763)."""

    class CopyVelocityResultFromBlocksFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *block_velocity):
            domain.CreateVelocityResult()
            domain.UpdateDomainData()
            PISOtorch.CopyVelocityResultFromBlocks(domain)
            return domain.velocityResult

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, vr_grad):
            for b in domain.getBlocks():
                b.setVelocityGrad(torch.zeros_like(b.velocity))
            domain.UpdateDomainData()
            check(_lib.load().pict_copy_field(ctypes.byref(domain._desc), 3, 1, _p(vr_grad.contiguous()), 0, _stream()),
                  "copy grad")
            return tuple(b.velocityGrad for b in domain.getBlocks())

    CopyVelocityResultFromBlocksFunction.apply(*[b.velocity for b in domain.getBlocks()])


def CopyPressureResultToBlocks(domain):
    """Blocks' pressure = pressureResult (PISOtorch_diff.py:765-800)."""

    class CopyPressureResultToBlocksFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, pressure_result):
            domain.CreatePressureOnBlocks()
            domain.UpdateDomainData()
            PISOtorch.CopyPressureResultToBlocks(domain)
            return tuple(b.pressure for b in domain.getBlocks())

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, *blocks_pressure_grad):
            for b, gp in zip(domain.getBlocks(), blocks_pressure_grad):
                b.setPressureGrad(torch.zeros_like(b.pressure) if gp is None else gp.contiguous())
            domain.UpdateDomainData()
            out = torch.zeros(domain.getTotalSize(), dtype=domain.getDtype(), device=domain.getDevice())
            check(_lib.load().pict_copy_field(ctypes.byref(domain._desc), 4, 0, _p(out), 0, _stream()), "copy grad")
            return out

    CopyPressureResultToBlocksFunction.apply(domain.pressureResult)


def CopyScalarResultToBlocks(domain):
    """Blocks' passive scalar = scalarResult."""
    C = domain.getPassiveScalarChannels()

    class CopyScalarResultToBlocksFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, scalar_result):
            for b in domain.getBlocks():
                b.setPassiveScalar(torch.empty_like(b.passiveScalar))
            domain.UpdateDomainData()
            PISOtorch.CopyScalarResultToBlocks(domain)
            return tuple(b.passiveScalar for b in domain.getBlocks())

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, *grads):
            parts = [(torch.zeros_like(b.passiveScalar) if gs is None else gs).reshape(C, -1)
                     for b, gs in zip(domain.getBlocks(), grads)]
            return torch.cat(parts, dim=1).reshape(-1).contiguous()

    CopyScalarResultToBlocksFunction.apply(domain.scalarResult)


def CopyScalarResultFromBlocks(domain):
    """scalarResult = blocks' passive scalar."""
    C, N = domain.getPassiveScalarChannels(), domain.getTotalSize()

    class CopyScalarResultFromBlocksFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, *block_scalar):
            domain.CreateScalarResult()
            domain.UpdateDomainData()
            PISOtorch.CopyScalarResultFromBlocks(domain)
            return domain.scalarResult

        @staticmethod
        @torch.autograd.function.once_differentiable
        def backward(ctx, sr_grad):
            g = sr_grad.reshape(C, N)
            return tuple(g[:, b.globalOffset:b.globalOffset + b.pressure.numel()].reshape(b.passiveScalar.shape).contiguous()
                         for b in domain.getBlocks())

    CopyScalarResultFromBlocksFunction.apply(*[b.passiveScalar for b in domain.getBlocks()])


# ------------------------------------------------------------------------------------------ housekeeping

def reset_domain(domain):
    """PISOtorch_diff.py:1238-1246: fresh block tensors (releases the graph held by the domain)."""
    domain.CreateVelocityOnBlocks()
    domain.CreatePressureOnBlocks()


def detach_domain_fwd(domain):
    domain.DetachFwd()


def is_tensor_empty(tensor):
    return tensor is None or tensor.numel() == 0


def detach_domain_grad(domain):
    domain.DetachGrad()


def detach_domain(domain):
    domain.Detach()
