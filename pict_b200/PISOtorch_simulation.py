"""Drop-in mirror of the reference's simulation driver (PISOtorch_simulation.py).

``Simulation`` keeps the reference's constructor arguments, properties, hook
stages (``prep_fn``) and run loop (PISOtorch_simulation.py:398-1518).  Two
execution paths produce the same step:

* the generic path issues the operators one by one exactly like the reference's
  ``_PISO_split_step`` orthogonal branch (PISOtorch_simulation.py:1054-1327), so every
  ``prep_fn`` stage fires and the differentiable backend can record the graph;
* the fused path (no hooks, not differentiable, FD corrector, GPU solves) hands
  the whole step to :class:`pict_b200.engine.PISOStepper`, which launches it
  without host synchronisation.

With ``non_orthogonal=True`` and a domain whose metrics are not orthogonal, the step follows
the reference's non-orthogonal branch operator by operator, with the non-orthogonal matrix and
RHS terms (nonOrthoFlags) of the operators (on orthogonal metrics the terms vanish identically
and the fused step runs).  Image/VTK output belongs to the reference's post-processing utilities
and is not part of this package; the corresponding arguments are accepted and ignored with a
warning.
"""
from __future__ import annotations

import logging
import numbers
import signal
import warnings
from contextlib import nullcontext

import numpy as np
import torch

from . import PISOtorch
from .engine import LinsolveError, PISOStepper, default_tolerance

_LOG = logging.getLogger("PISOsim")
cpu_device = torch.device("cpu")


class StopHandler:
    """SIGINT handler polled by the run loop (PISOtorch_simulation.py:27-50)."""

    def __init__(self, log=None):
        self._log = log
        self.reset()

    def stop(self):
        if self._log is not None:
            self._log.warning("Simulation interrupted, stopping..." if not self._stop else "Simulation still stopping...")
        self._stop = True

    def signal_stop(self, sig, frame):
        self.stop()

    def __call__(self):
        return self._stop

    def register_signal(self):
        signal.signal(signal.SIGINT, self.signal_stop)

    def unregister_signal(self):
        signal.signal(signal.SIGINT, signal.SIG_DFL)

    def reset(self):
        self._stop = False


def ntonp(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def get_max_time_step(domain, time_step_target, CFL_cond=0.8, with_transformations=True):
    """PISOtorch_simulation.py:55-64."""
    max_vel = float(domain.getMaxVelocity(True, with_transformations).item())
    max_time_step = CFL_cond / max_vel
    if max_time_step >= time_step_target:
        return time_step_target, 1
    ss = int(np.ceil(time_step_target / max_time_step))
    return time_step_target / ss, ss


def tensor_as_np(tensor):
    return tensor.detach().cpu().numpy()


def getVelocityResultMaxMag(domain):
    """Largest velocity magnitude in domain.velocityResult, 0 for a zero field (PISOtorch_simulation.py:67-73)."""
    vel = domain.velocityResult.reshape(domain.getSpatialDims(), domain.getTotalSize())
    if float(torch.max(torch.abs(vel)).item()) > 0:
        return float(torch.max(torch.linalg.vector_norm(vel, dim=0)).item())
    return 0


def getVelocityResultMaxVel(domain):
    """Largest velocity component magnitude in domain.velocityResult (PISOtorch_simulation.py:75-78)."""
    return float(torch.max(torch.abs(domain.velocityResult)).item())


# ------------------------------------------------------------------ outflow boundaries (PISOtorch_simulation.py:80-312)
# Written against the boundary interface only (GetFluxes, velocity, transform, setVelocity, ...), so the
# same functions drive this package's domains and any object with the PISOtorch boundary interface.

def _is_fixed_boundary(bound):
    return type(bound).__name__ == "FixedBoundary"


def _solver_tolerance(tol, dtype):
    """Default solver tolerance by dtype (PISOtorch_diff.py:183-189)."""
    if tol is None:
        return 1e-8 if dtype == torch.float64 else 1e-5
    return tol


def get_fixed_boundary_flux(bound, bound_idx):
    """Total flux through a Dirichlet face: the sum of FixedBoundary.GetFluxes() (PISOtorch_simulation.py:80-90)."""
    if not _is_fixed_boundary(bound):
        raise AssertionError("get_fixed_boundary_flux needs a FixedBoundary")
    if int(bound.velocityType) != int(PISOtorch.BoundaryConditionType.DIRICHLET):
        raise ValueError("Only DIRICHLET boundaries are supportet")
    return torch.sum(bound.GetFluxes())


def get_fixed_boundary_fluxes(list_idx_bound):
    """Net outward flux of a list of (face index, FixedBoundary): the flux of an upper face (odd index)
    counts positive, of a lower face negative (PISOtorch_simulation.py:92-107)."""
    domain = list_idx_bound[0][1].getParentDomain()
    total = torch.zeros([1], dtype=domain.getDtype(), device=domain.getDevice())
    for face, bound in list_idx_bound:
        if not _is_fixed_boundary(bound):
            raise TypeError("boundary type not supported.")
        flux = get_fixed_boundary_flux(bound, face)
        total = total + flux if (face & 1) else total - flux
    return total


def get_advective_velocity(velms, velm_idx, bound, bound_idx):
    """Face-normal transport velocity of an outflow face, [1,1] for a static velocity on an
    untransformed face, else [1,1,(z),y,x] over the face cells: the face-normal component of the
    characteristic velocity `velms` (one [1,D] or [1,D,(z),y,x] tensor, or a list indexed by
    velm_idx), in computational coordinates (row `axis` of the face transform's inverse) when the face
    carries a transform (PISOtorch_simulation.py:145-172)."""
    velm = velms if isinstance(velms, torch.Tensor) else velms[velm_idx]
    dims = bound.getSpatialDims()
    axis = bound_idx >> 1
    sizes = bound.getSizes()
    face_shape = [int(sizes[dims - 1 - d]) for d in range(dims)]  # z, y, x
    static = velm.dim() == 2
    if not static:
        assert all(velm.size(2 + d) == face_shape[d] for d in range(dims)), "varying velm size must match boundary"
    has_transform = bound.hasTransform() if callable(getattr(bound, "hasTransform", None)) else bound.hasTransform
    if not has_transform:
        return velm[:, axis:axis + 1]
    if static:
        velm = velm.reshape([1, dims] + [1] * dims).expand([1, dims] + face_shape)
    row = bound.transform[..., dims * dims + axis * dims: dims * dims + (axis + 1) * dims]  # [1,(z),y,x,D]
    v = torch.movedim(velm, 1, -1)  # [1,(z),y,x,D]
    adv = torch.matmul(row.reshape(-1, 1, dims), v.reshape(-1, dims, 1))
    return adv.reshape([1, 1] + face_shape)


def balance_boundary_fluxes(domain, free_bounds, tol=None):
    """Scale the velocity of the free (outflow) faces so that the net flux through all Dirichlet faces
    vanishes, unless it already does to 1% of the solver tolerance (PISOtorch_simulation.py:174-208)."""
    with torch.no_grad():
        faces = []
        for block in domain.getBlocks():
            faces.extend(block.getFixedBoundaries())
        fixed = [fb for fb in faces if fb[1] not in free_bounds]
        free = [fb for fb in faces if fb[1] in free_bounds]
        fixed_flux = get_fixed_boundary_fluxes(fixed)
        free_flux = get_fixed_boundary_fluxes(free)
    atol = _solver_tolerance(tol, domain.getDtype()) * 0.01
    if not torch.allclose(fixed_flux + free_flux, torch.zeros_like(fixed_flux), atol=atol):
        scale = -fixed_flux / free_flux
        for _, bound in free:
            bound.setVelocity(bound.velocity * scale)


def _face_layer(t, face):
    """The cell layer of a block field [1,C,(z),y,x] next to `face` (kept as a size-1 axis)."""
    dim = t.dim() - 1 - (face >> 1)
    return t.narrow(dim, t.size(dim) - 1 if (face & 1) else 0, 1)


def update_advective_boundaries(domain, bounds, velms, dt, tol=None):
    """Advective outflow: every face in `bounds` (varying Dirichlet FixedBoundary objects) moves its
    velocity (and passive scalar) towards the adjacent cell layer by the implicit upwind weight
    t = 1 - 1/(1 + 2 dt c), c = get_advective_velocity(velms, ...), then the free faces are rescaled to
    balance the domain's boundary fluxes (PISOtorch_simulation.py:210-312)."""
    with torch.no_grad():
        dims = domain.getSpatialDims()
        assert isinstance(bounds, list) and len(bounds) > 0
        assert (isinstance(velms, torch.Tensor) and velms.dim() == 2 and velms.size(0) == 1 and velms.size(1) == dims) \
            or (isinstance(velms, list) and len(velms) == len(bounds) and all(
                isinstance(v, torch.Tensor) and v.dim() in (2, dims + 2) and v.size(0) == 1 and v.size(1) == dims
                for v in velms)), "velms tensors have wrong shape"
        entries = []
        for bi in range(domain.getNumBlocks()):
            block = domain.getBlock(bi)
            for face in range(2 * dims):
                bound = block.getBoundary(face)
                if _is_fixed_boundary(bound) and bound in bounds:
                    entries.append((block, face, bound))
        if len(entries) != len(bounds):
            raise ValueError("Bounds passed as advective outflow are not (all) part of the domain.")
        for block, face, bound in entries:
            vel_layer = _face_layer(block.velocity, face)
            alpha = dt * 2 * get_advective_velocity(velms, bounds.index(bound), bound, face)
            t = 1 - 1 / (1 + alpha)
            if bound.isVelocityStatic:
                raise ValueError("outflow boundaries must be varying. Use FixedBoundary.makeVelocityVarying() to make the velocity varying.")
            scalar_bound = None
            if block.hasPassiveScalar() and bound.hasPassiveScalar():
                if bound.isPassiveScalarStatic():
                    raise ValueError("outflow boundary passive scalar must be varying.")
                if any(int(c) != int(PISOtorch.BoundaryConditionType.DIRICHLET) for c in bound.passiveScalarTypes):
                    raise ValueError("passive scalar outflow boundary condition must be Dirichlet.")
                scalar_bound = bound.passiveScalar
            vel = bound.velocity
            bound.setVelocity(vel - t * (vel - vel_layer))
            if scalar_bound is not None:
                scalar_layer = _face_layer(block.passiveScalar, face)
                bound.setPassiveScalar(scalar_bound - t * (scalar_bound - scalar_layer))
    balance_boundary_fluxes(domain, bounds, tol=tol)


def metrics_are_orthogonal(domain, rtol=1e-6):
    """True if every cell transform has mutually orthogonal Minv rows (non-orthogonal terms vanish)."""
    D = domain.getSpatialDims()
    for b in domain.getBlocks():
        if not b.hasTransform():
            continue
        T = b.transform.reshape(-1, 2 * D * D + 1)
        Minv = T[:, D * D:2 * D * D].reshape(-1, D, D)
        G = torch.bmm(Minv, Minv.transpose(1, 2))
        diag = torch.diagonal(G, dim1=1, dim2=2)
        off = G - torch.diag_embed(diag)
        scale = diag.abs().max(dim=1).values.clamp_min(1e-300)
        if (off.abs().amax(dim=(1, 2)) / scale).max().item() > rtol:
            return False
    return True


class Simulation:
    NON_ORTHO_DIRECT_MATRIX = 1
    NON_ORTHO_DIRECT_RHS = 2
    NON_ORTHO_DIAGONAL_MATRIX = 4
    NON_ORTHO_DIAGONAL_RHS = 8
    NON_ORTHO_CENTER_MATRIX = 16
    _NON_ORTHO_MODE = NON_ORTHO_CENTER_MATRIX | NON_ORTHO_DIRECT_MATRIX | NON_ORTHO_DIAGONAL_RHS

    def __init__(self, domain=None, *, time_step=1.0, substeps=1, corrector_steps=2, density_viscosity=None,
                 adaptive_CFL=0.8, prep_fn=None, advection_use_BiCG=True, pressure_use_BiCG=False,
                 scipy_solve_advection=False, scipy_solve_pressure=False, preconditionBiCG=False,
                 BiCG_precondition_fallback=True, advection_tol=None, pressure_tol=None, convergence_tol=None,
                 solver_double_fallback=False, advect_non_ortho_steps=1, pressure_non_ortho_steps=1,
                 advect_reuse_result=False, pressure_reuse_result=False, normalize_pressure_result=True,
                 pressure_return_best_result=False, advect_passive_scalar=True, pressure_time_step_normalized=False,
                 velocity_corrector="FD", non_orthogonal=True, differentiable=False,
                 exclude_advection_solve_gradients=False, exclude_pressure_solve_gradients=False, log_dir=None,
                 log_interval=0, log_images=True, log_vtk=False, norm_vel=False, block_layout=None,
                 output_mode3D="slice", log_fn=None, output_resampling_coords=None, output_resampling_shape=None,
                 output_resampling_fill_max_steps=0, save_domain_name=None, stop_fn=lambda: False):
        if density_viscosity is not None:
            raise NotImplementedError("Simulation.density_viscosity is superseded by Domain.scalarViscosity.")
        self.domain = domain
        self.prep_fn = prep_fn
        self.non_orthogonal = non_orthogonal
        self.time_step = time_step
        self.substeps = substeps
        self.corrector_steps = corrector_steps
        self.convergence_tol = convergence_tol
        self.adaptive_CFL = adaptive_CFL
        self.scipy_solve_advection = scipy_solve_advection
        self.advection_use_BiCG = advection_use_BiCG
        self.advect_non_ortho_steps = advect_non_ortho_steps
        self.advection_tol = advection_tol
        self.advect_passive_scalar = advect_passive_scalar
        self.advect_reuse_result = advect_reuse_result
        self.scipy_solve_pressure = scipy_solve_pressure
        self.pressure_use_BiCG = pressure_use_BiCG
        self.pressure_non_ortho_steps = pressure_non_ortho_steps
        self.pressure_tol = pressure_tol
        self.normalize_pressure_result = normalize_pressure_result
        self.pressure_return_best_result = pressure_return_best_result
        self.pressure_time_step_normalized = pressure_time_step_normalized
        self.pressure_reuse_result = pressure_reuse_result
        self.solver_double_fallback = solver_double_fallback
        self.linear_solve_max_iterations = 5000
        self.preconditionBiCG = preconditionBiCG
        self.BiCG_precondition_fallback = BiCG_precondition_fallback
        self._velocity_corrector_versions = {"FD": 1, "FVM_CENTER": 5, "FVM_FACE": 6}
        self.velocity_corrector = velocity_corrector
        self.log_dir = log_dir
        self.log_interval = log_interval or 0
        self.log_images = log_images
        self.log_vtk = log_vtk
        self.norm_vel = norm_vel
        self.block_layout = block_layout
        self.log_fn = log_fn
        self.save_domain_name = save_domain_name
        self.differentiable = differentiable
        self.exclude_advection_solve_gradients = exclude_advection_solve_gradients
        self.exclude_pressure_solve_gradients = exclude_pressure_solve_gradients
        self.stop_fn = stop_fn
        self.use_fused_step = True
        self._stepper = None
        self._stepper_key = None
        self.reset_step_counters()

    # ------------------------------------------------------------------ properties (PISOtorch_simulation.py:478-860)
    @property
    def domain(self):
        return self._domain

    @domain.setter
    def domain(self, domain):
        if domain is not None:
            if not isinstance(domain, PISOtorch.Domain):
                raise TypeError("domain must be a PISOtorch.Domain object or None.")
            if not domain.IsInitialized():
                raise RuntimeError("domain must be initilized. Call domain.PrepareSolve() before assignment.")
        self._domain = domain
        self._stepper = None

    def _check_domain(self):
        if self._domain is None:
            raise ValueError("no domain set.")

    def _get_dtype(self):
        self._check_domain()
        return self.domain.getBlock(0).velocity.dtype

    @property
    def differentiable(self):
        return self._differentiable

    @differentiable.setter
    def differentiable(self, differentiable):
        if not isinstance(differentiable, bool):
            raise TypeError("differentiable must be bool.")
        self._differentiable = differentiable
        if differentiable:
            from . import PISOtorch_diff
            self._backend = PISOtorch_diff
        else:
            self._backend = PISOtorch

    @property
    def non_orthogonal(self):
        return self._non_orthogonal

    @non_orthogonal.setter
    def non_orthogonal(self, v):
        if not isinstance(v, bool):
            raise TypeError("non_orthogonal must be bool.")
        self._non_orthogonal = v

    @property
    def time_step(self):
        return self._time_step

    @time_step.setter
    def time_step(self, v):
        if not isinstance(v, numbers.Real):
            raise TypeError("time_step must be float.")
        self._time_step = v

    def _get_time_step_torch(self):
        return torch.tensor([self._time_step], device=cpu_device, dtype=self._get_dtype())

    @property
    def substeps(self):
        return self._substeps

    @substeps.setter
    def substeps(self, v):
        if isinstance(v, str) and v.upper() == "ADAPTIVE":
            v = -1
        elif not isinstance(v, numbers.Integral):
            raise TypeError("substeps must be integral type or 'ADAPTIVE'.")
        elif not v > 0 and v not in (-1, -2):
            raise ValueError("substeps must be positive.")
        self._substeps = v

    @property
    def corrector_steps(self):
        return self._corrector_steps

    @corrector_steps.setter
    def corrector_steps(self, v):
        if not isinstance(v, numbers.Integral):
            raise TypeError("corrector_steps must be integral type.")
        if v < 0:
            raise ValueError("corrector_steps must not be negative.")
        self._corrector_steps = v

    @property
    def advection_tol(self):
        return default_tolerance(self._get_dtype()) if self._advection_tol is None else self._advection_tol

    @advection_tol.setter
    def advection_tol(self, v):
        if v is not None and not (isinstance(v, numbers.Real) and v > 0):
            raise ValueError("advection_tol must be positive float or None.")
        self._advection_tol = v

    @property
    def pressure_tol(self):
        return default_tolerance(self._get_dtype()) if self._pressure_tol is None else self._pressure_tol

    @pressure_tol.setter
    def pressure_tol(self, v):
        if v is not None and not (isinstance(v, numbers.Real) and v > 0):
            raise ValueError("pressure_tol must be positive float or None.")
        self._pressure_tol = v

    @property
    def velocity_corrector(self):
        return self._velocity_corrector

    @velocity_corrector.setter
    def velocity_corrector(self, v):
        if v not in self._velocity_corrector_versions:
            raise ValueError("velocity_corrector must be one of: %s" % (list(self._velocity_corrector_versions.keys()),))
        self._velocity_corrector = v
        self._velocity_corrector_version = self._velocity_corrector_versions[v]

    @property
    def stop_fn(self):
        return self._stop_fn

    @stop_fn.setter
    def stop_fn(self, v):
        if v is None:
            v = lambda: False
        if not callable(v):
            raise TypeError("stop_fn must be callable or None.")
        self._stop_fn = v

    def _check_stop(self):
        return self._stop_fn is not None and self._stop_fn()

    @property
    def prep_fn(self):
        return self._prep_fn

    @prep_fn.setter
    def prep_fn(self, v):
        if not (v is None or isinstance(v, dict)):
            raise TypeError("prep_fn must be dict or None.")
        self._prep_fn = v

    def _run_prep_fn(self, name, **kwargs):
        if self._prep_fn and name in self._prep_fn and self._prep_fn[name] is not None:
            fns = self._prep_fn[name]
            if not isinstance(fns, (list, tuple)):
                fns = [fns]
            for fn in fns:
                if fn is not None:
                    fn(**kwargs)

    # ------------------------------------------------------------------ counters
    def reset_total_step(self):
        self.total_step = 0

    def reset_total_time(self):
        self.total_time = 0

    def end_step(self, time_step=0):
        self.total_step += 1
        self.total_time += float(ntonp(time_step).reshape(-1)[0])

    def reset_step_counters(self):
        self.reset_total_step()
        self.reset_total_time()

    # ------------------------------------------------------------------ solves (PISOtorch_simulation.py:861-904)
    def linear_solve(self, csrMat, rhs, x=None, use_BiCG=False, tol=None, max_iter=None, matrix_rank_deficient=False,
                     residual_reset_step=0, use_scipy=False, return_best_result=False):
        if use_scipy:
            raise NotImplementedError("SciPy solves are not part of the B200 step; use the GPU solvers")
        if max_iter is None:
            max_iter = self.linear_solve_max_iterations
        tol = default_tolerance(rhs.dtype) if tol is None else tol
        if self._backend is PISOtorch:
            if x is None:
                x = torch.zeros_like(rhs)
            if bool(rhs.eq(0).all()):
                x.zero_()
                return x, True
            pre = bool(use_BiCG and self.preconditionBiCG)
            infos = PISOtorch.SolveLinear(csrMat, rhs, x, max_iter, tol, PISOtorch.ConvergenceCriterion.NORM2_NORMALIZED,
                                          use_BiCG, False, residual_reset_step, False, False, return_best_result,
                                          BiCGwithPreconditioner=pre)
            if self.BiCG_precondition_fallback and use_BiCG and not pre and _not_solved(infos, return_best_result):
                # PISOtorch_diff.py:276-286: repeat a failed unpreconditioned BiCGStab solve, preconditioned
                _LOG.warning("Not preconditioned BiCG solve failed, trying preconditioned.")
                x.zero_()
                infos = PISOtorch.SolveLinear(csrMat, rhs, x, max_iter, tol, PISOtorch.ConvergenceCriterion.NORM2_NORMALIZED,
                                              use_BiCG, False, residual_reset_step, False, False, return_best_result,
                                              BiCGwithPreconditioner=True)
            _check_infos(infos, use_BiCG, tol, max_iter, return_best_result)
            return x, True
        return self._backend.linear_solve_GPU(csrMat, rhs, transpose=False, use_BiCG=use_BiCG, tol=tol,
                                              max_iter=max_iter, return_best_result=return_best_result,
                                              BiCG_with_preconditioner=self.preconditionBiCG,
                                              BiCG_precondition_fallback=self.BiCG_precondition_fallback), True

    # ------------------------------------------------------------------ step
    def _fused_eligible(self):
        d = self.domain
        return (self.use_fused_step and not self.differentiable and not self._prep_fn and self.convergence_tol is None
                and self._velocity_corrector_version == 1 and not self.pressure_time_step_normalized
                and not self.scipy_solve_advection and not self.scipy_solve_pressure and self.advection_use_BiCG
                and not self.pressure_use_BiCG and self.normalize_pressure_result
                and not (self.advect_passive_scalar and d.hasPassiveScalar()))

    def _non_ortho_flags(self):
        """The nonOrthoFlags of this step: the driver's mode (PISOtorch_simulation.py:390-396, 579-585) when
        non_orthogonal is set and some block's metric is not exactly orthogonal; 0 otherwise (the terms
        vanish identically on orthogonal metrics, so the orthogonal step is taken)."""
        if not self.non_orthogonal:
            return 0
        key = id(self.domain)
        if getattr(self, "_ortho_key", None) != key:
            self._ortho_flags = 0 if metrics_are_orthogonal(self.domain, rtol=0.0) else Simulation._NON_ORTHO_MODE
            self._ortho_key = key
        return self._ortho_flags

    def _check_non_ortho(self):
        """The non-orthogonal branch runs through the operators of the backend (PISOtorch_diff when
        differentiable, whose gradient operators include the non-orthogonal terms); nothing to reject."""
        return self._non_ortho_flags()

    def _get_stepper(self):
        key = (id(self.domain), self.corrector_steps, self.advection_tol, self.pressure_tol,
               self.linear_solve_max_iterations)
        if self._stepper is None or self._stepper_key != key:
            self._stepper = PISOStepper(self.domain, corrector_steps=self.corrector_steps,
                                        advection_tol=self.advection_tol, pressure_tol=self.pressure_tol,
                                        max_iterations=self.linear_solve_max_iterations)
            self._stepper_key = key
        return self._stepper

    def _PISO_split_step(self, iterations, time_step=None):
        self._check_domain()
        self._check_non_ortho()
        if time_step is None:
            time_step = self._get_time_step_torch()
        if isinstance(iterations, torch.Tensor):
            iterations = int(iterations.numpy()[0])
        assert iterations > 0
        domain = self.domain
        if self._fused_eligible() and not self._non_ortho_flags():
            if domain.IsTensorChanged():
                domain.UpdateDomainData()
            st = self._get_stepper()
            st.desc = domain._make_desc()
            for _ in range(iterations):
                st.step(time_step)
                st.check()
                if self._check_stop():
                    break
                self.end_step(time_step)
            return True
        return self._PISO_split_step_ops(iterations, time_step)

    def _advect_scalar(self, step, time_step, flags, non_ortho_branch=None):
        """Passive scalar advection at the start of a step (PISOtorch_simulation.py:1085-1167).  The channels are
        solved together with one matrix (BiCGStab with C right-hand sides) unless the scalar viscosity
        or the boundary types differ per channel; without non_orthogonal the RHS is set up once, else
        the blocks' scalar is copied to scalarResult for the explicit terms and advect_non_ortho_steps
        solves are made.  Returns (solve ok, whether the scalar matrix also serves the velocity: the
        reference reuses it when neither a scalar or block viscosity nor per-channel settings exist)."""
        domain = self.domain
        B = self._backend
        C = domain.getPassiveScalarChannels()
        n = domain.getTotalSize()
        split = not (domain.isPassiveScalarViscosityStatic() and domain.isAllFixedBoundariesPassiveScalarTypeStatic())
        matrix_for_velocity = not (domain.hasPassiveScalarViscosity() or domain.hasBlockViscosity()
                                   or domain.hasPassiveScalarBlockViscosity() or split)
        matrices = []
        if split:
            for ch in range(C):
                B.SetupAdvectionMatrix(domain, time_step, flags, forPassiveScalar=True, passiveScalarChannel=ch)
                matrices.append(domain.C.clone())
        else:
            B.SetupAdvectionMatrix(domain, time_step, flags, forPassiveScalar=True, passiveScalarChannel=0)
        ortho = not (self.non_orthogonal if non_ortho_branch is None else non_ortho_branch)
        reuse = self.advect_reuse_result and not self.differentiable
        if not ortho:
            B.CopyScalarResultFromBlocks(domain)
        solve_ok = True
        for no_step in range(1 if ortho else self.advect_non_ortho_steps):
            B.SetupAdvectionScalar(domain, time_step, 0 if ortho else flags)
            self._run_prep_fn("POST_SCALAR_SETUP", domain=domain, no_step=no_step, local_step=step, time_step=time_step,
                              total_step=self.total_step, total_time=self.total_time)
            first = ortho or no_step == 0 or not reuse
            with torch.no_grad() if self.exclude_advection_solve_gradients else nullcontext():
                if split:
                    xs = [None] * C if first else [x.clone() for x in torch.split(domain.scalarResult, n)]
                    rhs = torch.split(domain.scalarRHS, n)
                    parts = []
                    for ch in range(C):
                        sr, solve_ok = self.linear_solve(matrices[ch], rhs[ch], x=xs[ch], use_BiCG=self.advection_use_BiCG,
                                                         use_scipy=self.scipy_solve_advection, tol=self.advection_tol)
                        parts.append(sr)
                    scalar_result = torch.cat(parts)
                else:
                    x = None if first else domain.scalarResult.clone()
                    scalar_result, solve_ok = self.linear_solve(domain.C, domain.scalarRHS, x=x,
                                                                use_BiCG=self.advection_use_BiCG,
                                                                use_scipy=self.scipy_solve_advection,
                                                                tol=self.advection_tol)
            domain.setScalarResult(scalar_result)
            domain.UpdateDomainData()
            if not ortho and (not solve_ok or self._check_stop()):
                return solve_ok, matrix_for_velocity
        B.CopyScalarResultToBlocks(domain)
        return solve_ok, matrix_for_velocity

    def advect_static(self, iterations, time_step=None):
        """Advect only the passive scalar with the current velocity (PISOtorch_simulation.py:907-983)."""
        self._check_domain()
        if isinstance(iterations, torch.Tensor):
            iterations = int(iterations.numpy()[0])
        if time_step is None:
            time_step = self._get_time_step_torch()
        domain = self.domain
        if not domain.hasPassiveScalar():
            raise ValueError("Domain has no passive scalar to advect.")
        flags = self._non_ortho_flags()
        solve_ok = True
        for step in range(iterations):
            self._run_prep_fn("PRE", domain=domain, local_step=step, time_step=time_step, total_step=self.total_step,
                              total_time=self.total_time)
            domain.UpdateDomainData()
            # the reference's static advection always takes the non-orthogonal branch of the scalar solve
            solve_ok, _ = self._advect_scalar(step, time_step, flags, non_ortho_branch=True)
            self._run_prep_fn("POST", domain=domain, local_step=step, time_step=time_step, total_step=self.total_step,
                              total_time=self.total_time)
            if not solve_ok or self._check_stop():
                break
            self.end_step(time_step)
        return solve_ok

    def _PISO_split_step_ops(self, iterations, time_step):
        """Operator-by-operator step, PISOtorch_simulation.py:1054-1327 (orthogonal branch, or the non-orthogonal
        branch PISOtorch_simulation.py:1194-1296 when the domain's metrics are not orthogonal)."""
        domain = self.domain
        B = self._backend
        vcv = self._velocity_corrector_version
        solve_ok = True
        advect_use_prev_result = self.advect_reuse_result and not self.differentiable
        flags = self._non_ortho_flags()
        if flags:
            return self._PISO_split_step_non_ortho(iterations, time_step, flags)
        for step in range(iterations):
            if self.convergence_tol is not None:
                B.CopyVelocityResultFromBlocks(domain)
                last_vel = domain.velocityResult.clone().detach()
            self._run_prep_fn("PRE", domain=domain, local_step=step, time_step=time_step, total_step=self.total_step,
                              total_time=self.total_time)
            domain.UpdateDomainData()
            matrix_for_velocity = False
            if self.advect_passive_scalar and domain.hasPassiveScalar():
                solve_ok, matrix_for_velocity = self._advect_scalar(step, time_step, 0)
                if not solve_ok or self._check_stop():
                    return solve_ok
            self._run_prep_fn("PRE_VELOCITY_SETUP", domain=domain, local_step=step, time_step=time_step,
                              total_step=self.total_step, total_time=self.total_time)
            if not matrix_for_velocity:
                B.SetupAdvectionMatrix(domain, time_step, 0)
            B.SetupAdvectionVelocity(domain, time_step, 0, False)
            self._run_prep_fn("POST_VELOCITY_SETUP", domain=domain, no_step=0, local_step=step, time_step=time_step,
                              total_step=self.total_step, total_time=self.total_time)
            with torch.no_grad() if self.exclude_advection_solve_gradients else nullcontext():
                x = None if not advect_use_prev_result else domain.velocityResult
                velocityResult, solve_ok = self.linear_solve(domain.C, domain.velocityRHS, x=x,
                                                             use_BiCG=self.advection_use_BiCG,
                                                             use_scipy=self.scipy_solve_advection, tol=self.advection_tol)
            domain.setVelocityResult(velocityResult)
            domain.UpdateDomainData()
            self._run_prep_fn("POST_PREDICTION", domain=domain, local_step=step, time_step=time_step,
                              total_step=self.total_step, total_time=self.total_time)
            if self._check_stop():
                break
            for cstep in range(self.corrector_steps):
                B.SetupPressureCorrection(domain, time_step, 0, False, timeStepNorm=self.pressure_time_step_normalized)
                self._run_prep_fn("POST_PRESSURE_SETUP", domain=domain, local_step=step, time_step=time_step,
                                  total_step=self.total_step, total_time=self.total_time)
                with torch.no_grad() if self.exclude_pressure_solve_gradients else nullcontext():
                    pressureResult, solve_ok = self.linear_solve(domain.P, domain.pressureRHSdiv, x=None,
                                                                 use_BiCG=self.pressure_use_BiCG,
                                                                 use_scipy=self.scipy_solve_pressure,
                                                                 tol=self.pressure_tol,
                                                                 return_best_result=self.pressure_return_best_result)
                if self.normalize_pressure_result:
                    pressureResult = pressureResult - torch.mean(pressureResult)
                domain.setPressureResult(pressureResult)
                domain.UpdateDomainData()
                self._run_prep_fn("POST_PRESSURE_RESULT", domain=domain, local_step=step, time_step=time_step,
                                  total_step=self.total_step, total_time=self.total_time)
                self._run_prep_fn("POST_PRESSURE_NON_ORTHO", domain=domain, local_step=step, time_step=time_step,
                                  total_step=self.total_step, total_time=self.total_time)
                B.CopyPressureResultToBlocks(domain)
                B.CorrectVelocity(domain, time_step, version=vcv, timeStepNorm=self.pressure_time_step_normalized)
                self._run_prep_fn("POST_VELOCITY_CORRECTION", domain=domain, local_step=step, time_step=time_step,
                                  total_step=self.total_step, total_time=self.total_time)
                if self._check_stop():
                    break
            B.CopyVelocityResultToBlocks(domain)
            self._run_prep_fn("POST", domain=domain, local_step=step, time_step=time_step, total_step=self.total_step,
                              total_time=self.total_time)
            if self.convergence_tol is not None:
                diff = torch.max(torch.abs(last_vel - domain.velocityResult)).item()
                if diff < self.convergence_tol:
                    _LOG.info("Simulation step max difference is under convergence tolerance.")
                    solve_ok = False
            if not solve_ok or self._check_stop():
                break
            self.end_step(time_step)
        return solve_ok

    def _PISO_split_step_non_ortho(self, iterations, time_step, flags):
        """The non-orthogonal branch of Simulation._PISO_split_step, PISOtorch_simulation.py:1180-1296: the velocity
        result is copied from the blocks for the explicit terms of the velocity RHS (advect_non_ortho_steps
        solves); each corrector builds P once and solves pressure_non_ortho_steps times, the first with
        a fresh H/A field, the next ones with its divergence plus the explicit terms of the latest pressure
        result (CG with a residual reset every 100 iterations, as the reference driver asks)."""
        domain = self.domain
        B = self._backend
        vcv = self._velocity_corrector_version
        solve_ok = True
        advect_reuse = self.advect_reuse_result and not self.differentiable
        pressure_reuse = self.pressure_reuse_result and not self.differentiable
        for step in range(iterations):
            if self.convergence_tol is not None:
                B.CopyVelocityResultFromBlocks(domain)
                last_vel = domain.velocityResult.clone().detach()
            self._run_prep_fn("PRE", domain=domain, local_step=step, time_step=time_step, total_step=self.total_step,
                              total_time=self.total_time)
            domain.UpdateDomainData()
            matrix_for_velocity = False
            if self.advect_passive_scalar and domain.hasPassiveScalar():
                solve_ok, matrix_for_velocity = self._advect_scalar(step, time_step, flags)
                if not solve_ok or self._check_stop():
                    return solve_ok
            self._run_prep_fn("PRE_VELOCITY_SETUP", domain=domain, local_step=step, time_step=time_step,
                              total_step=self.total_step, total_time=self.total_time)
            if not matrix_for_velocity:
                B.SetupAdvectionMatrix(domain, time_step, flags)
            B.CopyVelocityResultFromBlocks(domain)
            for no_step in range(self.advect_non_ortho_steps):
                B.SetupAdvectionVelocity(domain, time_step, flags, False)
                self._run_prep_fn("POST_VELOCITY_SETUP", domain=domain, no_step=no_step, local_step=step,
                                  time_step=time_step, total_step=self.total_step, total_time=self.total_time)
                with torch.no_grad() if self.exclude_advection_solve_gradients else nullcontext():
                    x = None if (no_step == 0 or not advect_reuse) else domain.velocityResult
                    velocityResult, solve_ok = self.linear_solve(domain.C, domain.velocityRHS, x=x,
                                                                 use_BiCG=self.advection_use_BiCG,
                                                                 use_scipy=self.scipy_solve_advection,
                                                                 tol=self.advection_tol)
                domain.setVelocityResult(velocityResult)
                domain.UpdateDomainData()
                if not solve_ok or self._check_stop():
                    return solve_ok
            self._run_prep_fn("POST_PREDICTION", domain=domain, local_step=step, time_step=time_step,
                              total_step=self.total_step, total_time=self.total_time)
            if self._check_stop():
                break
            for cstep in range(self.corrector_steps):
                B.SetupPressureMatrix(domain, time_step, flags, False)
                for pstep in range(self.pressure_non_ortho_steps):
                    if pstep == 0:
                        B.SetupPressureRHS(domain, time_step, flags, False, timeStepNorm=self.pressure_time_step_normalized)
                    else:
                        B.SetupPressureRHSdiv(domain, time_step, flags, False,
                                              timeStepNorm=self.pressure_time_step_normalized)
                    self._run_prep_fn("POST_PRESSURE_SETUP", domain=domain, local_step=step, time_step=time_step,
                                      total_step=self.total_step, total_time=self.total_time)
                    with torch.no_grad() if self.exclude_pressure_solve_gradients else nullcontext():
                        x = None if (pstep == 0 or not pressure_reuse) else domain.pressureResult
                        pressureResult, solve_ok = self.linear_solve(domain.P, domain.pressureRHSdiv, x=x,
                                                                     residual_reset_step=100,
                                                                     use_BiCG=self.pressure_use_BiCG,
                                                                     use_scipy=self.scipy_solve_pressure,
                                                                     tol=self.pressure_tol,
                                                                     return_best_result=self.pressure_return_best_result)
                    if self.normalize_pressure_result:
                        pressureResult = pressureResult - torch.mean(pressureResult)
                    domain.setPressureResult(pressureResult)
                    domain.UpdateDomainData()
                    self._run_prep_fn("POST_PRESSURE_RESULT", domain=domain, local_step=step, time_step=time_step,
                                      total_step=self.total_step, total_time=self.total_time)
                    if not solve_ok:
                        return solve_ok
                    if self._check_stop():
                        break
                self._run_prep_fn("POST_PRESSURE_NON_ORTHO", domain=domain, local_step=step, time_step=time_step,
                                  total_step=self.total_step, total_time=self.total_time)
                B.CopyPressureResultToBlocks(domain)
                B.CorrectVelocity(domain, time_step, version=vcv, timeStepNorm=self.pressure_time_step_normalized)
                self._run_prep_fn("POST_VELOCITY_CORRECTION", domain=domain, local_step=step, time_step=time_step,
                                  total_step=self.total_step, total_time=self.total_time)
                if self._check_stop():
                    break
            B.CopyVelocityResultToBlocks(domain)
            self._run_prep_fn("POST", domain=domain, local_step=step, time_step=time_step, total_step=self.total_step,
                              total_time=self.total_time)
            if self.convergence_tol is not None:
                diff = torch.max(torch.abs(last_vel - domain.velocityResult)).item()
                if diff < self.convergence_tol:
                    _LOG.info("Simulation step max difference is under convergence tolerance.")
                    solve_ok = False
            if not solve_ok or self._check_stop():
                break
            self.end_step(time_step)
        return solve_ok

    def _PISO_adaptive_step(self, CFL_cond=None, max_subsetps=1000):
        """PISOtorch_simulation.py:1329-1372."""
        time_step_target = self.time_step
        domain = self.domain
        CFL_cond = CFL_cond if CFL_cond is not None else self.adaptive_CFL
        substep = 0
        while time_step_target > 0 and not np.isclose(time_step_target, 0):
            max_vel = float(domain.getMaxVelocity(True, True).item())
            max_time_step = time_step_target if np.isclose(max_vel, 0) else CFL_cond / max_vel
            if max_time_step >= time_step_target:
                ts = time_step_target
            else:
                ts = time_step_target / int(np.ceil(time_step_target / max_time_step))
            time_step_target -= ts
            ok = self._PISO_split_step(iterations=1, time_step=torch.tensor([ts], dtype=self._get_dtype()))
            substep += 1
            if not ok or self._check_stop():
                return False
        return True

    def make_divergence_free(self, iterations=1, max_iter=1000):
        """Pressure projection of the current velocity with A = 1, dt = 1 (PISOtorch_simulation.py:985-1052), with
        the non-orthogonal terms (pressure_non_ortho_steps solves) on non-orthogonal metrics."""
        self._check_domain()
        self._check_non_ortho()
        domain = self.domain
        B = self._backend
        flags = self._non_ortho_flags()
        pressure_reuse = self.pressure_reuse_result and not self.differentiable
        if isinstance(iterations, torch.Tensor):
            iterations = int(iterations.numpy()[0])
        time_step = torch.tensor([1], device=cpu_device, dtype=domain.A.dtype)
        domain.setA(torch.ones_like(domain.A))
        solve_ok = True
        for step in range(iterations):
            self._run_prep_fn("PRE", domain=domain, local_step=step, time_step=time_step, total_step=self.total_step,
                              total_time=self.total_time)
            domain.UpdateDomainData()
            B.CopyVelocityResultFromBlocks(domain)
            domain.setPressureRHS(domain.velocityResult)
            domain.UpdateDomainData()
            B.SetupPressureMatrix(domain, time_step, flags, False)
            for pstep in range(self.pressure_non_ortho_steps if flags else 1):
                B.SetupPressureRHSdiv(domain, time_step, flags, False, timeStepNorm=self.pressure_time_step_normalized)
                x = None if (pstep == 0 or not pressure_reuse) else domain.pressureResult
                pressureResult, solve_ok = self.linear_solve(domain.P, domain.pressureRHSdiv, x=x,
                                                             use_BiCG=self.pressure_use_BiCG, tol=self.pressure_tol,
                                                             max_iter=max_iter,
                                                             return_best_result=self.pressure_return_best_result)
                if self.normalize_pressure_result:
                    pressureResult = pressureResult - torch.mean(pressureResult)
                domain.setPressureResult(pressureResult)
                domain.UpdateDomainData()
                if not solve_ok:
                    return solve_ok
                if self._check_stop():
                    break
            B.CopyPressureResultToBlocks(domain)
            B.CorrectVelocity(domain, time_step, version=self._velocity_corrector_version,
                              timeStepNorm=self.pressure_time_step_normalized)
            B.CopyVelocityResultToBlocks(domain)
            if not solve_ok or self._check_stop():
                return solve_ok
            self.end_step(time_step)
        return solve_ok

    def run(self, iterations, static=False, log_domain=True):
        """PISOtorch_simulation.py:1374-1518 without image/VTK output; ``static`` advects only the passive scalar."""
        self._check_domain()
        domain = self.domain
        if self.log_interval > 0 and (self.log_images or self.log_vtk):
            warnings.warn("image/VTK output is not part of pict_b200; log_images/log_vtk are ignored")
        if domain.GetCoordinateOrientation() == 0:
            _LOG.warning("Domain coordinate systems have mixed orientation. This can lead to issues with the simulation.")
        flux = abs(float(domain.GetBoundaryFluxBalance().item()))
        if flux > float(self.pressure_tol):
            _LOG.warning("Domain boundary is not divergence free (flux balance: %.03e). This can prevent pressure solve "
                         "convergence.", flux)
            return False
        sim_ok = True
        substeps = self.substeps
        time_step = None
        adaptive = substeps == -1
        if substeps == -2:
            ts, substeps = get_max_time_step(domain, self.time_step, 0.8, with_transformations=True)
            time_step = torch.tensor([ts], dtype=self._get_dtype())
        for it in range(1, iterations + 1):
            try:
                if static:
                    sim_ok = self.advect_static(iterations=substeps, time_step=time_step)
                elif adaptive:
                    sim_ok = self._PISO_adaptive_step()
                else:
                    sim_ok = self._PISO_split_step(iterations=substeps, time_step=time_step)
            except LinsolveError:
                _LOG.exception("Simulation failed in major step %d (total step %d):", it, self.total_step)
                break
            max_mag = float(domain.getMaxVelocityMagnitude(False).item())
            if np.isnan(max_mag):
                _LOG.warning("NaN encountered in velocity, stopping")
                sim_ok = False
                break
            if self.log_interval > 0 and it % self.log_interval == 0:
                div = PISOtorch.ComputeVelocityDivergence(domain).abs()
                p = domain.pressureResult
                _LOG.info("%d/%d Stats: max mag=%.03e, p mean=%.03e min=%.03e max=%.03e, |div| mean=%.03e max=%.03e",
                          it, iterations, max_mag, p.mean().item(), p.min().item(), p.max().item(),
                          div.mean().item(), div.max().item())
            if self.log_fn is not None:
                self.log_fn(domain=domain, out_dir=self.log_dir, it=it, out_it=0, total_step=self.total_step)
            if self._check_stop() or not sim_ok:
                break
        return sim_ok


def _not_solved(infos, return_best_result):
    return (not return_best_result and any(not i.converged for i in infos)) or \
        (return_best_result and any(not i.isFiniteResidual for i in infos))


def _check_infos(infos, use_BiCG, tol, max_iter, return_best_result):
    """_check_solver_return_infos, PISOtorch_diff.py:199-243."""
    if any(not i.isFiniteResidual for i in infos):
        bad = [k for k, i in enumerate(infos) if not i.isFiniteResidual]
        raise LinsolveError("Linear solve (BiCG:%s, tol:%.03e) reported non-finite residual for RHS %s of %d. Solver infos:\n%s."
                            % (use_BiCG, tol, bad, len(infos), "\n".join("\t%s" % i for i in infos)))
    if any(not i.converged for i in infos):
        bad = [k for k, i in enumerate(infos) if not i.converged]
        msg = "Linear solve (BiCG:%s, tol:%.03e) RHS %s of %d did not converge after %d iterations." % (
            use_BiCG, tol, bad, len(infos), max_iter)
        if return_best_result:
            _LOG.warning(msg)
        else:
            raise LinsolveError(msg)
