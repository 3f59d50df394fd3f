"""ctypes binding of ``libpict_b200.so`` (declared in ``include/pict_b200.h``).

The shared library is the product's compute path; when it is missing or fails
to load, every operation raises ``PictLibraryError`` -- there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpict_b200.so")

PICT_OK = 0
PICT_F32 = 0
PICT_F64 = 1
PICT_FACE_FIXED = 0
PICT_FACE_PERIODIC = 1
PICT_FACE_CONNECTED = 2
PICT_CONV_NORM2 = 0
PICT_CONV_NORM2_NORMALIZED = 1
PICT_PRECOND_AS_REFERENCE = 0
PICT_PRECOND_ILU0 = 1


class PictLibraryError(RuntimeError):
    pass


class PictError(RuntimeError):
    """A C-ABI entry point returned a non-zero status."""


c_i32 = ctypes.c_int32
c_vp = ctypes.c_void_p


class Face(ctypes.Structure):
    _fields_ = [
        ("type", c_i32),
        ("conn_block", c_i32),
        ("conn_axes", c_i32 * 3),
        ("vel_static", c_i32),
        ("velocity", c_vp),
        ("transform", c_vp),
        ("velocity_grad", c_vp),
        ("scalar_static", c_i32),
        ("scalar_neumann", ctypes.c_uint32),
        ("scalar", c_vp),
        ("scalar_grad", c_vp),
    ]


class BlockDesc(ctypes.Structure):
    _fields_ = [
        ("size", c_i32 * 3),
        ("offset", c_i32),
        ("sim", c_i32),
        ("viscosity_static", c_i32),
        ("source_static", c_i32),
        ("pad0", c_i32),
        ("velocity", c_vp),
        ("pressure", c_vp),
        ("transform", c_vp),
        ("viscosity", c_vp),
        ("source", c_vp),
        ("velocity_grad", c_vp),
        ("pressure_grad", c_vp),
        ("viscosity_grad", c_vp),
        ("source_grad", c_vp),
        ("face", Face * 6),
        ("face_transform", c_vp),
        ("scalar", c_vp),
        ("scalar_grad", c_vp),
    ]


class DomainDesc(ctypes.Structure):
    _fields_ = [
        ("dims", c_i32),
        ("num_blocks", c_i32),
        ("num_cells", c_i32),
        ("num_sims", c_i32),
        ("dtype", c_i32),
        ("max_sim_cells", c_i32),
        ("blocks", c_vp),
        ("nbr", c_vp),
        ("cell_block", c_vp),
        ("sim_cells", c_vp),
        ("sim_blocks", c_vp),
        ("tiles", c_vp),
        ("sim_tiles", c_vp),
        ("num_tiles", c_i32),
        ("tile_cells", c_i32),
        ("sim_viscosity", c_vp),
        ("sim_dt", c_vp),
        ("C", c_vp),
        ("A", c_vp),
        ("P", c_vp),
        ("velocity_rhs", c_vp),
        ("velocity_result", c_vp),
        ("pressure_rhs", c_vp),
        ("pressure_rhs_div", c_vp),
        ("pressure_result", c_vp),
        ("scalar_channels", c_i32),
        ("scalar_viscosity_static", c_i32),
        ("scalar_viscosity", c_vp),
        ("scalar_rhs", c_vp),
        ("scalar_result", c_vp),
    ]


class MgLevel(ctypes.Structure):
    _fields_ = [
        ("num_cells", c_i32),
        ("num_blocks", c_i32),
        ("dims", c_i32),
        ("dtype", c_i32),
        ("blocks", c_vp),
        ("cell_block", c_vp),
        ("coef", c_vp),
        ("num_tiles", c_i32),
        ("max_block_cells", c_i32),
        ("tiles", c_vp),
        ("max_block_sx", c_i32),
        ("sweeps", c_i32),
    ]


class SolveInfo(ctypes.Structure):
    _fields_ = [
        ("final_residual", ctypes.c_double),
        ("used_iterations", c_i32),
        ("converged", c_i32),
        ("finite", c_i32),
        ("status", c_i32),
    ]


class SolveParams(ctypes.Structure):
    _fields_ = [
        ("max_iterations", c_i32),
        ("use_bicg", c_i32),
        ("nrhs", c_i32),
        ("x_is_zero", c_i32),
        ("transpose", c_i32),
        ("convergence", c_i32),
        ("group_size", c_i32),
        ("threads", c_i32),
        ("subtract_mean", c_i32),
        ("write_block_pressure", c_i32),
        ("variant", c_i32),
        ("residual_reset_steps", c_i32),
        ("return_best_result", c_i32),
        ("rank_deficient", c_i32),
        ("tolerance", ctypes.c_double),
    ]


SOLVE_INFO_BYTES = ctypes.sizeof(SolveInfo)

# name -> (restype, argtypes); must match include/pict_b200.h
_PD = ctypes.POINTER(DomainDesc)
_PS = ctypes.POINTER(SolveParams)
SIGNATURES = {
    "pict_version": (ctypes.c_char_p, []),
    "pict_last_error": (ctypes.c_char_p, []),
    "pict_sizeof_block": (c_i32, []),
    "pict_sizeof_domain": (c_i32, []),
    "pict_build_topology": (c_i32, [ctypes.POINTER(BlockDesc), c_i32, c_i32, c_i32, c_vp, c_vp]),
    "pict_build_tiles": (c_i32, [ctypes.POINTER(BlockDesc), c_i32, c_i32, c_i32, c_vp, c_i32, c_vp, c_vp]),
    "pict_setup_advection_matrix": (c_i32, [_PD, ctypes.c_double, c_i32, c_vp]),
    "pict_setup_advection_velocity": (c_i32, [_PD, ctypes.c_double, c_i32, c_i32, c_vp]),
    "pict_setup_advection": (c_i32, [_PD, ctypes.c_double, c_vp]),
    "pict_setup_pressure_matrix": (c_i32, [_PD, c_i32, c_vp]),
    "pict_setup_pressure_rhs": (c_i32, [_PD, ctypes.c_double, c_i32, c_i32, c_vp]),
    "pict_setup_pressure_rhs_div": (c_i32, [_PD, ctypes.c_double, c_i32, c_i32, c_vp]),
    "pict_setup_pressure_correction": (c_i32, [_PD, ctypes.c_double, c_i32, c_i32, c_vp]),
    "pict_correct_velocity": (c_i32, [_PD, ctypes.c_double, c_i32, c_i32, c_i32, c_vp]),
    "pict_copy_velocity_result_to_blocks": (c_i32, [_PD, c_vp]),
    "pict_copy_velocity_result_from_blocks": (c_i32, [_PD, c_vp]),
    "pict_advection_guess": (c_i32, [_PD, c_vp, c_i32, c_vp]),
    "pict_copy_pressure_result_to_blocks": (c_i32, [_PD, c_vp]),
    "pict_copy_pressure_result_from_blocks": (c_i32, [_PD, c_vp]),
    "pict_velocity_divergence": (c_i32, [_PD, c_vp, c_vp]),
    "pict_solve_workspace_bytes": (ctypes.c_int64, [_PD, _PS]),
    "pict_solve": (c_i32, [_PD, c_vp, c_vp, c_vp, _PS, c_vp, c_vp, ctypes.c_int64, c_vp]),
    "pict_solve_static_scratch_bytes": (ctypes.c_int64, []),
    "pict_solve_static": (c_i32, [_PD, c_vp, c_vp, c_vp, _PS, c_vp, c_vp]),
    "pict_refine_residual": (c_i32, [_PD, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp]),
    "pict_refine_update": (c_i32, [_PD, c_vp, c_vp, c_vp]),
    "pict_refine_finish": (c_i32, [_PD, c_vp, c_vp, c_i32, c_i32, c_vp, c_vp]),
    "pict_vector_axpby": (c_i32, [c_i32, c_i32, ctypes.c_double, c_vp, ctypes.c_double, c_vp, c_vp, c_vp]),
    "pict_mg_set_bulk_staging": (None, [c_i32]),
    "pict_mg_set_smoothing_sweeps": (None, [c_i32]),
    "pict_mg_set_graph_loop": (None, [c_i32]),
    "pict_mg_set_dependent_launch": (None, [c_i32]),
    "pict_krylov_set_cluster_mode": (None, [c_i32]),
    "pict_krylov_set_bicgstab_variant": (None, [c_i32]),
    "pict_mb_pad_gather": (c_i32, [c_i32, c_i32, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pict_mb_pad_scatter_sum": (c_i32, [c_i32, c_i32, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                        c_vp]),
    "pict_ilu_analyze": (c_i32, [c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pict_bicgstab_ilu_workspace_bytes": (ctypes.c_int64, [c_i32, c_i32, c_i32]),
    "pict_ilu0_factor": (c_i32, [c_i32, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_vp]),
    "pict_bicgstab_ilu": (c_i32, [c_i32, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_i32,
                                  c_vp, c_vp, c_vp, c_i32, c_i32, ctypes.c_double, c_i32, c_i32, c_i32, c_i32, c_vp,
                                  c_vp, ctypes.c_int64, c_vp]),
    "pict_mg_galerkin": (c_i32, [ctypes.POINTER(MgLevel), ctypes.POINTER(MgLevel), c_vp]),
    "pict_pcg_mg_workspace_bytes": (ctypes.c_int64, [_PD, ctypes.POINTER(MgLevel), c_i32]),
    "pict_pcg_mg": (c_i32, [_PD, ctypes.POINTER(MgLevel), c_i32, c_vp, c_vp, c_i32, ctypes.c_double, c_i32, c_vp, c_vp,
                            ctypes.c_int64, ctypes.c_double, ctypes.c_double, c_i32, c_vp]),
    "pict_correct_velocity_grad": (c_i32, [_PD, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pict_sim_mean_project": (c_i32, [_PD, c_vp, c_vp]),
    "pict_divergence_grad": (c_i32, [_PD, c_vp, c_vp, c_vp, c_vp]),
    "pict_pressure_rhs_grad": (c_i32, [_PD, ctypes.c_double] + [c_vp] * 15),
    "pict_advection_grad": (c_i32, [_PD, ctypes.c_double] + [c_vp] * 9),
    "pict_adjoint_to_blocks": (c_i32, [_PD] + [c_vp] * 7),
    "pict_copy_field": (c_i32, [_PD, c_i32, c_i32, c_vp, c_i32, c_vp]),
    "pict_stencil_outer_product": (c_i32, [_PD, c_vp, c_vp, c_i32, c_vp, ctypes.c_double, c_vp]),
    "pict_pressure_matrix_grad": (c_i32, [_PD, c_vp, c_vp, c_vp, c_vp]),
    "pict_nonortho_grad": (c_i32, [_PD, c_i32, c_i32] + [c_vp] * 6),
    "pict_setup_scalar_matrix": (c_i32, [_PD, ctypes.c_double, c_i32, c_i32, c_vp]),
    "pict_setup_scalar_rhs": (c_i32, [_PD, ctypes.c_double, c_i32, c_vp]),
    "pict_copy_scalar_result": (c_i32, [_PD, c_i32, c_vp]),
    "pict_sgs_smagorinsky": (c_i32, [_PD, ctypes.c_double, c_vp, c_vp]),
    "pict_advective_outflow": (c_i32, [_PD, c_vp, c_i32, c_vp, ctypes.c_double, ctypes.c_double, c_vp]),
    "pict_scalar_grad": (c_i32, [_PD, ctypes.c_double, c_i32, c_i32, c_i32] + [c_vp] * 9),
    "pict_csr_row_ptr": (c_i32, [_PD, c_vp, c_vp]),
    "pict_stencil_to_csr": (c_i32, [_PD, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pict_csr_to_stencil": (c_i32, [_PD, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pict_coords_to_transforms": (c_i32, [c_vp, c_i32, ctypes.POINTER(c_i32), c_i32, c_vp, c_vp]),
    "pict_coords_to_face_transforms": (c_i32, [c_vp, c_i32, ctypes.POINTER(c_i32), c_i32, c_vp, c_vp]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the library (once) and set the prototypes of every exported symbol."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise PictLibraryError(
            "libpict_b200.so not found at %s; build it with `python -m pict_b200.build`" % path)
    try:
        lib = ctypes.CDLL(path)
    except OSError as e:
        raise PictLibraryError("failed to load %s: %s" % (path, e))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.pict_sizeof_block() != ctypes.sizeof(BlockDesc):
        raise PictLibraryError("pict_block_t layout mismatch (%d vs %d)" % (lib.pict_sizeof_block(), ctypes.sizeof(BlockDesc)))
    if lib.pict_sizeof_domain() != ctypes.sizeof(DomainDesc):
        raise PictLibraryError("pict_domain_t layout mismatch")
    _lib = lib
    return lib


def check(status: int, what: str = ""):
    if status != PICT_OK:
        msg = load().pict_last_error().decode(errors="replace")
        raise PictError("%s failed (status %d): %s" % (what or "pict call", status, msg))
