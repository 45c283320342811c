"""ctypes binding of libmpdg_b200.so (the C ABI declared in include/mpdg_gpu.h).

There is no fallback: if the library is missing or cannot be loaded, importing the operators
raises.  Build it with ``python -m meltpooldg_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MPDG_LIB_PATH") or os.path.join(HERE, "libmpdg_b200.so")

MPDG_OK = 0
MPDG_ERR_ARG = 1
MPDG_ERR_CUDA = 2
MPDG_ERR_NOT_CONVERGED = 3
MPDG_ERR_ZERO_DT = 4
MPDG_ERR_TIMEOUT = 5
MPDG_ERR_UNSUPPORTED = 6
MPDG_ERR_NOMEM = 7

MPDG_HEAT = 0
MPDG_ADVDIFF = 1
MPDG_REINIT = 2
MPDG_CG = 0
MPDG_GMRES = 1
MPDG_PRECOND_IDENTITY = 0
MPDG_PRECOND_JACOBI = 1


class MeshDesc(C.Structure):
    _fields_ = [
        ("degree", C.c_int32),
        ("cells", C.c_int32 * 3),
        ("origin", C.c_double * 3),
        ("length", C.c_double * 3),
        ("dirichlet_faces", C.c_uint32),
        ("dirichlet_mask", C.c_void_p),
    ]


class OpParams(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("reserved", C.c_int32),
        ("rho_cp", C.c_double),
        ("dt", C.c_double),
        ("conductivity", C.c_double),
        ("conductivity_cells", C.c_void_p),
        ("theta", C.c_double),
        ("diffusivity", C.c_double),
        ("velocity", C.c_double * 12),
    ]


class HeatBC(C.Structure):
    """mpdg_heat_bc: convection / radiation / Neumann terms on whole box faces (6-bit masks)."""

    _fields_ = [
        ("convection_faces", C.c_uint32),
        ("radiation_faces", C.c_uint32),
        ("neumann_faces", C.c_uint32),
        ("reserved", C.c_uint32),
        ("convection_coefficient", C.c_double),
        ("convection_temperature_infinity", C.c_double),
        ("emissivity", C.c_double),
        ("radiation_temperature_infinity", C.c_double),
        ("neumann_flux", C.c_double * 6),
    ]


class SolidLiquid(C.Structure):
    """mpdg_solid_liquid: liquid / solid density, specific heat and conductivity, liquidus and
    solidus temperature, transition type (0 mushy zone, 1 sharp)."""

    _fields_ = [
        ("liquid_density", C.c_double),
        ("liquid_specific_heat", C.c_double),
        ("liquid_conductivity", C.c_double),
        ("solid_density", C.c_double),
        ("solid_specific_heat", C.c_double),
        ("solid_conductivity", C.c_double),
        ("liquidus_temperature", C.c_double),
        ("solidus_temperature", C.c_double),
        ("sharp", C.c_int32),
        ("reserved", C.c_int32),
        ("latent_heat", C.c_double),
        ("capacity_type", C.c_int32),
        ("reserved2", C.c_int32),
    ]


class SolverParams(C.Structure):
    _fields_ = [
        ("solver", C.c_int32),
        ("precond", C.c_int32),
        ("max_it", C.c_int32),
        ("restart", C.c_int32),
        ("abs_tol", C.c_double),
        ("rel_tol", C.c_double),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("status", C.c_int32),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
        ("history", C.c_void_p),
        ("history_capacity", C.c_int32),
        ("inner_iterations", C.c_int32),
    ]


class MixedParams(C.Structure):
    _fields_ = [
        ("outer_rel_tol", C.c_double),
        ("inner_rel_tol", C.c_double),
        ("max_outer", C.c_int32),
        ("max_inner", C.c_int32),
        ("solver", C.c_int32),
        ("restart", C.c_int32),
        ("inexact_last", C.c_int32),
        ("reserved", C.c_int32),
    ]


class AdjointParams(C.Structure):
    _fields_ = [
        ("n_steps", C.c_int32),
        ("checkpoint_every", C.c_int32),
        ("cg_rel_tol", C.c_double),
        ("cg_max_it", C.c_int32),
        ("reserved", C.c_int32),
    ]


class AdjointResult(C.Structure):
    _fields_ = [
        ("objective", C.c_double),
        ("grad_amplitude", C.c_double),
        ("forward_solves", C.c_int32),
        ("adjoint_solves", C.c_int32),
        ("cg_iterations", C.c_int64),
    ]


# (name, argtypes, restype) for every exported entry point
P, D = C.c_void_p, C.c_double
SIGNATURES = [
    ("mpdg_op_create", [C.POINTER(MeshDesc), C.POINTER(OpParams), C.POINTER(C.c_void_p)], C.c_int),
    ("mpdg_op_destroy", [P], C.c_int),
    ("mpdg_op_n_dofs", [P], C.c_int64),
    ("mpdg_op_n_cells", [P], C.c_int64),
    ("mpdg_op_set_stream", [P, P], C.c_int),
    ("mpdg_op_reset_time_increment", [P, D], C.c_int),
    ("mpdg_op_reset_dof_index", [P, C.c_int], C.c_int),
    ("mpdg_op_set_conductivity", [P, P], C.c_int),
    ("mpdg_op_set_heat_bc", [P, C.POINTER(HeatBC)], C.c_int),
    ("mpdg_vec_dot", [P, P, P, P], C.c_int),
    ("mpdg_op_set_supg", [P, C.c_int, D], C.c_int),
    ("mpdg_op_set_reinit", [P, D, D, D, P, P, P], C.c_int),
    ("mpdg_level_set_normal_rhs", [P, P, C.c_int, P, P, P], C.c_int),
    ("mpdg_level_set_curvature_rhs", [P, P, P, P, D, P], C.c_int),
    ("mpdg_op_set_narrow_band", [P, P, D], C.c_int),
    ("mpdg_op_set_wetting", [P, C.c_uint32], C.c_int),
    ("mpdg_op_set_velocity_field", [P, P, P, P], C.c_int),
    ("mpdg_op_distribute_constraints", [P, P, P], C.c_int),
    ("mpdg_vec_alloc", [P, C.POINTER(C.c_void_p)], C.c_int),
    ("mpdg_vec_free", [P], C.c_int),
    ("mpdg_op_set_temperature", [P, P], C.c_int),
    ("mpdg_op_set_inflow_outflow", [P, C.c_uint32, P], C.c_int),
    ("mpdg_op_n_inflow", [P], C.c_int64),
    ("mpdg_op_set_inflow_outflow_pre_post", [P, C.c_int], C.c_int),
    ("mpdg_op_distribute_inflow", [P, P], C.c_int),
    ("mpdg_op_set_solidification", [P, C.POINTER(SolidLiquid)], C.c_int),
    ("mpdg_op_set_old_temperature", [P, P], C.c_int),
    ("mpdg_op_vmult", [P, P, P], C.c_int),
    ("mpdg_op_vmult_f32", [P, P, P], C.c_int),
    ("mpdg_op_vmult_host", [P, P, P], C.c_int),
    ("mpdg_op_vmult_add", [P, P, P, D], C.c_int),
    ("mpdg_op_residual", [P, P, P, P], C.c_int),
    ("mpdg_op_compute_inverse_diagonal", [P, P], C.c_int),
    ("mpdg_op_compute_inverse_diagonal_f32", [P, P], C.c_int),
    ("mpdg_op_create_rhs", [P, P, P, P, P], C.c_int),
    ("mpdg_solve", [P, P, P, C.POINTER(SolverParams), C.POINTER(SolveInfo)], C.c_int),
    ("mpdg_solve_f32", [P, P, P, C.POINTER(SolverParams), C.POINTER(SolveInfo)], C.c_int),
    ("mpdg_solve_mixed", [P, P, P, C.POINTER(MixedParams), C.POINTER(SolveInfo)], C.c_int),
    ("mpdg_op_device_errors", [P], C.c_int),
    ("mpdg_op_test_set_wait_limit", [P, C.c_uint], C.c_int),
    ("mpdg_op_set_cg_variant", [P, C.c_int], C.c_int),
    ("mpdg_op_test_set_ticket", [P, C.c_uint], C.c_int),
    ("mpdg_op_n_bricks", [P], C.c_int),
    ("mpdg_adjoint_heat", [P, P, P, D, P, C.POINTER(AdjointParams), P, C.POINTER(AdjointResult)], C.c_int),
    ("mpdg_heat_forward", [P, P, P, D, C.POINTER(AdjointParams), P], C.c_int),
    ("mpdg_heat_cell_stiffness_form", [P, P, P, P], C.c_int),
    ("mpdg_op_create_rhs_and_apply_dirichlet", [P, P, P, P, P, P, C.c_int], C.c_int),
    ("mpdg_vec_fill", [P, P, D], C.c_int),
    ("mpdg_vec_axpby", [P, P, D, P, D], C.c_int),
    ("mpdg_vec_norm", [P, P, C.POINTER(D)], C.c_int),
    ("mpdg_heat_vmult_noalloc", [P, P, P, P, P, P], C.c_int),
    ("mpdg_heat_vmult_noalloc_errors", [P, C.POINTER(C.c_int)], C.c_int),
    ("mpdg_last_error", [], C.c_char_p),
]
OPTIONAL = []

_lib = None


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m meltpooldg_b200.build`")
        L = C.CDLL(LIB_PATH)
        for required, table in ((True, SIGNATURES), (False, OPTIONAL)):
            for name, args, res in table:
                if not hasattr(L, name):
                    if required:
                        raise ImportError(f"{LIB_PATH} does not export {name}")
                    continue
                f = getattr(L, name)
                f.argtypes = args
                f.restype = res
        _lib = L
    return _lib


class MpdgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[mpdg error {code}] {msg}")
        self.code = code


class NoConvergence(MpdgError):
    """Raised like dealii::SolverControl::NoConvergence (linear_solver.hpp:124-129)."""


class ZeroTimeIncrement(MpdgError):
    """Raised like ExcZeroTimeIncrement (include/meltpooldg/core/exceptions.hpp:6)."""


def check(rc: int) -> None:
    if rc == MPDG_OK:
        return
    msg = lib().mpdg_last_error().decode()
    if rc == MPDG_ERR_NOT_CONVERGED:
        raise NoConvergence(rc, msg)
    if rc == MPDG_ERR_ZERO_DT:
        raise ZeroTimeIncrement(rc, msg)
    raise MpdgError(rc, msg)
