"""Host-side mirror of MeltPoolDG's matrix-free operator / solver interface over the C ABI.

Names and semantics follow the reference:
  * OperatorMatrixFree (include/meltpooldg/core/operator_base.hpp:189-283): vmult, create_rhs,
    compute_inverse_diagonal_from_matrixfree, reset_time_increment, reset_dof_index, pre/post/reinit
  * HeatDiffuseOperator  -> HeatDiffuseMultiPhaseOperator (source/heat/heat_diffuse_operator.cpp)
  * AdvectionDiffusionOperator (source/level_set/advection_diffusion_operator.cpp)
  * LinearSolverData / LinearSolver.solve (include/meltpooldg/linear_algebra/linear_solver_data.hpp,
    linear_solver.hpp:26-134): ReductionControl(max_iterations, abs_tolerance, rel_tolerance);
    non-convergence raises NoConvergence.
Vectors are torch tensors on the CUDA device (torch only provides device memory); their entries
are in lexicographic lattice order.  Every computation runs in libmpdg_b200.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import MpdgError, NoConvergence, ZeroTimeIncrement, check, lib  # noqa: F401


@dataclass
class Mesh:
    """Structured box of cells[0] x cells[1] x cells[2] axis-aligned hexahedra with FE_Q(degree)."""

    degree: int
    cells: Sequence[int]
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    length: Sequence[float] = (1.0, 1.0, 1.0)
    dirichlet_faces: int = 0
    dirichlet_mask: Optional[np.ndarray] = None  # uint8 per DoF (nonzero = constrained)

    @property
    def n(self):
        return tuple(self.degree * c + 1 for c in self.cells)

    @property
    def ndofs(self) -> int:
        a, b, c = self.n
        return a * b * c

    @property
    def ncells(self) -> int:
        return int(np.prod(self.cells))

    def _desc(self) -> L.MeshDesc:
        d = L.MeshDesc()
        d.degree = int(self.degree)
        for i in range(3):
            d.cells[i] = int(self.cells[i])
            d.origin[i] = float(self.origin[i])
            d.length[i] = float(self.length[i])
        d.dirichlet_faces = int(self.dirichlet_faces)
        if self.dirichlet_mask is not None:
            self._mask = np.ascontiguousarray(self.dirichlet_mask, dtype=np.uint8)
            if self._mask.size != self.ndofs:
                raise ValueError("dirichlet_mask must have one entry per DoF")
            d.dirichlet_mask = self._mask.ctypes.data
        else:
            d.dirichlet_mask = None
        return d


def _ptr(t, n: Optional[int] = None, dtype=None) -> Optional[int]:
    """Device address of a contiguous CUDA tensor, checked to hold at least n entries of dtype
    (either check skipped when None), so that no kernel is handed a buffer it would overrun."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("vectors must be contiguous CUDA tensors")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"expected a {dtype} vector, got {t.dtype}")
    if n is not None and t.numel() < n:
        raise ValueError(f"vector of {t.numel()} entries where {n} are needed")
    return t.data_ptr()


class OperatorMatrixFree:
    """Common handle logic; see include/meltpooldg/core/operator_base.hpp:189-283."""

    def __init__(self, mesh: Mesh, params: L.OpParams, stream=None):
        self.mesh = mesh
        self._params = params
        h = C.c_void_p()
        check(lib().mpdg_op_create(C.byref(mesh._desc()), C.byref(params), C.byref(h)))
        self._h = h
        if stream is not None:
            check(lib().mpdg_op_set_stream(self._h, C.c_void_p(stream)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().mpdg_op_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self._h = None

    def _v(self, t, dtype=None, n: Optional[int] = None) -> Optional[int]:
        """_ptr of a vector of this operator: n_dofs entries (or n) of dtype (float64 by default)."""
        import torch

        return _ptr(t, self.mesh.ndofs if n is None else n, torch.float64 if dtype is None else dtype)

    def set_stream(self, stream_handle: int) -> None:
        check(lib().mpdg_op_set_stream(self._h, C.c_void_p(stream_handle)))

    @property
    def n_dofs(self) -> int:
        return lib().mpdg_op_n_dofs(self._h)

    # OperatorBase
    def reset_time_increment(self, dt: float) -> None:
        check(lib().mpdg_op_reset_time_increment(self._h, float(dt)))

    def reset_dof_index(self, with_dirichlet: bool) -> None:
        check(lib().mpdg_op_reset_dof_index(self._h, 1 if with_dirichlet else 0))

    def pre(self) -> None:  # ghost updates: nothing to do on one device
        pass

    def post(self) -> None:
        pass

    def reinit(self) -> None:
        pass

    # OperatorMatrixFree
    def vmult(self, dst, src) -> None:
        import torch

        if src.dtype == torch.float64:
            check(lib().mpdg_op_vmult(self._h, self._v(dst), self._v(src)))
        elif src.dtype == torch.float32:
            check(lib().mpdg_op_vmult_f32(self._h, self._v(dst, torch.float32), self._v(src, torch.float32)))
        else:
            raise TypeError("vmult needs float64 or float32 vectors")

    def vmult_add(self, dst, src, scale: float = 1.0) -> None:
        check(lib().mpdg_op_vmult_add(self._h, self._v(dst), self._v(src), float(scale)))

    def residual(self, r, b, x) -> None:
        check(lib().mpdg_op_residual(self._h, self._v(r), self._v(b), self._v(x)))

    def vmult_host(self, dst: np.ndarray, src: np.ndarray) -> None:
        for a in (dst, src):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.size < self.mesh.ndofs:
                raise ValueError(f"host vectors must be C-contiguous float64 arrays of {self.mesh.ndofs} entries")
        check(lib().mpdg_op_vmult_host(self._h, dst.ctypes.data, src.ctypes.data))

    def compute_inverse_diagonal_from_matrixfree(self, diag) -> None:
        import torch

        if diag.dtype == torch.float64:
            check(lib().mpdg_op_compute_inverse_diagonal(self._h, self._v(diag)))
        else:
            check(lib().mpdg_op_compute_inverse_diagonal_f32(self._h, self._v(diag, torch.float32)))

    def create_rhs(self, dst, a, b=None, c=None) -> None:
        check(lib().mpdg_op_create_rhs(self._h, self._v(dst), self._v(a), self._v(b), self._v(c)))

    def create_rhs_and_apply_dirichlet(self, rhs, a, dirichlet_values, b=None, c=None, zero_out: bool = True) -> None:
        """create_rhs_and_apply_dirichlet_matrixfree (utilities_matrixfree.hpp:33-100): rhs (=|+=)
        -A x_D + create_rhs(a, b, c) without the Dirichlet constraints, then constrained rows 0;
        x_D = dirichlet_values on constrained DoFs, 0 elsewhere."""
        check(lib().mpdg_op_create_rhs_and_apply_dirichlet(self._h, self._v(rhs), self._v(a), self._v(b), self._v(c),
                                                          self._v(dirichlet_values), 1 if zero_out else 0))

    def level_set_normal_rhs(self, psi, nx, ny, nz, normalized: bool = False) -> None:
        """NormalVectorOperator::create_rhs on this operator's lattice: n_d += int (grad psi)_d phi."""
        check(lib().mpdg_level_set_normal_rhs(self._h, self._v(psi), 1 if normalized else 0, self._v(nx), self._v(ny),
                                               self._v(nz)))

    def level_set_curvature_rhs(self, dst, nx, ny, nz, normal_tolerance: float) -> None:
        """CurvatureOperator::create_rhs on this operator's lattice: dst = -int div(n) phi."""
        check(lib().mpdg_level_set_curvature_rhs(self._h, self._v(nx), self._v(ny), self._v(nz),
                                                 float(normal_tolerance), self._v(dst)))

    def device_errors(self) -> int:
        return lib().mpdg_op_device_errors(self._h)


class HeatDiffuseOperator(OperatorMatrixFree):
    """(rho c_p/dt) M + div(k grad) -- HeatDiffuseMultiPhaseOperator, single phase, no velocity."""

    def __init__(self, mesh: Mesh, rho_cp: float = 1.0, dt: float = 1.0, conductivity: float = 1.0,
                 conductivity_cells: Optional[np.ndarray] = None, stream=None):
        p = L.OpParams()
        p.kind = L.MPDG_HEAT
        p.rho_cp, p.dt, p.conductivity = float(rho_cp), float(dt), float(conductivity)
        if conductivity_cells is not None:
            self._k = np.ascontiguousarray(conductivity_cells, dtype=np.float64)
            if self._k.size != mesh.ncells:
                raise ValueError("conductivity_cells must have one entry per cell")
            p.conductivity_cells = self._k.ctypes.data
        super().__init__(mesh, p, stream)

    def set_conductivity(self, k_cells_device) -> None:
        check(lib().mpdg_op_set_conductivity(self._h, self._v(k_cells_device, n=self.mesh.ncells)))

    def set_boundary_conditions(self, convection_faces: int = 0, convection_coefficient: float = 0.0,
                                convection_temperature_infinity: float = 0.0, radiation_faces: int = 0,
                                emissivity: float = 0.0, radiation_temperature_infinity: float = 0.0,
                                neumann_faces: int = 0, neumann_flux=(0.0,) * 6) -> None:
        """HeatData's convection / radiation sections and a constant normal flux g.n per Neumann face
        (face masks: bit 2d = low face of dimension d, bit 2d+1 = high face)."""
        bc = L.HeatBC()
        bc.convection_faces, bc.radiation_faces, bc.neumann_faces = convection_faces, radiation_faces, neumann_faces
        bc.convection_coefficient = float(convection_coefficient)
        bc.convection_temperature_infinity = float(convection_temperature_infinity)
        bc.emissivity = float(emissivity)
        bc.radiation_temperature_infinity = float(radiation_temperature_infinity)
        for i in range(6):
            bc.neumann_flux[i] = float(neumann_flux[i])
        check(lib().mpdg_op_set_heat_bc(self._h, C.byref(bc)))

    def set_narrow_band(self, level_set, threshold: float) -> None:
        """Narrow band of the projection operators (NormalVectorData / CurvatureData::narrow_band):
        integrands masked where |level_set| >= threshold at the Gauss points; level_set is kept by
        reference; threshold <= 0 or level_set None removes the band."""
        self._band_ls = level_set
        ptr = None if level_set is None or threshold <= 0 else self._v(level_set)
        check(lib().mpdg_op_set_narrow_band(self._h, ptr, float(threshold)))

    CAPACITY_TYPES = {"qlq": 0, "quadratic_linear_quadratic": 0, "poly4_bell": 1, "constant": 2}

    def set_solidification(self, liquid=(1.0, 1.0, 1.0), solid=(1.0, 1.0, 1.0), liquidus_temperature: float = 1.0,
                           solidus_temperature: float = 0.0, sharp: bool = False, enabled: bool = True,
                           latent_heat: float = 0.0, capacity_type: str = "qlq") -> None:
        """Temperature-dependent material (MaterialTypes::liquid_solid); liquid and solid are
        (density, specific heat capacity, thermal conductivity); latent_heat > 0 adds the apparent
        capacity of the mushy zone of shape capacity_type ("qlq", the reference's default,
        "poly4_bell" or "constant")."""
        if not enabled:
            check(lib().mpdg_op_set_solidification(self._h, None))
            return
        m = L.SolidLiquid()
        m.liquid_density, m.liquid_specific_heat, m.liquid_conductivity = (float(v) for v in liquid)
        m.solid_density, m.solid_specific_heat, m.solid_conductivity = (float(v) for v in solid)
        m.liquidus_temperature, m.solidus_temperature = float(liquidus_temperature), float(solidus_temperature)
        m.sharp = 1 if sharp else 0
        m.latent_heat = float(latent_heat)
        if capacity_type not in self.CAPACITY_TYPES:
            raise ValueError(f"unknown apparent capacity type {capacity_type}")
        m.capacity_type = self.CAPACITY_TYPES[capacity_type]
        check(lib().mpdg_op_set_solidification(self._h, C.byref(m)))

    def set_old_temperature(self, temperature_old_device) -> None:
        """Old temperature of the solidification tangent (kept by reference)."""
        self._temperature_old = temperature_old_device
        check(lib().mpdg_op_set_old_temperature(self._h, self._v(temperature_old_device)))

    def set_temperature(self, temperature_device) -> None:
        """Linearisation temperature of the radiation tangent (kept by reference, as the reference's
        operator keeps a const reference to its temperature vector)."""
        self._temperature = temperature_device
        check(lib().mpdg_op_set_temperature(self._h, self._v(temperature_device)))

    def set_velocity_field(self, vx, vy, vz) -> None:
        """Convection velocity as a DoF vector (three device vectors on the lattice, kept by
        reference), as the reference heat operator's velocity (heat_diffuse_operator.cpp:448-453,
        1038-1041); constant conductivity and material only; None removes it."""
        self._vfield = (vx, vy, vz)
        if vx is None:
            check(lib().mpdg_op_set_velocity_field(self._h, None, None, None))
        else:
            check(lib().mpdg_op_set_velocity_field(self._h, self._v(vx), self._v(vy), self._v(vz)))


class AdvectionDiffusionOperator(OperatorMatrixFree):
    """M/dt + theta (v.grad + eps K) with an affine velocity v(x) = v0 + G x."""

    def __init__(self, mesh: Mesh, dt: float, theta: float = 1.0, diffusivity: float = 0.0,
                 velocity: Sequence[float] = (0.0,) * 12, stream=None):
        p = L.OpParams()
        p.kind = L.MPDG_ADVDIFF
        p.dt, p.theta, p.diffusivity = float(dt), float(theta), float(diffusivity)
        for i in range(12):
            p.velocity[i] = float(velocity[i])
        super().__init__(mesh, p, stream)

    def set_convection_stabilization(self, type: str = "SUPG", coefficient: float = -1.0) -> None:
        """AdvectionDiffusionData::conv_stab: type "none" or "SUPG"; coefficient < 0 selects
        tau_c = h_c / max |v| over the cell's quadrature points, otherwise tau_c = coefficient h_c."""
        if type not in ("none", "SUPG"):
            raise ValueError("convection stabilization type must be 'none' or 'SUPG'")
        check(lib().mpdg_op_set_supg(self._h, 1 if type == "SUPG" else 0, float(coefficient)))

    def set_velocity_field(self, vx, vy, vz) -> None:
        """Velocity as a DoF vector (three device vectors on the lattice, kept by reference), as the
        reference's advection_velocity; None returns to the affine velocity."""
        self._vfield = (vx, vy, vz)
        if vx is None:
            check(lib().mpdg_op_set_velocity_field(self._h, None, None, None))
        else:
            check(lib().mpdg_op_set_velocity_field(self._h, self._v(vx), self._v(vy), self._v(vz)))

    def set_inflow_outflow_bc(self, faces: int, values) -> int:
        """Inflow/outflow condition on the box faces in `faces` (bit 2d low / 2d+1 high face of dim
        d): AdvectionDiffusionOperation::create_inflow_outflow_constraints and the operator's
        set_inflow_outflow_bc (source/level_set/advection_diffusion_operation.cpp:369-499).  values:
        device vector with the condition's function at every DoF.  Returns the number of inflow
        DoFs; faces == 0 removes the condition."""
        check(lib().mpdg_op_set_inflow_outflow(self._h, int(faces), self._v(values) if faces else None))
        return int(lib().mpdg_op_n_inflow(self._h))

    def set_apply_inflow_outflow_constraints_pre_post_matrix_free(self, enabled: bool) -> None:
        check(lib().mpdg_op_set_inflow_outflow_pre_post(self._h, 1 if enabled else 0))

    def distribute_inflow(self, x) -> None:
        """x = prescribed values on the inflow DoFs (advection_diffusion_operation.cpp:288-296)."""
        check(lib().mpdg_op_distribute_inflow(self._h, self._v(x)))


class OlssonOperator(OperatorMatrixFree):
    """Conservative level-set reinitialisation operator (source/level_set/olsson_CG_operator.cpp):
    M/dt + div(D grad), D = eps_t I + (eps_n - eps_t) n n^T with the unit normal of a normal field."""

    def __init__(self, mesh: Mesh, dt: float, eps_normal: float, eps_tangential: float,
                 normal_tolerance: float = 1e-16, stream=None):
        p = L.OpParams()
        p.kind = L.MPDG_REINIT
        p.dt = float(dt)
        super().__init__(mesh, p, stream)
        self.eps_normal, self.eps_tangential, self.normal_tolerance = eps_normal, eps_tangential, normal_tolerance

    def set_normal(self, nx, ny, nz) -> None:
        """Normal field (three device vectors on the lattice, kept by reference)."""
        self._normal = (nx, ny, nz)
        check(lib().mpdg_op_set_reinit(self._h, float(self.eps_normal), float(self.eps_tangential),
                                       float(self.normal_tolerance), self._v(nx), self._v(ny), self._v(nz)))

    def set_wetting(self, faces: int) -> None:
        """Wetting boundary faces (OlssonOperator's boundary loops, olsson_CG_operator.cpp:550-716):
        box faces by bit, 2d low / 2d+1 high face of dimension d; 0 removes them."""
        check(lib().mpdg_op_set_wetting(self._h, int(faces)))


@dataclass
class LinearSolverData:
    """include/meltpooldg/linear_algebra/linear_solver_data.hpp:37-47 (defaults preserved)."""

    solver_type: str = "GMRES"  # "CG" | "GMRES"
    preconditioner_type: str = "Identity"  # "Identity" | "Diagonal"
    max_iterations: int = 10000
    rel_tolerance: float = 1e-12
    abs_tolerance: float = 1e-20
    restart: int = 30


@dataclass
class SolveStats:
    iterations: int
    initial_residual: float
    final_residual: float
    history: np.ndarray = field(default_factory=lambda: np.zeros(0))
    inner_iterations: int = 0


class LinearSolver:
    """LinearSolver::solve (include/meltpooldg/linear_algebra/linear_solver.hpp:26-134)."""

    @staticmethod
    def _params(data: LinearSolverData) -> L.SolverParams:
        p = L.SolverParams()
        p.solver = L.MPDG_CG if data.solver_type.upper() == "CG" else L.MPDG_GMRES
        p.precond = L.MPDG_PRECOND_JACOBI if data.preconditioner_type in ("Diagonal", "Jacobi") else L.MPDG_PRECOND_IDENTITY
        p.max_it, p.restart = int(data.max_iterations), int(data.restart)
        p.abs_tol, p.rel_tol = float(data.abs_tolerance), float(data.rel_tolerance)
        return p

    @staticmethod
    def solve(op: OperatorMatrixFree, solution, rhs, data: LinearSolverData, history: bool = False) -> SolveStats:
        import torch

        p = LinearSolver._params(data)
        info = L.SolveInfo()
        hist = np.zeros(data.max_iterations + 2) if history else None
        if hist is not None:
            info.history = hist.ctypes.data
            info.history_capacity = hist.size
        if solution.dtype not in (torch.float64, torch.float32):
            raise TypeError("solve needs float64 or float32 vectors")
        fn = lib().mpdg_solve if solution.dtype == torch.float64 else lib().mpdg_solve_f32
        rc = fn(op._h, op._v(solution, solution.dtype), op._v(rhs, solution.dtype), C.byref(p), C.byref(info))
        stats = SolveStats(info.iterations, info.initial_residual, info.final_residual,
                           hist[: info.iterations + 1] if hist is not None else np.zeros(0))
        check(rc)
        return stats

    @staticmethod
    def solve_mixed(op: HeatDiffuseOperator, solution, rhs, outer_rel_tol: float = 1e-8,
                    inner_rel_tol: float = 1e-4, max_outer: int = 50, max_inner: int = 10000,
                    solver: str = "CG", restart: int = 30, inexact_last: bool = False) -> SolveStats:
        p = L.MixedParams()
        p.outer_rel_tol, p.inner_rel_tol = float(outer_rel_tol), float(inner_rel_tol)
        p.inexact_last = 1 if inexact_last else 0
        p.max_outer, p.max_inner = int(max_outer), int(max_inner)
        p.solver = L.MPDG_CG if solver.upper() == "CG" else L.MPDG_GMRES
        p.restart = int(restart)
        info = L.SolveInfo()
        hist = np.zeros(max_outer + 2)
        info.history = hist.ctypes.data
        info.history_capacity = hist.size
        rc = lib().mpdg_solve_mixed(op._h, op._v(solution), op._v(rhs), C.byref(p), C.byref(info))
        stats = SolveStats(info.iterations, info.initial_residual, info.final_residual,
                           hist[: info.iterations + 1], info.inner_iterations)
        check(rc)
        return stats
