"""Adjoint of the transient implicit-Euler heat problem over the C ABI.

Forward problem on a HeatDiffuseOperator with per-cell conductivity k = exp(z):

    (rho c_p M / dt + K(k)) T_n = rho c_p M T_{n-1} / dt + A M qhat_n ,   n = 1..N,  T_0 = 0,

objective J = 1/2 sum_n |T_n - T*_n|^2 over the free DoFs.  ``objective_and_gradient`` returns J,
dJ/dz (one entry per cell) and dJ/dA from one forward sweep (states checkpointed every
``checkpoint_every`` steps), then a backward sweep that recomputes each segment from its checkpoint
and solves the transposed (symmetric) systems.  The reference has no adjoint; its forward operator
is the heat tangent of source/heat/heat_diffuse_operator.cpp:1029-1079, the source term is read like
heat_source in create_rhs (heat_diffuse_operator.cpp:445-447,493-495).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib as L
from ._lib import check, lib
from .operators import HeatDiffuseOperator


@dataclass
class AdjointStats:
    forward_solves: int
    adjoint_solves: int
    cg_iterations: int


class TransientHeatAdjoint:
    def __init__(self, op: HeatDiffuseOperator, n_steps: int, checkpoint_every: int = 5,
                 cg_rel_tol: float = 1e-12, cg_max_it: int = 10000):
        self.op = op
        self.p = L.AdjointParams()
        self.p.n_steps, self.p.checkpoint_every = int(n_steps), int(checkpoint_every)
        self.p.cg_rel_tol, self.p.cg_max_it = float(cg_rel_tol), int(cg_max_it)

    def forward(self, log_k, qhat, amplitude: float, T_out) -> None:
        """States T_1..T_N into T_out (N x n_dofs, float64 CUDA tensor)."""
        cells, states = self.op.mesh.ncells, self.p.n_steps * self.op.mesh.ndofs
        check(lib().mpdg_heat_forward(self.op._h, self.op._v(log_k, n=cells), self.op._v(qhat, n=states),
                                      float(amplitude), C.byref(self.p), self.op._v(T_out, n=states)))

    def objective_and_gradient(self, log_k, qhat, amplitude: float, target, grad_log_k=None):
        """(J, dJ/dA, stats); fills grad_log_k (n_cells float64 CUDA tensor) unless it is None."""
        res = L.AdjointResult()
        cells, states = self.op.mesh.ncells, self.p.n_steps * self.op.mesh.ndofs
        check(lib().mpdg_adjoint_heat(self.op._h, self.op._v(log_k, n=cells), self.op._v(qhat, n=states),
                                      float(amplitude), self.op._v(target, n=states), C.byref(self.p),
                                      self.op._v(grad_log_k, n=cells), C.byref(res)))
        return res.objective, res.grad_amplitude, AdjointStats(res.forward_solves, res.adjoint_solves,
                                                               res.cg_iterations)


def cell_stiffness_form(op: HeatDiffuseOperator, lam, T, form) -> None:
    """form_c = lam_c^T K_c T_c (unit conductivity) for every cell."""
    check(lib().mpdg_heat_cell_stiffness_form(op._h, op._v(lam), op._v(T), op._v(form, n=op.mesh.ncells)))
