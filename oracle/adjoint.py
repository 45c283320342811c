"""CPU ORACLE (test infrastructure only) of the transient heat adjoint.

Same problem as the product's adjoint entry point, restated with the oracle operator:
    (rho c_p M / dt + K(exp z)) T_n = rho c_p M T_{n-1} / dt + A M qhat_n,  T_0 = 0,
    J = 1/2 sum_n |T_n - T*_n|^2 (free DoFs).
The forward right-hand side is the heat create_rhs (source/heat/heat_diffuse_operator.cpp:445-447,
493-495) with T = 0, T_old = T_{n-1}, q = A qhat_n; the tangent is heat_diffuse_operator.cpp:1029-1079.
The gradient is assembled from the oracle's per-cell stiffness forms (no checkpointing: every state
is kept), so it checks the product's checkpoint / recompute logic as well as its kernels.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def _op(mesh, cmask, rho_cp, dt, log_k):
    return O.Operator(mesh, "heat", cmask=cmask, rho_cp=rho_cp, dt=dt, k=1.0, k_cell=np.exp(log_k))


def forward(mesh, cmask, rho_cp, dt, log_k, qhat, amplitude, rel_tol=1e-13):
    op = _op(mesh, cmask, rho_cp, dt, log_k)
    inv = op.inverse_diagonal()
    T = np.zeros(mesh.ndofs)
    out = []
    for s in range(qhat.shape[0]):
        rhs = np.zeros(mesh.ndofs)
        op.create_rhs(rhs, np.zeros(mesh.ndofs), T, amplitude * qhat[s])
        x = T.copy()
        O.solve(op, x, rhs, "cg", inv, rel_tol=rel_tol, abs_tol=0.0)
        T = x
        out.append(T.copy())
    return np.array(out)


def objective(mesh, cmask, rho_cp, dt, log_k, qhat, amplitude, target, rel_tol=1e-13):
    T = forward(mesh, cmask, rho_cp, dt, log_k, qhat, amplitude, rel_tol)
    free = np.ones(mesh.ndofs) if cmask is None else (np.asarray(cmask) == 0).astype(float)
    return 0.5 * float(np.sum(((T - target) * free) ** 2))


def gradient(mesh, cmask, rho_cp, dt, log_k, qhat, amplitude, target, rel_tol=1e-13):
    """(J, dJ/dz per cell, dJ/dA) by the discrete adjoint."""
    op = _op(mesh, cmask, rho_cp, dt, log_k)
    mass = O.Operator(mesh, "heat", cmask=cmask, rho_cp=rho_cp, dt=dt, k=0.0)  # rho c_p M / dt
    inv = op.inverse_diagonal()
    T = forward(mesh, cmask, rho_cp, dt, log_k, qhat, amplitude, rel_tol)
    free = np.ones(mesh.ndofs) if cmask is None else (np.asarray(cmask) == 0).astype(float)
    J = 0.5 * float(np.sum(((T - target) * free) ** 2))
    k = np.exp(log_k)
    gz = np.zeros(mesh.ncells)
    gA = 0.0
    lam_next = np.zeros(mesh.ndofs)
    for s in range(qhat.shape[0] - 1, -1, -1):
        rhs = mass.vmult(lam_next) + (T[s] - target[s]) * free
        lam = lam_next.copy()
        O.solve(op, lam, rhs, "cg", inv, rel_tol=rel_tol, abs_tol=0.0)
        gz -= k * op.cell_stiffness_form(lam, T[s])
        Mq = np.zeros(mesh.ndofs)  # M qhat with plain reads: create_rhs with rho_cp = 0
        op.with_(rho_cp=0.0).create_rhs(Mq, np.zeros(mesh.ndofs), None, qhat[s])
        gA += float(lam @ Mq)
        lam_next = lam
    return J, gz, gA
