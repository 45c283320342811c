"""SUPG streamline stabilisation of the advection-diffusion operator -- CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU SUPG terms, never by the
product path.

Restates source/level_set/advection_diffusion_operator.cpp for ConvectionStabilizationType::SUPG:
* tangent (:455-457, :483-490): the gradient test function gets tau_c v times the strong residual
  s = u/dt + theta v.grad u - theta eps lap u (the value part is submitted before SUPG changes it);
* rhs (:322-345): the same with theta replaced by theta - 1, plain reads of u_old;
* stabilisation parameter (:497-533): tau_c = (coefficient < 0 ? 1 / max_q |v(x_q)| (0 when below
  1e-6) : coefficient) times the cell size, the cell diameter / sqrt(dim)
  (source/core/scratch_data.cpp:262-277).
Per cell with QGauss(k+1); the second derivatives of the 1-D basis come from differentiating the
Lagrange polynomials on the Gauss-Lobatto nodes twice.  Vectorised over all cells with numpy.

The velocity is the affine field vel (12 coefficients, v = vel[0:3] + G x) or, when `field` is
given, a DoF vector: three FE_Q(k) components on the lattice read plainly per cell and evaluated at
the Gauss points (the reference's advection_velocity, advection_diffusion_operator.cpp:461-466,
:475-479), which also gives tau_c's max_q |v| (:510-520).
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from oracle.oracle import Mesh, basis


def tables(degree: int):
    nodes, qp, qw, B, G = basis(degree)
    n = degree + 1
    H = np.zeros((n, n))
    for i in range(n):
        others = np.delete(nodes, i)
        p = np.poly1d(np.poly(others)) / np.prod(nodes[i] - others)
        H[:, i] = p.deriv(2)(qp)
    return qp, qw, B, G, H


def _cells(mesh: Mesh):
    mx, my, mz = mesh.m
    cz, cy, cx = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
    return cx.ravel(), cy.ravel(), cz.ravel()


def _dof_index(mesh: Mesh, cx, cy, cz):
    K = mesh.degree
    n = K + 1
    nx, ny, _ = mesh.n
    l, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    I = K * cx[:, None, None, None] + i[None]
    J = K * cy[:, None, None, None] + j[None]
    L = K * cz[:, None, None, None] + l[None]
    return I + nx * (J + ny * L)  # (cells, l, j, i)


def _velocity(mesh: Mesh, vel, cx, cy, cz, qp):
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    X = mesh.origin[0] + h[0] * (cx[:, None, None, None] + qp[None, None, None, :])
    Y = mesh.origin[1] + h[1] * (cy[:, None, None, None] + qp[None, None, :, None])
    Z = mesh.origin[2] + h[2] * (cz[:, None, None, None] + qp[None, :, None, None])
    X, Y, Z = np.broadcast_arrays(X, Y, Z)  # (cells, qz, qy, qx)
    return [vel[d] + vel[3 + 3 * d] * X + vel[4 + 3 * d] * Y + vel[5 + 3 * d] * Z for d in range(3)]


def _qvel(mesh: Mesh, vel, field, cx, cy, cz):
    """The velocity at the Gauss points of every cell, (cells, qz, qy, qx) per component."""
    qp, _, B, _, _ = tables(mesh.degree)
    if field is None:
        return _velocity(mesh, vel, cx, cy, cz, qp)
    idx = _dof_index(mesh, cx, cy, cz)
    return [np.einsum("al,bj,ci,xlji->xabc", B, B, B, np.asarray(c, dtype=np.float64)[idx]) for c in field]


def supg_tau(mesh: Mesh, vel: Sequence[float], coefficient: float, field=None) -> np.ndarray:
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    size = np.sqrt(sum(x * x for x in h)) / np.sqrt(3.0)
    cx, cy, cz = _cells(mesh)
    if coefficient >= 0:
        return np.full(cx.size, coefficient * size)
    v = _qvel(mesh, vel, field, cx, cy, cz)
    vmax = np.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2).reshape(cx.size, -1).max(axis=1)
    tau = np.where(vmax >= 1e-6, 1.0 / np.where(vmax > 0, vmax, 1.0), 0.0)
    return tau * size


def supg_apply(mesh: Mesh, cmask: Optional[np.ndarray], vel, coefficient: float, inv_dt: float, th_adv: float,
               th_dif: float, u: np.ndarray, plain: bool = False, field=None) -> np.ndarray:
    """sum_c tau_c int (v.grad phi_i)(u/dt + th_adv v.grad u - th_dif lap u) over the free rows;
    u read with Dirichlet entries as 0 unless plain; v the affine vel or the DoF-vector field."""
    qp, qw, B, G, H = tables(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    det = h[0] * h[1] * h[2]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    idx = _dof_index(mesh, cx, cy, cz)
    uu = np.asarray(u, dtype=np.float64) if plain else np.where(free, u, 0.0)
    uc = uu[idx]
    ev = lambda Z, Y, X, f: np.einsum("al,bj,ci,xlji->xabc", Z, Y, X, f)  # noqa: E731
    uq = ev(B, B, B, uc)
    g = [ev(B, B, G, uc) / h[0], ev(B, G, B, uc) / h[1], ev(G, B, B, uc) / h[2]]
    lap = ev(B, B, H, uc) / h[0] ** 2 + ev(B, H, B, uc) / h[1] ** 2 + ev(H, B, B, uc) / h[2] ** 2
    v = _qvel(mesh, vel, field, cx, cy, cz)
    s = inv_dt * uq + th_adv * (v[0] * g[0] + v[1] * g[1] + v[2] * g[2]) - th_dif * lap
    W = det * np.einsum("a,b,c->abc", qw, qw, qw)
    tau = supg_tau(mesh, vel, coefficient, field)[:, None, None, None]
    f = [tau * W[None] * v[d] * s for d in range(3)]
    te = lambda Z, Y, X, F: np.einsum("al,bj,ci,xabc->xlji", Z, Y, X, F)  # noqa: E731
    loc = te(B, B, G, f[0]) / h[0] + te(B, G, B, f[1]) / h[1] + te(G, B, B, f[2]) / h[2]
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], loc[keep])
    return out


def supg_diagonal(mesh: Mesh, cmask: Optional[np.ndarray], vel, coefficient: float, inv_dt: float,
                  th_adv: float, th_dif: float, field=None) -> np.ndarray:
    """Diagonal of supg_apply's operator (0 on constrained rows)."""
    qp, qw, B, G, H = tables(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    det = h[0] * h[1] * h[2]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    idx = _dof_index(mesh, cx, cy, cz)
    o = lambda Z, Y, X: np.einsum("al,bj,ci->abclji", Z, Y, X)  # noqa: E731  (q, dof) tables
    phi = o(B, B, B)
    dphi = [o(B, B, G) / h[0], o(B, G, B) / h[1], o(G, B, B) / h[2]]
    lap = o(B, B, H) / h[0] ** 2 + o(B, H, B) / h[1] ** 2 + o(H, B, B) / h[2] ** 2
    v = _qvel(mesh, vel, field, cx, cy, cz)  # (cells, a, b, c)
    vg = sum(v[d][..., None, None, None] * dphi[d][None] for d in range(3))  # (cells, abc, lji)
    W = det * np.einsum("a,b,c->abc", qw, qw, qw)[None, :, :, :, None, None, None]
    tau = supg_tau(mesh, vel, coefficient, field)[:, None, None, None]
    loc = tau * np.sum(W * vg * (inv_dt * phi[None] + th_adv * vg - th_dif * lap[None]), axis=(1, 2, 3))
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], loc[keep])
    return out
