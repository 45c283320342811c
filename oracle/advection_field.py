"""Advection-diffusion operator with a velocity given as a finite-element DoF vector -- CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU kernels, never by the
product path.

Restates source/level_set/advection_diffusion_operator.cpp when the velocity is a DoF vector
(advection_velocity, not advection_velocity_function): the velocity is read per cell with
read_dof_values_plain (:461-466) and evaluated at the quadrature points (:475-479) -- here three
FE_Q(k) components on the same lattice as the advected field --, then
  tangent (:448-495):    val = u/dt + theta v.grad u,  grad = theta eps grad u;
  create_rhs (:274-358): val = u_old/dt - (1-theta) v.grad u_old, grad = -(1-theta) eps grad u_old;
  diagonal (:399-446):   the tangent's diagonal, inverted with 1e-14 max(1, |d|_inf).
Per cell with QGauss(k+1), vectorised over the cells with numpy.  Pinned by tests/
test_oracle_advection_field.py: a field sampled from an affine velocity (represented exactly by
FE_Q(k)) reproduces the C++ oracle's affine operator.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from oracle.oracle import Mesh
from oracle.supg import _cells, _dof_index, tables


def _setup(mesh: Mesh, cmask, field: Sequence[np.ndarray]):
    qp, qw, B, G, _ = tables(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    idx = _dof_index(mesh, cx, cy, cz)
    ev = lambda Z, Y, X, f: np.einsum("al,bj,ci,xlji->xabc", Z, Y, X, f)  # noqa: E731
    v = [ev(B, B, B, np.asarray(c, dtype=np.float64)[idx]) for c in field]  # plain reads
    W = h[0] * h[1] * h[2] * np.einsum("a,b,c->abc", qw, qw, qw)[None]
    return B, G, h, idx, free, v, W, ev


def _integrate(mesh, B, G, h, idx, free, val, flux):
    te = lambda Z, Y, X, F: np.einsum("al,bj,ci,xabc->xlji", Z, Y, X, F)  # noqa: E731
    loc = te(B, B, B, val) + te(B, B, G, flux[0]) / h[0] + te(B, G, B, flux[1]) / h[1] + te(G, B, B, flux[2]) / h[2]
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], loc[keep])
    return out


def _form(mesh: Mesh, cmask, field, inv_dt, th_adv, th_dif, u, plain: bool):
    B, G, h, idx, free, v, W, ev = _setup(mesh, cmask, field)
    uc = (np.asarray(u, dtype=np.float64) if plain else np.where(free, u, 0.0))[idx]
    uq = ev(B, B, B, uc)
    g = [ev(B, B, G, uc) / h[0], ev(B, G, B, uc) / h[1], ev(G, B, B, uc) / h[2]]
    val = W * (inv_dt * uq + th_adv * (v[0] * g[0] + v[1] * g[1] + v[2] * g[2]))
    return _integrate(mesh, B, G, h, idx, free, val, [W * th_dif * c for c in g])


def tangent_apply(mesh: Mesh, cmask: Optional[np.ndarray], field, dt, theta, eps, u) -> np.ndarray:
    """vmult: u with Dirichlet entries 0, constrained rows 0."""
    return _form(mesh, cmask, field, 1.0 / dt, theta, theta * eps, u, plain=False)


def create_rhs(mesh: Mesh, cmask: Optional[np.ndarray], field, dt, theta, eps, u_old) -> np.ndarray:
    """create_rhs: plain reads, accumulate form (returned), constrained rows 0."""
    return _form(mesh, cmask, field, 1.0 / dt, theta - 1.0, (theta - 1.0) * eps, u_old, plain=True)


def diagonal(mesh: Mesh, cmask: Optional[np.ndarray], field, dt, theta, eps) -> np.ndarray:
    """Diagonal of the tangent (constrained rows 1)."""
    B, G, h, idx, free, v, W, ev = _setup(mesh, cmask, field)
    o = lambda Z, Y, X: np.einsum("al,bj,ci->abclji", Z, Y, X)[None]  # noqa: E731
    phi = o(B, B, B)
    dphi = [o(B, B, G) / h[0], o(B, G, B) / h[1], o(G, B, B) / h[2]]
    e = lambda a: a[..., None, None, None]  # noqa: E731
    vg = sum(e(v[d]) * dphi[d] for d in range(3))
    pp = sum(dp * dp for dp in dphi)
    term = e(W) * (phi * phi / dt + theta * vg * phi + theta * eps * pp)
    loc = term.sum(axis=(1, 2, 3))
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], loc[keep])
    if cmask is not None:
        out[np.asarray(cmask) != 0] = 1.0
    return out


def inverse_diagonal(mesh: Mesh, cmask, field, dt, theta, eps) -> np.ndarray:
    d = diagonal(mesh, cmask, field, dt, theta, eps)
    thr = 1e-14 * max(1.0, np.max(np.abs(d)))
    return np.where(np.abs(d) > thr, 1.0 / np.where(d != 0, d, 1.0), 1.0)
