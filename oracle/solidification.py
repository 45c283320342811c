"""Heat operator with temperature-dependent material (solid / liquid phases) -- CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU solidification kernels,
never by the product path.

Restates source/heat/heat_diffuse_operator.cpp for do_solidification with MaterialTypes::liquid_solid
and no latent heat:
* material (include/meltpooldg/core/material.templates.hpp:296-360, :540-620, :748-765;
  include/meltpooldg/level_set/level_set_tools.hpp:66-89): solid fraction
  f_s = clamp((T_liquidus - T) / (T_liquidus - T_solidus), 0, 1) (mushy zone) or T < T_solidus
  (sharp); property v_l + (v_s - v_l)(3 f_s^2 - 2 f_s^3), exactly v_l / v_s at f_s = 0 / 1; its
  temperature derivative -(v_s - v_l)(6 f_s - 6 f_s^2) / (T_liquidus - T_solidus), 0 at f_s = 0, 1;
* tangent (:1029-1050): (rho c_p / dt + d(rho c_p)/dT (T - T_old) / dt) u tested with phi,
  k grad u + dk/dT grad T u tested with grad phi; u with Dirichlet entries 0, T and T_old plain;
* residual part of create_rhs (:485-527): -rho c_p(T) (T - T_old) / dt phi - k(T) grad T . grad phi.
Per cell with QGauss(k+1), vectorised over the cells with numpy.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from oracle.oracle import Mesh
from oracle.supg import _cells, _dof_index, tables


@dataclass
class SolidLiquid:
    liquid: tuple = (1.0, 1.0, 1.0)  # density, specific heat capacity, conductivity
    solid: tuple = (1.0, 1.0, 1.0)
    liquidus_temperature: float = 1.0
    solidus_temperature: float = 0.0
    sharp: bool = False


def material(m: SolidLiquid, T: np.ndarray):
    """rho c_p, k and their temperature derivatives at the temperatures T."""
    T = np.asarray(T, dtype=np.float64)
    if m.sharp:
        fs = np.where(T < m.solidus_temperature, 1.0, 0.0)
        inv = 0.0
    else:
        inv = 1.0 / (m.liquidus_temperature - m.solidus_temperature)
        fs = np.clip((m.liquidus_temperature - T) * inv, 0.0, 1.0)
    end = (fs == 0.0) | (fs == 1.0)
    w = (3.0 - 2.0 * fs) * fs * fs
    dw = -inv * (6.0 * fs - 6.0 * fs * fs)

    def pr(vl, vs):
        return np.where(fs == 0.0, vl, np.where(fs == 1.0, vs, vl + (vs - vl) * w))

    def dpr(vl, vs):
        return np.where(end, 0.0, (vs - vl) * dw)

    (rl, cl, kl), (rs, cs, ks) = m.liquid, m.solid
    rho, cp = pr(rl, rs), pr(cl, cs)
    return rho * cp, pr(kl, ks), dpr(rl, rs) * cp + rho * dpr(cl, cs), dpr(kl, ks)


def _fields(mesh: Mesh, cmask, u, T, Told, plain_u: bool):
    qp, qw, B, G, _ = tables(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    idx = _dof_index(mesh, cx, cy, cz)
    ev = lambda Z, Y, X, f: np.einsum("al,bj,ci,xlji->xabc", Z, Y, X, f)  # noqa: E731
    out = {}
    for name, v, plain in (("u", u, plain_u), ("T", T, True), ("To", Told, True)):
        if v is None:
            continue
        vv = np.asarray(v, dtype=np.float64) if plain else np.where(free, v, 0.0)
        c = vv[idx]
        out[name] = ev(B, B, B, c)
        out[name + "_g"] = [ev(B, B, G, c) / h[0], ev(B, G, B, c) / h[1], ev(G, B, B, c) / h[2]]
    W = h[0] * h[1] * h[2] * np.einsum("a,b,c->abc", qw, qw, qw)[None]
    return out, W, B, G, h, idx, free


def _test(mesh, val, grad, B, G, h, idx, free):
    te = lambda Z, Y, X, F: np.einsum("al,bj,ci,xabc->xlji", Z, Y, X, F)  # noqa: E731
    loc = te(B, B, B, val) + te(B, B, G, grad[0]) / h[0] + te(B, G, B, grad[1]) / h[1] + te(G, B, B, grad[2]) / h[2]
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], loc[keep])
    return out


def tangent_apply(mesh: Mesh, cmask, m: SolidLiquid, dt: float, T, Told, u) -> np.ndarray:
    f, W, B, G, h, idx, free = _fields(mesh, cmask, u, T, Told, plain_u=False)
    rc, k, drc, dk = material(m, f["T"])
    val = W * (rc + drc * (f["T"] - f["To"])) / dt * f["u"]
    grad = [W * (k * f["u_g"][d] + dk * f["T_g"][d] * f["u"]) for d in range(3)]
    return _test(mesh, val, grad, B, G, h, idx, free)


def residual(mesh: Mesh, cmask, m: SolidLiquid, dt: float, T, Told) -> np.ndarray:
    f, W, B, G, h, idx, free = _fields(mesh, cmask, None, T, Told, plain_u=True)
    rc, k, _, _ = material(m, f["T"])
    val = -W * rc * (f["T"] - f["To"]) / dt
    grad = [-W * k * f["T_g"][d] for d in range(3)]
    return _test(mesh, val, grad, B, G, h, idx, free)


def diagonal(mesh: Mesh, cmask, m: SolidLiquid, dt: float, T, Told) -> np.ndarray:
    """Diagonal of the tangent (0 on constrained rows)."""
    qp, qw, B, G, _ = tables(mesh.degree)
    f, W, _, _, h, idx, free = _fields(mesh, cmask, None, T, Told, plain_u=True)
    rc, k, drc, dk = material(m, f["T"])
    o = lambda Z, Y, X: np.einsum("al,bj,ci->abclji", Z, Y, X)  # noqa: E731
    phi = o(B, B, B)[None]
    dphi = [o(B, B, G)[None] / h[0], o(B, G, B)[None] / h[1], o(G, B, B)[None] / h[2]]
    e = lambda a: a[..., None, None, None]  # noqa: E731
    cm = e(W * (rc + drc * (f["T"] - f["To"])) / dt)
    term = cm * phi * phi + e(W * k) * sum(dp * dp for dp in dphi)
    term = term + e(W * dk) * sum(e(f["T_g"][d]) * dphi[d] for d in range(3)) * phi
    loc = term.sum(axis=(1, 2, 3))
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], loc[keep])
    return out
