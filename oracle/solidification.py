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
* residual part of create_rhs (:485-527): -rho c_p(T) (T - T_old) / dt phi - k(T) grad T . grad phi;
* latent heat of fusion L > 0 (include/meltpooldg/core/material.hpp:654-655): the specific heat gains
  an apparent capacity C(f_s) over the mushy zone and its derivative gains dC/dT
  (material.templates.hpp:561-614; source/heat/apparent_capacity.cpp:157-300), zero at f_s <= 0 and
  f_s >= 1, in one of three shapes, each of integral L over [T_solidus, T_liquidus]:
  "constant" L / dT; "poly4_bell" L (2 / dT) b(1 - 2 f_s) with b(x) = 15/16 (1 - x^2)^2;
  "qlq" (the default) a tent of peak 2 L / dT at the mid temperature, each flank linear with
  quadratic, zero-slope ends of width dT / 6, evaluated at T = T_liquidus - f_s dT.
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
    latent_heat: float = 0.0  # latent heat of fusion per unit mass; > 0 adds the apparent capacity
    capacity_type: str = "qlq"  # "qlq" | "poly4_bell" | "constant"


def _zero_slope_ramp(x, x1, x2, y1, y2, delta):
    """Value and derivative of the ramp from (x1, y1) to (x2, y2) that is flat at both ends: a
    quadratic on [x1, x1 + delta], a line of slope s = (y2 - y1) / (x2 - x1 - delta) in between,
    and a quadratic on [x2 - delta, x2]; value and slope are continuous."""
    s = (y2 - y1) / (x2 - x1 - delta)
    lo, hi = x < x1 + delta, x > x2 - delta
    val = np.where(lo, y1 + 0.5 * s * (x - x1) ** 2 / delta,
                   np.where(hi, y2 - 0.5 * s * (x2 - x) ** 2 / delta, y1 + s * (x - x1 - 0.5 * delta)))
    der = np.where(lo, s * (x - x1) / delta, np.where(hi, s * (x2 - x) / delta, s))
    return val, der


def apparent_capacity(m: SolidLiquid, fs):
    """Apparent specific heat capacity of the latent heat and its temperature derivative at the
    solid fractions fs (0 where fs <= 0 or fs >= 1 and where latent_heat is 0)."""
    fs = np.asarray(fs, dtype=np.float64)
    if m.latent_heat <= 0.0:
        return np.zeros_like(fs), np.zeros_like(fs)
    Ts, Tl, L = m.solidus_temperature, m.liquidus_temperature, m.latent_heat
    dT = Tl - Ts
    inside = (fs > 0.0) & (fs < 1.0)
    if m.capacity_type == "constant":
        c, dc = np.full_like(fs, L / dT), np.zeros_like(fs)
    elif m.capacity_type == "poly4_bell":
        r = 2.0 / dT
        x = 1.0 - 2.0 * fs
        c = L * r * (15.0 / 16.0) * (1.0 - x * x) ** 2
        dc = L * r * r * (15.0 / 4.0) * (x * x - 1.0) * x
    elif m.capacity_type == "qlq":
        T = Tl - fs * dT
        Tp, peak, delta = 0.5 * (Ts + Tl), 2.0 * L / dT, dT / 6.0
        up, dup = _zero_slope_ramp(T, Ts, Tp, 0.0, peak, delta)
        down, ddown = _zero_slope_ramp(T, Tp, Tl, peak, 0.0, delta)
        c, dc = np.where(T <= Tp, up, down), np.where(T <= Tp, dup, ddown)
    else:
        raise ValueError(f"unknown apparent capacity type {m.capacity_type}")
    return np.where(inside, c, 0.0), np.where(inside, dc, 0.0)


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
    ca, dca = apparent_capacity(m, fs)
    rho, cp, dcp = pr(rl, rs), pr(cl, cs) + ca, dpr(cl, cs) + dca
    return rho * cp, pr(kl, ks), dpr(rl, rs) * cp + rho * dcp, dpr(kl, ks)


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
