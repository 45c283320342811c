"""Boundary-face terms of the heat operator -- CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU face kernels, never by the
product path.

Restates, for whole faces of a structured box mesh (face f: bit 2d = low face of dimension d,
bit 2d+1 = high face):

* the tangent's boundary operation, source/heat/heat_diffuse_operator.cpp:1088-1129 (called from
  vmult's boundary face loop :239-264 and from the diagonal's boundary operation :297-357):
  per Gauss point, (h [convection] + 4 eps sigma T^3 [radiation]) * u, tested with phi;
* the right-hand side's boundary loop, :719-781: per Gauss point
  -[eps sigma (T^4 - T_inf^4) + h (T - T_inf) + g.n], tested with phi (g.n one constant per face
  here; the reference evaluates a Function);
* sigma = 5.670374419e-8 (include/meltpooldg/utilities/physical_constants.hpp:6).

Face quadrature is QGauss(k+1) in both face directions.  FEFaceEvaluation semantics: the tangent
reads u and T with constraints (Dirichlet DoFs as 0, gather_evaluate / read_dof_values), the rhs
reads T plainly (read_dof_values_plain); distribute_local_to_global / integrate_scatter skip
constrained rows.  Every face patch is handled with numpy over all patches of a face at once.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from oracle.oracle import Mesh, basis

SIGMA = 5.670374419e-8


@dataclass
class HeatBC:
    convection_faces: int = 0
    convection_coefficient: float = 0.0
    convection_temperature_infinity: float = 0.0
    radiation_faces: int = 0
    emissivity: float = 0.0
    radiation_temperature_infinity: float = 0.0
    neumann_faces: int = 0
    neumann_flux: Sequence[float] = field(default_factory=lambda: [0.0] * 6)


def _face_patches(mesh: Mesh, f: int):
    """DoF indices (P, N, N) [patch, j along db, i along da] and the area factor of face f."""
    k = mesh.degree
    N = k + 1
    d = f >> 1
    da, db = [e for e in range(3) if e != d]
    n = mesh.n
    m = mesh.m
    plane = 0 if (f & 1) == 0 else n[d] - 1
    ca, cb = np.meshgrid(np.arange(m[da]), np.arange(m[db]), indexing="xy")  # (m[db], m[da])
    ca, cb = ca.ravel(), cb.ravel()  # patch p = ca + m[da] * cb
    i = np.arange(N)
    A = (k * ca)[:, None, None] + i[None, None, :]
    Bv = (k * cb)[:, None, None] + i[None, :, None]
    A, Bv = np.broadcast_arrays(A, Bv)
    c = [None, None, None]
    c[d] = np.full(A.shape, plane)
    c[da], c[db] = A, Bv
    idx = c[0] + n[0] * (c[1] + n[1] * c[2])
    h = [mesh.length[e] / m[e] for e in range(3)]
    return idx, h[da] * h[db]


def _terms(bc: HeatBC, f: int):
    bit = 1 << f
    return bool(bc.convection_faces & bit), bool(bc.radiation_faces & bit), bool(bc.neumann_faces & bit)


def _quad(mesh: Mesh):
    _, _, qw, B, _ = basis(mesh.degree)
    return B, np.outer(qw, qw)  # B[q, i]; W[qb, qa]


def _free(mesh: Mesh, cmask: Optional[np.ndarray]) -> np.ndarray:
    return np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0


def _tangent_coef(bc: HeatBC, conv: bool, rad: bool, tq: np.ndarray) -> np.ndarray:
    c = np.zeros_like(tq)
    if conv:
        c += bc.convection_coefficient
    if rad:
        c += 4.0 * bc.emissivity * SIGMA * tq ** 3
    return c


def face_tangent(mesh: Mesh, cmask, bc: HeatBC, T: Optional[np.ndarray], u: np.ndarray) -> np.ndarray:
    """F(T) u: the boundary-face part of the heat tangent applied to u."""
    B, W = _quad(mesh)
    free = _free(mesh, cmask)
    out = np.zeros(mesh.ndofs)
    uc = np.where(free, u, 0.0)
    Tc = np.zeros(mesh.ndofs) if T is None else np.where(free, T, 0.0)
    for f in range(6):
        conv, rad, _ = _terms(bc, f)
        if not (conv or rad):
            continue
        idx, area = _face_patches(mesh, f)
        uq = np.einsum("bj,ai,pji->pba", B, B, uc[idx])
        tq = np.einsum("bj,ai,pji->pba", B, B, Tc[idx])
        fq = _tangent_coef(bc, conv, rad, tq) * uq * W[None] * area
        loc = np.einsum("bj,ai,pba->pji", B, B, fq)
        keep = free[idx]
        np.add.at(out, idx[keep], loc[keep])
    return out


def face_rhs(mesh: Mesh, cmask, bc: HeatBC, T: np.ndarray) -> np.ndarray:
    """The boundary-face part of create_rhs for temperature T (to be added to dst)."""
    B, W = _quad(mesh)
    free = _free(mesh, cmask)
    out = np.zeros(mesh.ndofs)
    for f in range(6):
        conv, rad, neu = _terms(bc, f)
        if not (conv or rad or neu):
            continue
        idx, area = _face_patches(mesh, f)
        tq = np.einsum("bj,ai,pji->pba", B, B, np.asarray(T)[idx])
        v = np.zeros_like(tq)
        if rad:
            v -= bc.emissivity * SIGMA * (tq ** 4 - bc.radiation_temperature_infinity ** 4)
        if conv:
            v -= bc.convection_coefficient * (tq - bc.convection_temperature_infinity)
        if neu:
            v -= bc.neumann_flux[f]
        loc = np.einsum("bj,ai,pba->pji", B, B, v * W[None] * area)
        keep = free[idx]
        np.add.at(out, idx[keep], loc[keep])
    return out


def face_diagonal(mesh: Mesh, cmask, bc: HeatBC, T: Optional[np.ndarray]) -> np.ndarray:
    """Diagonal of F(T) (0 on constrained rows)."""
    B, W = _quad(mesh)
    free = _free(mesh, cmask)
    out = np.zeros(mesh.ndofs)
    Tc = np.zeros(mesh.ndofs) if T is None else np.where(free, T, 0.0)
    for f in range(6):
        conv, rad, _ = _terms(bc, f)
        if not (conv or rad):
            continue
        idx, area = _face_patches(mesh, f)
        tq = np.einsum("bj,ai,pji->pba", B, B, Tc[idx])
        cw = _tangent_coef(bc, conv, rad, tq) * W[None] * area
        loc = np.einsum("bj,ai,pba->pji", B ** 2, B ** 2, cw)
        keep = free[idx]
        np.add.at(out, idx[keep], loc[keep])
    return out
