"""Conservative level-set reinitialisation operator (Olsson) -- CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU reinitialisation kernels,
never by the product path.

Restates source/level_set/olsson_CG_operator.cpp without the interface penalty:
* tangent (:438-470): dpsi / dt tested with phi, eps_n (grad dpsi . n) n + eps_t (grad dpsi -
  (grad dpsi . n) n) tested with grad phi; dpsi with Dirichlet entries 0;
* rhs (:197-260): [c(psi) n - eps_n (grad psi . n) n - eps_t (grad psi - (grad psi . n) n)] tested
  with grad phi, c(psi) = (1 - psi^2) / 2 (:24-29), psi read plainly, dst overwritten, constrained
  rows 0;
* n = normalize(n_h, tol): n_h / |n_h| above tol, n_h / tol otherwise
  (include/meltpooldg/utilities/dealii_tensor.hpp:175-191); n_h read plainly;
* wetting boundary faces (loops :550-623, face operations :625-716, enabled by
  set_wetting_boundary_condition_ids :64-69; the GPU operator has none of them yet): on each
  such face the tangent adds (D grad dpsi . n_f) tested with phi and the rhs adds
  -((-c(psi) n + D grad psi) . n_f) tested with phi, n_f the outward face normal, n the unit
  interface normal at the face points (``wetting_tangent_apply``, ``wetting_rhs``); the face
  operations read the per-cell diffusion lengths with the face batch's index (:631-640,
  :676-685), which is the same value here because the lengths are uniform.
Per cell with QGauss(k+1), vectorised over the cells with numpy.
"""
from __future__ import annotations

import numpy as np

from oracle.oracle import Mesh, basis
from oracle.supg import _cells, _dof_index, tables


def _setup(mesh: Mesh, cmask, normal, tol):
    qp, qw, B, G, _ = tables(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    idx = _dof_index(mesh, cx, cy, cz)
    ev = lambda Z, Y, X, f: np.einsum("al,bj,ci,xlji->xabc", Z, Y, X, f)  # noqa: E731
    nq = [ev(B, B, B, np.asarray(c, dtype=np.float64)[idx]) for c in normal]
    norm = np.sqrt(nq[0] ** 2 + nq[1] ** 2 + nq[2] ** 2)
    inv = np.where(norm > tol, 1.0 / np.where(norm > 0, norm, 1.0), 1.0 / tol)
    n = [c * inv for c in nq]
    W = h[0] * h[1] * h[2] * np.einsum("a,b,c->abc", qw, qw, qw)[None]
    return B, G, h, idx, free, n, W, ev


def _grad(ev, B, G, h, c):
    return [ev(B, B, G, c) / h[0], ev(B, G, B, c) / h[1], ev(G, B, B, c) / h[2]]


def _scatter(mesh, B, G, h, idx, free, val, flux):
    te = lambda Z, Y, X, F: np.einsum("al,bj,ci,xabc->xlji", Z, Y, X, F)  # noqa: E731
    loc = te(B, B, G, flux[0]) / h[0] + te(B, G, B, flux[1]) / h[1] + te(G, B, B, flux[2]) / h[2]
    if val is not None:
        loc = loc + te(B, B, B, val)
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], loc[keep])
    return out


def tangent_apply(mesh: Mesh, cmask, dt, eps_n, eps_t, normal, tol, u) -> np.ndarray:
    B, G, h, idx, free, n, W, ev = _setup(mesh, cmask, normal, tol)
    uc = np.where(free, u, 0.0)[idx]
    uq = ev(B, B, B, uc)
    g = _grad(ev, B, G, h, uc)
    gn = g[0] * n[0] + g[1] * n[1] + g[2] * n[2]
    flux = [W * (eps_t * g[d] + (eps_n - eps_t) * gn * n[d]) for d in range(3)]
    return _scatter(mesh, B, G, h, idx, free, W * uq / dt, flux)


def create_rhs(mesh: Mesh, cmask, eps_n, eps_t, normal, tol, psi_old) -> np.ndarray:
    B, G, h, idx, free, n, W, ev = _setup(mesh, cmask, normal, tol)
    pc = np.asarray(psi_old, dtype=np.float64)[idx]
    pq = ev(B, B, B, pc)
    g = _grad(ev, B, G, h, pc)
    gn = g[0] * n[0] + g[1] * n[1] + g[2] * n[2]
    cf = 0.5 * (1.0 - pq * pq)
    flux = [W * (cf * n[d] - eps_t * g[d] - (eps_n - eps_t) * gn * n[d]) for d in range(3)]
    return _scatter(mesh, B, G, h, idx, free, None, flux)


def diagonal(mesh: Mesh, cmask, dt, eps_n, eps_t, normal, tol) -> np.ndarray:
    """Diagonal of the tangent (0 on constrained rows)."""
    B, G, h, idx, free, n, W, ev = _setup(mesh, cmask, normal, tol)
    o = lambda Z, Y, X: np.einsum("al,bj,ci->abclji", Z, Y, X)[None]  # noqa: E731
    phi = o(B, B, B)
    dphi = [o(B, B, G) / h[0], o(B, G, B) / h[1], o(G, B, B) / h[2]]
    e = lambda a: a[..., None, None, None]  # noqa: E731
    pn = sum(e(n[d]) * dphi[d] for d in range(3))
    pp = sum(dp * dp for dp in dphi)
    term = e(W / dt) * phi * phi + e(W) * (eps_t * pp + (eps_n - eps_t) * pn * pn)
    loc = term.sum(axis=(1, 2, 3))
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], loc[keep])
    return out


def _band_mask(ev, B, idx, level_set, narrow_band):
    """Narrow-band mask at the Gauss points: 1 where |level set| < narrow_band, else 0
    (include/meltpooldg/level_set/level_set_tools.hpp:357-368); 1 everywhere without a band."""
    if narrow_band is None:
        return 1.0
    lq = ev(B, B, B, np.asarray(level_set, dtype=np.float64)[idx])
    return np.where(np.abs(lq) >= narrow_band, 0.0, 1.0)


def normal_rhs(mesh: Mesh, cmask, psi, normalized: bool = False, narrow_band=None):
    """NormalVectorOperator::create_rhs (source/level_set/normal_vector_operator.cpp:160-240):
    int g_d phi with g = grad psi, or g normalised (divided by 1e-16 at or below it); with a
    narrow band the gradient is masked by |psi| < narrow_band at each point first."""
    qp, qw, B, G, _ = tables(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    idx = _dof_index(mesh, cx, cy, cz)
    ev = lambda Z, Y, X, f: np.einsum("al,bj,ci,xlji->xabc", Z, Y, X, f)  # noqa: E731
    pc = np.asarray(psi, dtype=np.float64)[idx]
    mask = _band_mask(ev, B, idx, psi, narrow_band)
    g = [c * mask for c in _grad(ev, B, G, h, pc)]
    if normalized:
        nn = np.sqrt(g[0] ** 2 + g[1] ** 2 + g[2] ** 2)
        s = np.where(nn > 1e-16, 1.0 / np.where(nn > 0, nn, 1.0), 1e16)
        g = [c * s for c in g]
    W = h[0] * h[1] * h[2] * np.einsum("a,b,c->abc", qw, qw, qw)[None]
    te = lambda Z, Y, X, F: np.einsum("al,bj,ci,xabc->xlji", Z, Y, X, F)  # noqa: E731
    out = []
    for d in range(3):
        o = np.zeros(mesh.ndofs)
        keep = free[idx]
        np.add.at(o, idx[keep], te(B, B, B, W * g[d])[keep])
        out.append(o)
    return out


def curvature_rhs(mesh: Mesh, cmask, normal, tol, level_set=None, narrow_band=None):
    """CurvatureOperator::create_rhs (source/level_set/curvature_operator.cpp:190-255):
    -int div(n) phi with n = normalize(n_i, tol) at every DoF, masked by |level_set| < narrow_band
    at each point when a band is given; constrained rows 0."""
    qp, qw, B, G, _ = tables(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    idx = _dof_index(mesh, cx, cy, cz)
    nv = [np.asarray(c, dtype=np.float64) for c in normal]
    nn = np.sqrt(nv[0] ** 2 + nv[1] ** 2 + nv[2] ** 2)
    s = np.where(nn > tol, 1.0 / np.where(nn > 0, nn, 1.0), 1.0 / tol)
    nv = [c * s for c in nv]
    ev = lambda Z, Y, X, f: np.einsum("al,bj,ci,xlji->xabc", Z, Y, X, f)  # noqa: E731
    div = (ev(B, B, G, nv[0][idx]) / h[0] + ev(B, G, B, nv[1][idx]) / h[1] + ev(G, B, B, nv[2][idx]) / h[2])
    div = div * _band_mask(ev, B, idx, level_set, narrow_band)
    W = h[0] * h[1] * h[2] * np.einsum("a,b,c->abc", qw, qw, qw)[None]
    te = lambda Z, Y, X, F: np.einsum("al,bj,ci,xabc->xlji", Z, Y, X, F)  # noqa: E731
    out = np.zeros(mesh.ndofs)
    keep = free[idx]
    np.add.at(out, idx[keep], te(B, B, B, -W * div)[keep])
    return out


def _endpoint_rows(degree: int):
    """Values and derivatives of the FE_Q(degree) Lagrange basis at x = 0 and x = 1 (rows of the
    nodal differentiation matrix D_ji = l_i'(x_j), from the barycentric weights of the
    Gauss-Lobatto nodes, whose first and last nodes are 0 and 1)."""
    nodes = basis(degree)[0]
    n = len(nodes)
    w = np.array([1.0 / np.prod([nodes[i] - nodes[m] for m in range(n) if m != i]) for i in range(n)])
    D = np.zeros((n, n))
    for j in range(n):
        for i in range(n):
            if i != j:
                D[j, i] = w[i] / w[j] / (nodes[j] - nodes[i])
        D[j, j] = -D[j].sum()
    return np.eye(n)[[0, n - 1]], D[[0, n - 1]]


def _wetting(mesh: Mesh, cmask, faces: int, eps_n, eps_t, normal, tol, u, rhs: bool):
    qp, qw, B, G, _ = tables(mesh.degree)
    Vend, Dend = _endpoint_rows(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    cc = (cx, cy, cz)
    ev = lambda Z, Y, X, f: np.einsum("al,bj,ci,xlji->xabc", Z, Y, X, f)  # noqa: E731
    te = lambda Z, Y, X, F: np.einsum("al,bj,ci,xabc->xlji", Z, Y, X, F)  # noqa: E731
    out = np.zeros(mesh.ndofs)
    for f in range(6):
        if not (faces >> f) & 1:
            continue
        d, side = f >> 1, f & 1
        sel = cc[d] == (mesh.m[d] - 1 if side else 0)
        idx = _dof_index(mesh, cx[sel], cy[sel], cz[sel])
        # per dimension (x, y, z): value / derivative tables at the face points
        val = [B, B, B]
        der = [G / h[0], G / h[1], G / h[2]]
        val[d], der[d] = Vend[side:side + 1], Dend[side:side + 1] / h[d]
        wts = [qw, qw, qw]
        wts[d] = np.ones(1)
        W = np.einsum("a,b,c->abc", wts[2], wts[1], wts[0])[None] * (h[0] * h[1] * h[2] / h[d])

        def at(c, grad_dim=None):
            t = [der[e] if e == grad_dim else val[e] for e in range(3)]
            return ev(t[2], t[1], t[0], c)

        nq = [at(np.asarray(c, dtype=np.float64)[idx]) for c in normal]
        norm = np.sqrt(nq[0] ** 2 + nq[1] ** 2 + nq[2] ** 2)
        inv = np.where(norm > tol, 1.0 / np.where(norm > 0, norm, 1.0), 1.0 / tol)
        n = [c * inv for c in nq]
        uc = (np.asarray(u, dtype=np.float64) if rhs else np.where(free, u, 0.0))[idx]
        g = [at(uc, e) for e in range(3)]
        gn = g[0] * n[0] + g[1] * n[1] + g[2] * n[2]
        # D grad u . n_f with n_f = (+-1) e_d
        flux_d = eps_t * g[d] + (eps_n - eps_t) * gn * n[d]
        sgn = 1.0 if side else -1.0
        if rhs:
            uq = at(uc)
            integrand = -sgn * (-0.5 * (1.0 - uq * uq) * n[d] + flux_d)
        else:
            integrand = sgn * flux_d
        loc = te(val[2], val[1], val[0], W * integrand)
        keep = free[idx]
        np.add.at(out, idx[keep], loc[keep])
    return out


def wetting_tangent_apply(mesh: Mesh, cmask, faces: int, eps_n, eps_t, normal, tol, u) -> np.ndarray:
    """Wetting boundary faces' part of the tangent (faces: bit 2d low, 2d+1 high face of
    dimension d); u with Dirichlet entries 0, constrained rows 0."""
    return _wetting(mesh, cmask, faces, eps_n, eps_t, normal, tol, u, rhs=False)


def wetting_rhs(mesh: Mesh, cmask, faces: int, eps_n, eps_t, normal, tol, psi) -> np.ndarray:
    """Wetting boundary faces' part of create_rhs (psi read plainly, constrained rows 0)."""
    return _wetting(mesh, cmask, faces, eps_n, eps_t, normal, tol, psi, rhs=True)


def projection_apply(mesh: Mesh, cmask, damping, u, level_set=None, narrow_band=None) -> np.ndarray:
    """The normal-vector / curvature projection operator M + damping K per component
    (normal_vector_operator.cpp:326-358, curvature_operator.cpp:337-369), u with Dirichlet entries
    0; with a narrow band both terms are masked by |level_set| < narrow_band at each point."""
    qp, qw, B, G, _ = tables(mesh.degree)
    h = [mesh.length[d] / mesh.m[d] for d in range(3)]
    free = np.ones(mesh.ndofs, bool) if cmask is None else np.asarray(cmask) == 0
    cx, cy, cz = _cells(mesh)
    idx = _dof_index(mesh, cx, cy, cz)
    ev = lambda Z, Y, X, f: np.einsum("al,bj,ci,xlji->xabc", Z, Y, X, f)  # noqa: E731
    W = h[0] * h[1] * h[2] * np.einsum("a,b,c->abc", qw, qw, qw)[None]
    W = W * _band_mask(ev, B, idx, level_set, narrow_band)
    uc = np.where(free, u, 0.0)[idx]
    g = _grad(ev, B, G, h, uc)
    return _scatter(mesh, B, G, h, idx, free, W * ev(B, B, B, uc), [W * damping * c for c in g])
