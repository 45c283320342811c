"""Independent assembled-matrix restatement of the two operators (test helper).

Element matrices are built from numpy's own Gauss-Legendre rule and Lagrange polynomials on
Gauss-Lobatto nodes (computed here from numpy.polynomial, not from the oracle), then assembled
into a scipy sparse matrix -- the pattern of the reference's
compute_system_matrix_from_matrixfree (source/heat/heat_diffuse_operator.cpp:286-295).
Constrained rows/columns are dropped (rows left zero), like the matrix-free vmult.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from numpy.polynomial import legendre as npleg


def lobatto_nodes(k: int) -> np.ndarray:
    if k == 1:
        return np.array([0.0, 1.0])
    c = np.zeros(k + 1)
    c[k] = 1.0
    inner = np.sort(npleg.legroots(npleg.legder(c)).real)
    return np.concatenate([[0.0], 0.5 * (inner + 1.0), [1.0]])


def lagrange_tables(nodes: np.ndarray, x: np.ndarray):
    n = len(nodes)
    V = np.zeros((len(x), n))
    D = np.zeros((len(x), n))
    for i in range(n):
        others = np.delete(nodes, i)
        p = np.poly1d(np.poly(others) / np.prod(nodes[i] - others))
        V[:, i] = p(x)
        D[:, i] = p.deriv()(x)
    return V, D


def element_1d(k: int):
    nodes = lobatto_nodes(k)
    xg, wg = npleg.leggauss(k + 1)
    xq, wq = 0.5 * (xg + 1.0), 0.5 * wg
    V, D = lagrange_tables(nodes, xq)
    return nodes, xq, wq, V, D


def assemble(kind: str, degree: int, m, origin=(0, 0, 0), length=(1, 1, 1), cmask=None,
             rho_cp=1.0, dt=1.0, k=1.0, k_cell=None, theta=1.0, eps=0.0, vel=None):
    """Sparse A with the same lexicographic lattice numbering as the oracle."""
    nodes, xq, wq, V, D = element_1d(degree)
    n = degree + 1
    m = tuple(int(v) for v in m)
    h = [length[d] / m[d] for d in range(3)]
    nl = [degree * m[d] + 1 for d in range(3)]
    # 3-D tables at q-points, local index (l, j, i) with i = x fastest
    Vx, Vy, Vz = V, V, V
    rows, cols, vals = [], [], []
    li = np.arange(n)
    vel = np.zeros(12) if vel is None else np.asarray(vel, float)
    for cz in range(m[2]):
        for cy in range(m[1]):
            for cx in range(m[0]):
                cell = cx + m[0] * (cy + m[1] * cz)
                I = degree * cx + li
                J = degree * cy + li
                K = degree * cz + li
                gidx = (I[None, None, :] + nl[0] * (J[None, :, None] + nl[1] * K[:, None, None])).ravel()
                # basis at quadrature points: phi[q, i] as kron
                phi = np.einsum("ca,bd,ef->cbeadf", Vz, Vy, Vx).reshape(n ** 3, n ** 3)
                dphx = np.einsum("ca,bd,ef->cbeadf", Vz, Vy, D).reshape(n ** 3, n ** 3) / h[0]
                dphy = np.einsum("ca,bd,ef->cbeadf", Vz, D, Vx).reshape(n ** 3, n ** 3) / h[1]
                dphz = np.einsum("ca,bd,ef->cbeadf", D, Vy, Vx).reshape(n ** 3, n ** 3) / h[2]
                W = np.einsum("a,b,c->abc", wq, wq, wq).ravel() * h[0] * h[1] * h[2]
                if kind == "heat":
                    kc = k if k_cell is None else k_cell[cell]
                    Ae = (rho_cp / dt) * phi.T @ (W[:, None] * phi)
                    for dph in (dphx, dphy, dphz):
                        Ae += kc * dph.T @ (W[:, None] * dph)
                else:
                    qz, qy, qx = np.meshgrid(xq, xq, xq, indexing="ij")
                    X = origin[0] + h[0] * (cx + qx.ravel())
                    Y = origin[1] + h[1] * (cy + qy.ravel())
                    Z = origin[2] + h[2] * (cz + qz.ravel())
                    vx = vel[0] + vel[3] * X + vel[4] * Y + vel[5] * Z
                    vy = vel[1] + vel[6] * X + vel[7] * Y + vel[8] * Z
                    vz = vel[2] + vel[9] * X + vel[10] * Y + vel[11] * Z
                    adv = vx[:, None] * dphx + vy[:, None] * dphy + vz[:, None] * dphz
                    Ae = (1.0 / dt) * phi.T @ (W[:, None] * phi) + theta * phi.T @ (W[:, None] * adv)
                    for dph in (dphx, dphy, dphz):
                        Ae += theta * eps * dph.T @ (W[:, None] * dph)
                r, c = np.meshgrid(gidx, gidx, indexing="ij")
                rows.append(r.ravel())
                cols.append(c.ravel())
                vals.append(Ae.ravel())
    N = nl[0] * nl[1] * nl[2]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    if cmask is not None:
        free = (np.asarray(cmask) == 0).astype(float)
        Dm = sp.diags(free)
        A = Dm @ A @ Dm
    return A.tocsr()
