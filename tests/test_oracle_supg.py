"""Pins of the SUPG oracle (oracle/supg.py) without the reference: an independent single-cell
assembly from Lagrange polynomials and numpy's Gauss-Legendre rule, the diagonal against unit-vector
applies, and the scaling of tau_c."""
import numpy as np
import pytest

from oracle.oracle import Mesh, basis
from oracle.supg import supg_apply, supg_diagonal, supg_tau

VEL = [0.1, 0.2, -0.3, 0.0, -1.0, 0.3, 1.0, 0.1, 0.0, 0.2, 0.1, -0.2]


def lagrange_1d(degree):
    nodes = basis(degree)[0]
    polys = []
    for i in range(degree + 1):
        others = np.delete(nodes, i)
        polys.append(np.poly1d(np.poly(others)) / np.prod(nodes[i] - others))
    return polys


@pytest.mark.parametrize("degree", [1, 2])
@pytest.mark.parametrize("coef", [-1.0, 0.7])
def test_single_cell_against_direct_assembly(degree, coef):
    origin, length = (0.2, -0.1, 0.3), (0.5, 0.4, 0.6)
    mesh = Mesh(degree, (1, 1, 1), origin=origin, length=length)
    inv_dt, th_adv, th_dif = 20.0, 0.5, 0.5 * 3e-2
    n = degree + 1
    P = lagrange_1d(degree)
    xg, wg = np.polynomial.legendre.leggauss(n)
    xg, wg = 0.5 * (xg + 1.0), 0.5 * wg
    val = np.array([[p(x) for p in P] for x in xg])  # [q, i]
    der = np.array([[p.deriv()(x) for p in P] for x in xg])
    sec = np.array([[p.deriv(2)(x) for p in P] for x in xg])
    h = np.array(length)
    S = np.zeros((n ** 3, n ** 3))
    vmax = 0.0
    pts = []
    for a in range(n):
        for b in range(n):
            for c in range(n):
                x = np.array([origin[0] + h[0] * xg[c], origin[1] + h[1] * xg[b], origin[2] + h[2] * xg[a]])
                v = np.array([VEL[d] + VEL[3 + 3 * d: 6 + 3 * d] @ x for d in range(3)])
                vmax = max(vmax, np.linalg.norm(v))
                pts.append((a, b, c, v, wg[a] * wg[b] * wg[c] * np.prod(h)))
    size = np.linalg.norm(h) / np.sqrt(3)
    tau = (1.0 / vmax if coef < 0 else coef) * size
    assert abs(supg_tau(mesh, VEL, coef)[0] - tau) <= 1e-14 * tau
    for (a, b, c, v, W) in pts:
        phi, grad, lap = [], [], []
        for l in range(n):
            for j in range(n):
                for i in range(n):
                    phi.append(val[c, i] * val[b, j] * val[a, l])
                    grad.append(np.array([der[c, i] * val[b, j] * val[a, l] / h[0],
                                          val[c, i] * der[b, j] * val[a, l] / h[1],
                                          val[c, i] * val[b, j] * der[a, l] / h[2]]))
                    lap.append(sec[c, i] * val[b, j] * val[a, l] / h[0] ** 2 +
                               val[c, i] * sec[b, j] * val[a, l] / h[1] ** 2 +
                               val[c, i] * val[b, j] * sec[a, l] / h[2] ** 2)
        vg = np.array([v @ g for g in grad])
        strong = inv_dt * np.array(phi) + th_adv * vg - th_dif * np.array(lap)
        S += tau * W * np.outer(vg, strong)
    u = np.random.default_rng(1).uniform(-1, 1, n ** 3)
    got = supg_apply(mesh, None, VEL, coef, inv_dt, th_adv, th_dif, u)
    assert np.max(np.abs(got - S @ u)) <= 1e-12 * np.max(np.abs(S @ u))
    d = supg_diagonal(mesh, None, VEL, coef, inv_dt, th_adv, th_dif)
    assert np.max(np.abs(d - np.diag(S))) <= 1e-12 * np.max(np.abs(np.diag(S)))


def test_diagonal_against_unit_vectors_with_constraints():
    mesh = Mesh(2, (2, 2, 1), origin=(0, 0.1, -0.2), length=(1.0, 0.9, 1.1))
    cmask = mesh.face_mask(0b010001)
    args = (VEL, -1.0, 50.0, 1.0, 1e-2)
    d = supg_diagonal(mesh, cmask, *args)
    ref = np.array([supg_apply(mesh, cmask, *args, np.eye(mesh.ndofs)[i])[i] for i in range(mesh.ndofs)])
    assert np.max(np.abs(d - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.all(d[cmask != 0] == 0)


def test_tau_scaling_and_zero_velocity():
    mesh = Mesh(1, (3, 2, 2))
    u = np.random.default_rng(2).uniform(-1, 1, mesh.ndofs)
    a = supg_apply(mesh, None, VEL, 0.5, 10.0, 1.0, 1e-3, u)
    b = supg_apply(mesh, None, VEL, 1.0, 10.0, 1.0, 1e-3, u)
    assert np.max(np.abs(2 * a - b)) <= 1e-13 * np.max(np.abs(b))
    zero = [0.0] * 12
    assert np.all(supg_tau(mesh, zero, -1.0) == 0)
    assert np.max(np.abs(supg_apply(mesh, None, zero, 0.5, 10.0, 1.0, 1e-3, u))) == 0
