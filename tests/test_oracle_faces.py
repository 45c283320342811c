"""Pins of the boundary-face oracle (oracle/faces.py) without the reference: an independently
assembled face mass matrix (exact polynomial integration of the Lagrange basis on the Gauss-Lobatto
nodes), the linearisation identity between rhs and tangent, partition of unity and symmetry."""
import numpy as np
import pytest

from oracle.faces import SIGMA, HeatBC, face_diagonal, face_rhs, face_tangent
from oracle.oracle import Mesh, basis


def exact_mass_1d(degree, m, length):
    """Global 1-D FE_Q(degree) mass matrix on m cells of [0, length], integrated exactly."""
    nodes = basis(degree)[0]
    n = degree + 1
    polys = []
    for i in range(n):
        others = np.delete(nodes, i)
        p = np.poly1d(np.poly(others)) / np.prod(nodes[i] - others)
        polys.append(p)
    Me = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            P = np.polyint(polys[i] * polys[j])
            Me[i, j] = P(1.0) - P(0.0)
    h = length / m
    M = np.zeros((degree * m + 1,) * 2)
    for c in range(m):
        s = slice(c * degree, c * degree + n)
        M[s, s] += h * Me
    return M


@pytest.mark.parametrize("degree", [1, 2, 3, 4])
@pytest.mark.parametrize("face", [0, 1, 2, 3, 4, 5])
def test_convection_tangent_is_the_face_mass_matrix(degree, face):
    mesh = Mesh(degree, (3, 2, 4), length=(0.7, 1.1, 0.9))
    h = 2.5
    bc = HeatBC(convection_faces=1 << face, convection_coefficient=h)
    rng = np.random.default_rng(1)
    u = rng.uniform(-1, 1, mesh.ndofs)
    got = face_tangent(mesh, None, bc, None, u).reshape(mesh.n[::-1])
    d = face >> 1
    da, db = [e for e in range(3) if e != d]
    Ma = exact_mass_1d(degree, mesh.m[da], mesh.length[da])
    Mb = exact_mass_1d(degree, mesh.m[db], mesh.length[db])
    U = u.reshape(mesh.n[::-1])  # axes (z, y, x)
    axis = 2 - d
    plane = 0 if face % 2 == 0 else -1
    Up = np.take(U, plane, axis=axis)  # 2-D array, axes ordered (db, da) since db > da
    ref_plane = h * (Mb @ Up @ Ma.T)
    got_plane = np.take(got, plane, axis=axis)
    # the monomial-basis integration of degree-8 products carries ~1e-12 of its own rounding
    assert np.max(np.abs(got_plane - ref_plane)) <= 1e-11 * np.max(np.abs(ref_plane))
    # nothing off the face
    rest = got.copy()
    idx = [slice(None)] * 3
    idx[axis] = plane
    rest[tuple(idx)] = 0
    assert np.max(np.abs(rest)) == 0


def test_partition_of_unity_and_symmetry():
    mesh = Mesh(2, (3, 4, 2), length=(1.0, 0.5, 2.0))
    bc = HeatBC(convection_faces=0b110011, convection_coefficient=3.0, radiation_faces=0b001100, emissivity=0.4)
    T0 = 700.0
    T = np.full(mesh.ndofs, T0)
    ones = np.ones(mesh.ndofs)
    areas = {0: 0.5 * 2.0, 1: 0.5 * 2.0, 2: 1.0 * 2.0, 3: 1.0 * 2.0, 4: 0.5, 5: 0.5}
    expect = sum(3.0 * areas[f] for f in (0, 1, 4, 5)) + sum(4 * 0.4 * SIGMA * T0 ** 3 * areas[f] for f in (2, 3))
    assert abs(face_tangent(mesh, None, bc, T, ones).sum() - expect) <= 1e-12 * expect
    rng = np.random.default_rng(2)
    T = rng.uniform(300, 900, mesh.ndofs)
    x, y = rng.uniform(-1, 1, (2, mesh.ndofs))
    a = x @ face_tangent(mesh, None, bc, T, y)
    b = y @ face_tangent(mesh, None, bc, T, x)
    assert abs(a - b) <= 1e-12 * abs(a)


def test_rhs_at_equilibrium_and_total_flux():
    mesh = Mesh(3, (2, 3, 2))
    bc = HeatBC(convection_faces=0b000011, convection_coefficient=5.0, convection_temperature_infinity=400.0,
                radiation_faces=0b001100, emissivity=0.8, radiation_temperature_infinity=400.0,
                neumann_faces=0b110000, neumann_flux=[0, 0, 0, 0, 2.0, -3.0])
    T = np.full(mesh.ndofs, 400.0)
    r = face_rhs(mesh, None, bc, T)
    # only the Neumann faces contribute: -g.n * area (z faces have area 1)
    assert abs(r.sum() - (-(2.0 - 3.0))) <= 1e-10  # T_q = 400 up to the rounding of sum_i phi_i = 1
    T = np.full(mesh.ndofs, 500.0)
    r = face_rhs(mesh, None, bc, T)
    expect = -(5.0 * 100.0 * 2 + 0.8 * SIGMA * (500.0 ** 4 - 400.0 ** 4) * 2 + (2.0 - 3.0))
    assert abs(r.sum() - expect) <= 1e-12 * abs(expect)


def test_tangent_is_the_derivative_of_minus_rhs():
    mesh = Mesh(2, (2, 3, 2))
    bc = HeatBC(convection_faces=0b000101, convection_coefficient=5.0, convection_temperature_infinity=300.0,
                radiation_faces=0b111010, emissivity=0.6, radiation_temperature_infinity=350.0)
    rng = np.random.default_rng(3)
    T = rng.uniform(400, 800, mesh.ndofs)
    dT = rng.uniform(-1, 1, mesh.ndofs)
    eps = 1e-3
    fd = -(face_rhs(mesh, None, bc, T + eps * dT) - face_rhs(mesh, None, bc, T - eps * dT)) / (2 * eps)
    tan = face_tangent(mesh, None, bc, T, dT)
    assert np.max(np.abs(fd - tan)) <= 1e-7 * np.max(np.abs(tan))


def test_diagonal_is_the_diagonal_of_the_tangent():
    mesh = Mesh(2, (2, 2, 1))
    cmask = mesh.face_mask(0b000001)
    bc = HeatBC(convection_faces=0b000010, convection_coefficient=2.0, radiation_faces=0b111100, emissivity=0.5)
    rng = np.random.default_rng(4)
    T = rng.uniform(300, 600, mesh.ndofs)
    d = face_diagonal(mesh, cmask, bc, T)
    ref = np.zeros(mesh.ndofs)
    for i in range(mesh.ndofs):
        e = np.zeros(mesh.ndofs)
        e[i] = 1.0
        ref[i] = face_tangent(mesh, cmask, bc, T, e)[i]
    assert np.max(np.abs(d - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.all(d[cmask != 0] == 0)
