"""Pins of the reinitialisation oracle (oracle/reinit.py): the isotropic limit is the C++ oracle's
heat operator, the tangent is symmetric, a constant field with a constant normal has a zero-sum
rhs, and the diagonal is the tangent's."""
import numpy as np
import pytest

from oracle.oracle import Mesh, Operator
from oracle.reinit import create_rhs, diagonal, tangent_apply


def radial_normal(mesh):
    X, Y, Z = mesh.coords()
    return [X - 0.45, Y - 0.5, Z - 0.55]


@pytest.mark.parametrize("degree", [1, 2])
def test_isotropic_limit_is_the_heat_operator(degree):
    mesh = Mesh(degree, (3, 4, 2), length=(0.7, 0.9, 0.5))
    cmask = mesh.face_mask(0b010001)
    u = np.random.default_rng(1).uniform(-1, 1, mesh.ndofs)
    o = Operator(mesh, "heat", cmask=cmask, rho_cp=1.0, dt=1e-2, k=0.03)
    ref = o.vmult(u)
    got = tangent_apply(mesh, cmask, 1e-2, 0.03, 0.03, radial_normal(mesh), 1e-12, u)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_symmetry_and_rhs_of_a_constant_field():
    mesh = Mesh(2, (3, 2, 3))
    rng = np.random.default_rng(2)
    n = radial_normal(mesh)
    x, y = rng.uniform(-1, 1, (2, mesh.ndofs))
    a = x @ tangent_apply(mesh, None, 1e-2, 0.05, 0.01, n, 1e-12, y)
    b = y @ tangent_apply(mesh, None, 1e-2, 0.05, 0.01, n, 1e-12, x)
    assert abs(a - b) <= 1e-12 * abs(a)
    const = [np.full(mesh.ndofs, 0.3), np.full(mesh.ndofs, -0.4), np.full(mesh.ndofs, 0.5)]
    r = create_rhs(mesh, None, 0.05, 0.01, const, 1e-12, np.full(mesh.ndofs, 0.2))
    assert abs(r.sum()) <= 1e-14 and np.max(np.abs(r)) > 1e-3


def test_diagonal_is_the_tangents():
    mesh = Mesh(2, (2, 2, 1))
    cmask = mesh.face_mask(0b000001)
    n = radial_normal(mesh)
    d = diagonal(mesh, cmask, 1e-2, 0.05, 0.01, n, 1e-12)
    ref = np.array([tangent_apply(mesh, cmask, 1e-2, 0.05, 0.01, n, 1e-12, np.eye(mesh.ndofs)[i])[i]
                    for i in range(mesh.ndofs)])
    assert np.max(np.abs(d - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.all(d[cmask != 0] == 0)
