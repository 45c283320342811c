"""The DoF-vector velocity oracle (oracle/advection_field.py) against the C++ oracle's affine
velocity: FE_Q(k) represents an affine field exactly, so sampling one at the support points must
reproduce the affine operator, its create_rhs and its diagonal."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from oracle import advection_field as AF
from oracle.oracle import Mesh, Operator


@pytest.mark.parametrize("degree,m,faces", [(1, (5, 4, 3), 0), (2, (4, 3, 5), 0b010101), (3, (3, 3, 2), 0)])
def test_affine_field_reproduces_the_affine_operator(degree, m, faces):
    mesh = Mesh(degree, m, origin=(0.1, -0.2, 0.3), length=(1.0, 0.7, 1.2))
    cm = mesh.face_mask(faces) if faces else None
    vel = [0.3, -0.2, 0.1, 0.5, -1.0, 0.2, 1.0, 0.1, -0.3, 0.05, 0.2, -0.4]
    X, Y, Z = mesh.coords()
    field = [vel[d] + vel[3 + 3 * d] * X + vel[4 + 3 * d] * Y + vel[5 + 3 * d] * Z for d in range(3)]
    dt, theta, eps = 1e-2, 0.5, 3e-3
    op = Operator(mesh, "advdiff", cmask=cm, dt=dt, theta=theta, eps=eps, vel=vel)
    u = uniform_dofs(mesh, seed=1)
    ref = op.vmult(u)
    got = AF.tangent_apply(mesh, cm, field, dt, theta, eps, u)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    r = np.zeros(mesh.ndofs)
    op.create_rhs(r, u)
    assert np.max(np.abs(AF.create_rhs(mesh, cm, field, dt, theta, eps, u) - r)) <= 1e-12 * np.max(np.abs(r))
    dref = op.diagonal()
    assert np.max(np.abs(AF.diagonal(mesh, cm, field, dt, theta, eps) - dref)) <= 1e-12 * np.max(np.abs(dref))


def test_nonaffine_field_diagonal_by_unit_vectors():
    mesh = Mesh(2, (3, 2, 2))
    X, Y, Z = mesh.coords()
    field = [np.sin(3 * Y) * Z, np.cos(2 * X) - Z * Z, X * Y]
    d = AF.diagonal(mesh, None, field, 1e-2, 1.0, 1e-3)
    e = np.array([AF.tangent_apply(mesh, None, field, 1e-2, 1.0, 1e-3, np.eye(1, mesh.ndofs, i).ravel())[i]
                  for i in range(mesh.ndofs)])
    assert np.max(np.abs(d - e)) <= 1e-12 * np.max(np.abs(e))


@pytest.mark.parametrize("degree,m,coef", [(1, (4, 3, 3), -1.0), (2, (3, 4, 2), -1.0), (2, (3, 2, 3), 0.7),
                                           (3, (2, 2, 2), -1.0)])
def test_affine_field_reproduces_the_affine_supg_terms(degree, m, coef):
    """oracle/supg.py with the velocity as a DoF vector: an affine field sampled at the support points
    gives the affine form's tau, SUPG apply, rhs and diagonal."""
    from oracle import supg as S

    mesh = Mesh(degree, m, origin=(0.1, -0.2, 0.3), length=(1.0, 0.7, 1.2))
    cm = mesh.face_mask(0b100110)
    vel = [0.3, -0.2, 0.1, 0.5, -1.0, 0.2, 1.0, 0.1, -0.3, 0.05, 0.2, -0.4]
    X, Y, Z = mesh.coords()
    field = [vel[d] + vel[3 + 3 * d] * X + vel[4 + 3 * d] * Y + vel[5 + 3 * d] * Z for d in range(3)]
    u = uniform_dofs(mesh, seed=2)
    tol = lambda r: 1e-12 * np.max(np.abs(r))  # noqa: E731
    t0, t1 = S.supg_tau(mesh, vel, coef), S.supg_tau(mesh, None, coef, field=field)
    assert np.max(np.abs(t1 - t0)) <= tol(t0)
    for plain in (False, True):
        r0 = S.supg_apply(mesh, cm, vel, coef, 50.0, 0.5, 1e-3, u, plain=plain)
        r1 = S.supg_apply(mesh, cm, None, coef, 50.0, 0.5, 1e-3, u, plain=plain, field=field)
        assert np.max(np.abs(r1 - r0)) <= tol(r0)
    d0 = S.supg_diagonal(mesh, cm, vel, coef, 50.0, 0.5, 1e-3)
    d1 = S.supg_diagonal(mesh, cm, None, coef, 50.0, 0.5, 1e-3, field=field)
    assert np.max(np.abs(d1 - d0)) <= tol(d0)


def test_nonaffine_field_supg_diagonal_by_unit_vectors():
    from oracle import supg as S

    mesh = Mesh(2, (3, 2, 2))
    X, Y, Z = mesh.coords()
    field = [np.sin(3 * Y) * Z + 0.4, np.cos(2 * X) - Z * Z, X * Y - 0.3]
    d = S.supg_diagonal(mesh, None, None, -1.0, 50.0, 1.0, 1e-3, field=field)
    e = np.array([S.supg_apply(mesh, None, None, -1.0, 50.0, 1.0, 1e-3, np.eye(1, mesh.ndofs, i).ravel(),
                               field=field)[i] for i in range(mesh.ndofs)])
    assert np.max(np.abs(d - e)) <= 1e-12 * np.max(np.abs(e))
