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
