"""Pins of the solidification oracle (oracle/solidification.py) without the reference: with equal
solid and liquid properties it is the constant-material heat operator of the C++ oracle, its tangent
is the derivative of minus its residual, and its diagonal is the tangent's."""
import numpy as np
import pytest

from oracle.oracle import Mesh, Operator
from oracle.solidification import SolidLiquid, diagonal, material, residual, tangent_apply

MAT = SolidLiquid(liquid=(7.4, 0.8, 30.0), solid=(7.9, 0.6, 20.0), liquidus_temperature=1700.0,
                  solidus_temperature=1600.0)


@pytest.mark.parametrize("degree", [1, 2])
def test_constant_material_is_the_heat_operator(degree):
    mesh = Mesh(degree, (3, 4, 2), length=(0.7, 0.9, 0.5))
    cmask = mesh.face_mask(0b010001)
    m = SolidLiquid(liquid=(2.0, 1.5, 0.7), solid=(2.0, 1.5, 0.7))
    rng = np.random.default_rng(1)
    T, Told, u = rng.uniform(-1, 1, (3, mesh.ndofs))
    dt = 1e-2
    o = Operator(mesh, "heat", cmask=cmask, rho_cp=3.0, dt=dt, k=0.7)
    ref = o.vmult(u)
    assert np.max(np.abs(tangent_apply(mesh, cmask, m, dt, T, Told, u) - ref)) <= 1e-12 * np.max(np.abs(ref))
    r = np.zeros(mesh.ndofs)
    o.create_rhs(r, T, Told, None)
    assert np.max(np.abs(residual(mesh, cmask, m, dt, T, Told) - r)) <= 1e-12 * np.max(np.abs(r))


@pytest.mark.parametrize("degree", [1, 2])
@pytest.mark.parametrize("sharp", [False, True])
def test_tangent_is_the_derivative_of_minus_the_residual(degree, sharp):
    mesh = Mesh(degree, (3, 2, 3))
    cmask = mesh.face_mask(0b000100)
    m = SolidLiquid(MAT.liquid, MAT.solid, MAT.liquidus_temperature, MAT.solidus_temperature, sharp)
    rng = np.random.default_rng(2)
    T = rng.uniform(1560.0, 1740.0, mesh.ndofs)
    Told = T + rng.uniform(-5, 5, mesh.ndofs)
    dT = np.where(cmask == 0, rng.uniform(-1, 1, mesh.ndofs), 0.0)
    eps = 1e-5
    fd = -(residual(mesh, cmask, m, 1e-3, T + eps * dT, Told) - residual(mesh, cmask, m, 1e-3, T - eps * dT, Told))
    fd /= 2 * eps
    tan = tangent_apply(mesh, cmask, m, 1e-3, T, Told, dT)
    assert np.max(np.abs(fd - tan)) <= 1e-6 * np.max(np.abs(tan))


def test_material_blend_and_derivative():
    T = np.linspace(1550.0, 1750.0, 2001)
    rc, k, drc, dk = material(MAT, T)
    assert rc[0] == 7.9 * 0.6 and rc[-1] == 7.4 * 0.8 and k[0] == 20.0 and k[-1] == 30.0
    h = 1e-4
    rc1, k1, _, _ = material(MAT, T + h)
    rc0, k0, _, _ = material(MAT, T - h)
    inner = (T > 1600.0 + 2 * h) & (T < 1700.0 - 2 * h)
    assert np.max(np.abs((k1 - k0)[inner] / (2 * h) - dk[inner])) <= 1e-6
    assert np.max(np.abs((rc1 - rc0)[inner] / (2 * h) - drc[inner])) <= 1e-6
    assert np.all(dk[~inner & ((T < 1600.0) | (T > 1700.0))] == 0)


def test_diagonal_is_the_tangents():
    mesh = Mesh(2, (2, 2, 1))
    cmask = mesh.face_mask(0b000001)
    rng = np.random.default_rng(3)
    T = rng.uniform(1590.0, 1710.0, mesh.ndofs)
    Told = T - 3.0
    d = diagonal(mesh, cmask, MAT, 1e-3, T, Told)
    ref = np.array([tangent_apply(mesh, cmask, MAT, 1e-3, T, Told, np.eye(mesh.ndofs)[i])[i]
                    for i in range(mesh.ndofs)])
    assert np.max(np.abs(d - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.all(d[cmask != 0] == 0)
