"""Pins of the solidification oracle (oracle/solidification.py) without the reference: with equal
solid and liquid properties it is the constant-material heat operator of the C++ oracle, its tangent
is the derivative of minus its residual, and its diagonal is the tangent's; the apparent capacity of
the latent heat releases exactly the latent heat over the mushy zone, in each of its shapes."""
import numpy as np
import pytest

from oracle.oracle import Mesh, Operator
from oracle.solidification import SolidLiquid, apparent_capacity, diagonal, material, residual, tangent_apply

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


LATENT = 2.7e5


def latent(ctype, **kw):
    return SolidLiquid(MAT.liquid, MAT.solid, MAT.liquidus_temperature, MAT.solidus_temperature,
                       latent_heat=LATENT, capacity_type=ctype, **kw)


@pytest.mark.parametrize("ctype", ["qlq", "poly4_bell", "constant"])
def test_apparent_capacity_releases_the_latent_heat(ctype):
    m = latent(ctype)
    n = 100000
    T = 1600.0 + (np.arange(n) + 0.5) * (100.0 / n)  # midpoints of [T_solidus, T_liquidus]
    c, dc = apparent_capacity(m, (1700.0 - T) / 100.0)
    assert abs(c.sum() * (100.0 / n) - LATENT) <= 1e-8 * LATENT
    h = 1e-3
    cp_, _ = apparent_capacity(m, (1700.0 - (T + h)) / 100.0)
    cm_, _ = apparent_capacity(m, (1700.0 - (T - h)) / 100.0)
    inner = (T > 1600.0 + 2 * h) & (T < 1700.0 - 2 * h)
    assert np.max(np.abs((cp_ - cm_)[inner] / (2 * h) - dc[inner])) <= 1e-6 * np.max(np.abs(c))
    out, dout = apparent_capacity(m, np.array([-0.5, 0.0, 1.0, 1.5]))
    assert np.all(out == 0) and np.all(dout == 0)
    # the material's specific heat carries it: rho c_p grows by rho C, d(rho c_p)/dT by rho dC/dT + ...
    T2 = np.linspace(1590.0, 1710.0, 241)
    rc, _, drc, _ = material(m, T2)
    rc0, _, drc0, _ = material(MAT, T2)
    fs = np.clip((1700.0 - T2) / 100.0, 0.0, 1.0)
    rho = np.where(fs == 0, 7.4, np.where(fs == 1, 7.9, 7.4 + 0.5 * (3 - 2 * fs) * fs * fs))
    c2, _ = apparent_capacity(m, fs)
    assert np.max(np.abs(rc - rc0 - rho * c2)) <= 1e-12 * np.max(rc)


def test_qlq_shape():
    m = latent("qlq")
    dT, peak = 100.0, 2.0 * LATENT / 100.0
    T = np.array([1600.0 + 1e-9, 1650.0, 1700.0 - 1e-9, 1600.0 + dT / 6, 1700.0 - dT / 6])
    c, dc = apparent_capacity(m, (1700.0 - T) / dT)
    assert abs(c[1] - peak) <= 1e-9 * peak  # the tent's top at the mid temperature
    assert c[0] <= 1e-9 * peak and c[2] <= 1e-9 * peak and abs(dc[0]) <= 1e-6 and abs(dc[2]) <= 1e-6
    slope = peak / (dT / 2 - dT / 6)  # the linear flank
    assert abs(dc[3] - slope) <= 1e-9 * slope and abs(dc[4] + slope) <= 1e-9 * slope


@pytest.mark.parametrize("ctype", ["qlq", "poly4_bell"])
def test_tangent_with_latent_heat_is_the_derivative_of_minus_the_residual(ctype):
    mesh = Mesh(2, (3, 2, 3))
    cmask = mesh.face_mask(0b000100)
    m = latent(ctype)
    rng = np.random.default_rng(4)
    T = rng.uniform(1590.0, 1710.0, mesh.ndofs)
    Told = T + rng.uniform(-5, 5, mesh.ndofs)
    dT = np.where(cmask == 0, rng.uniform(-1, 1, mesh.ndofs), 0.0)
    eps = 1e-5
    fd = -(residual(mesh, cmask, m, 1e-3, T + eps * dT, Told) - residual(mesh, cmask, m, 1e-3, T - eps * dT, Told))
    fd /= 2 * eps
    tan = tangent_apply(mesh, cmask, m, 1e-3, T, Told, dT)
    assert np.max(np.abs(fd - tan)) <= 1e-6 * np.max(np.abs(tan))
