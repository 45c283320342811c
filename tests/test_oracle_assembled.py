"""The CPU oracle against an independently assembled sparse matrix and analytic identities."""
import numpy as np
import pytest

from oracle.oracle import Mesh, Operator
from meltpooldg_b200.inputs import uniform_dofs, normal_cells
from tests.assembled import assemble


@pytest.mark.parametrize("degree", [1, 2, 4])
@pytest.mark.parametrize("m", [(1, 1, 1), (2, 3, 2), (4, 4, 4)])
def test_heat_vmult_matches_assembled(degree, m):
    if degree == 4 and m == (4, 4, 4):
        m = (3, 2, 3)
    mesh = Mesh(degree, m, origin=(0.1, -0.2, 0.3), length=(1.0, 0.7, 1.3))
    cm = mesh.face_mask(0b110101)
    kc = np.exp(normal_cells(mesh, seed=2, sigma=0.5))
    op = Operator(mesh, "heat", cmask=cm, rho_cp=1.7, dt=1e-2, k_cell=kc)
    x = uniform_dofs(mesh, seed=1)
    A = assemble("heat", degree, m, mesh.origin, mesh.length, cmask=cm, rho_cp=1.7, dt=1e-2, k_cell=kc)
    y_ref = A @ x
    y = op.vmult(x)
    assert np.max(np.abs(y - y_ref)) <= 1e-12 * np.max(np.abs(y_ref))
    d = op.diagonal()
    dref = A.diagonal().copy()
    dref[cm == 1] = 1.0
    assert np.allclose(d, dref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_advdiff_vmult_matches_assembled(degree):
    m = (3, 2, 2)
    mesh = Mesh(degree, m, origin=(0, 0, 0), length=(1, 1, 1))
    vel = [0.1, 0.2, -0.3, 0, -1, 0, 1, 0, 0, 0.2, 0.1, 0]
    cm = mesh.face_mask(0b000011)
    op = Operator(mesh, "advdiff", cmask=cm, dt=5e-3, theta=0.5, eps=1e-3, vel=vel)
    A = assemble("advdiff", degree, m, cmask=cm, dt=5e-3, theta=0.5, eps=1e-3, vel=vel)
    x = uniform_dofs(mesh, seed=4)
    y = op.vmult(x)
    y_ref = A @ x
    assert np.max(np.abs(y - y_ref)) <= 1e-12 * np.max(np.abs(y_ref))
    d = op.diagonal()
    dref = A.diagonal().copy()
    dref[cm == 1] = 1.0
    assert np.allclose(d, dref, rtol=1e-12)


def test_mass_of_one_is_volume():
    """A.1 with k irrelevant on a Neumann mesh sums to rho_cp/dt * |domain| (stiffness kills 1)."""
    mesh = Mesh(2, (3, 4, 2), length=(0.5, 2.0, 1.5))
    op = Operator(mesh, "heat", rho_cp=2.0, dt=0.25, k=7.0)
    y = op.vmult(np.ones(mesh.ndofs))
    assert abs(y.sum() - 2.0 / 0.25 * 0.5 * 2.0 * 1.5) < 1e-12 * 24


@pytest.mark.parametrize("degree", [1, 2, 4])
def test_stiffness_annihilates_linears(degree):
    mesh = Mesh(degree, (2, 2, 3))
    X, Y, Z = mesh.coords()
    op = Operator(mesh, "heat", rho_cp=0.0, dt=1.0, k=1.0)
    interior = mesh.face_mask(63) == 0
    assert np.max(np.abs(op.vmult(np.ones_like(X)))) < 1e-12
    for f in (X, Y, 2 * Z - X + 0.5 * Y):
        # K f vanishes on interior rows (boundary rows carry the natural flux)
        assert np.max(np.abs(op.vmult(f)[interior])) < 1e-12


def test_heat_symmetry():
    mesh = Mesh(2, (3, 3, 3))
    cm = mesh.face_mask(63)
    kc = np.exp(normal_cells(mesh, seed=3, sigma=0.5))
    op = Operator(mesh, "heat", cmask=cm, dt=1e-3, k_cell=kc)
    x = uniform_dofs(mesh, seed=1) * (cm == 0)
    y = uniform_dofs(mesh, seed=2) * (cm == 0)
    a, b = x @ op.vmult(y), y @ op.vmult(x)
    assert abs(a - b) <= 1e-13 * abs(a)


def test_advection_zero_velocity_is_mass_over_dt():
    mesh = Mesh(2, (2, 2, 2))
    x = uniform_dofs(mesh, seed=9)
    adv = Operator(mesh, "advdiff", dt=0.1, theta=1.0, eps=0.0)
    heat = Operator(mesh, "heat", rho_cp=1.0, dt=0.1, k=0.0)
    assert np.allclose(adv.vmult(x), heat.vmult(x), rtol=1e-14, atol=1e-15)


def test_rhs_is_minus_residual():
    """create_rhs(T, T_old, q) = M q - (rho cp/dt) M (T - T_old) - K T, on free rows."""
    mesh = Mesh(2, (3, 2, 2))
    cm = mesh.face_mask(63)
    op = Operator(mesh, "heat", cmask=cm, rho_cp=1.5, dt=0.1, k=2.0)
    T, To, q = (uniform_dofs(mesh, seed=s) for s in (1, 2, 3))
    rhs = np.zeros(mesh.ndofs)
    op.create_rhs(rhs, T, To, q)
    nb = op.with_(cmask=None)
    M = Operator(mesh, "heat", rho_cp=1.0, dt=1.0, k=0.0)
    K = Operator(mesh, "heat", rho_cp=0.0, dt=1.0, k=2.0)
    ref = M.vmult(q) - 1.5 / 0.1 * M.vmult(T - To) - K.vmult(T)
    ref[cm == 1] = 0.0
    assert np.allclose(rhs, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    assert nb is not None


@pytest.mark.parametrize("degree,m,faces", [(1, (9, 7, 5), 0b101101), (2, (17, 9, 6), 63), (3, (8, 7, 9), 0),
                                            (4, (10, 6, 5), 0b010010)])
def test_batched_cpu_apply_matches_the_quadrature_form(degree, m, faces):
    """The cell-batched SIMD heat apply (the timed CPU baseline) equals the oracle's apply."""
    from meltpooldg_b200.inputs import normal_cells, uniform_dofs
    from oracle.oracle import Mesh, Operator

    om = Mesh(degree, m, length=(1.0, 0.8, 1.2))
    cm = om.face_mask(faces) if faces else None
    kc = np.exp(normal_cells(om, seed=2, sigma=0.5))
    op = Operator(om, "heat", cmask=cm, rho_cp=1.3, dt=1e-2, k_cell=kc)
    x = uniform_dofs(om, seed=1)
    a = op.vmult(x)
    assert np.max(np.abs(op.vmult_batched(x) - a)) <= 1e-13 * np.max(np.abs(a))
