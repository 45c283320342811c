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


def test_normal_and_curvature_rhs_of_simple_fields():
    from oracle.reinit import curvature_rhs, normal_rhs

    mesh = Mesh(2, (3, 2, 4), length=(0.6, 0.8, 1.2))
    X, Y, Z = mesh.coords()
    vol = 0.6 * 0.8 * 1.2
    # linear level set: the gradient is constant, so each component sums to a_d * volume
    a = (0.3, -1.2, 0.7)
    n = normal_rhs(mesh, None, a[0] * X + a[1] * Y + a[2] * Z + 0.1)
    for d in range(3):
        assert abs(n[d].sum() - a[d] * vol) <= 1e-13
    nn = normal_rhs(mesh, None, a[0] * X + a[1] * Y + a[2] * Z, normalized=True)
    norm = np.sqrt(sum(c * c for c in a))
    for d in range(3):
        assert abs(nn[d].sum() - a[d] / norm * vol) <= 1e-13
    # a normal field below the tolerance is divided by it: n = (alpha x, 0, 0) / tol, div = alpha / tol
    alpha, tol = 1e-4, 1.0
    c = curvature_rhs(mesh, None, [alpha * X, 0 * X, 0 * X], tol)
    assert abs(c.sum() + alpha / tol * vol) <= 1e-15


@pytest.mark.parametrize("degree", [1, 2])
def test_anisotropic_cell_against_direct_assembly(degree):
    """Single cell, varying normal: the tangent matrix M/dt + int grad(phi_i) . D grad(phi_j) with
    D = eps_t I + (eps_n - eps_t) n n^T, and the rhs int [c(psi) n - D grad psi] . grad(phi_i), built
    point by point from numpy's Lagrange polynomials and Gauss-Legendre rule."""
    from tests.assembled import element_1d

    origin, length = (0.1, -0.2, 0.3), (0.5, 0.4, 0.7)
    mesh = Mesh(degree, (1, 1, 1), origin=origin, length=length)
    dt, eps_n, eps_t, tol = 1e-2, 0.05, 0.01, 1e-12
    nodes, xq, wq, V, D = element_1d(degree)
    n = degree + 1
    h = np.array(length)
    nh = radial_normal(mesh)
    psi = np.random.default_rng(4).uniform(-0.9, 0.9, mesh.ndofs)
    A = np.zeros((n ** 3, n ** 3))
    rhs = np.zeros(n ** 3)
    for a in range(n):
        for b in range(n):
            for c in range(n):
                W = wq[a] * wq[b] * wq[c] * np.prod(h)
                phi = np.array([V[c, i] * V[b, j] * V[a, l] for l in range(n) for j in range(n) for i in range(n)])
                grad = np.array([[D[c, i] * V[b, j] * V[a, l] / h[0], V[c, i] * D[b, j] * V[a, l] / h[1],
                                  V[c, i] * V[b, j] * D[a, l] / h[2]]
                                 for l in range(n) for j in range(n) for i in range(n)])
                nq = np.array([phi @ nh[d] for d in range(3)])
                nq = nq / max(np.linalg.norm(nq), tol)
                Dm = eps_t * np.eye(3) + (eps_n - eps_t) * np.outer(nq, nq)
                A += W * (np.outer(phi, phi) / dt + grad @ Dm @ grad.T)
                pq = phi @ psi
                gp = grad.T @ psi
                rhs += W * grad @ (0.5 * (1.0 - pq * pq) * nq - Dm @ gp)
    u = np.random.default_rng(5).uniform(-1, 1, mesh.ndofs)
    got = tangent_apply(mesh, None, dt, eps_n, eps_t, nh, tol, u)
    assert np.max(np.abs(got - A @ u)) <= 1e-12 * np.max(np.abs(A @ u))
    r = create_rhs(mesh, None, eps_n, eps_t, nh, tol, psi)
    assert np.max(np.abs(r - rhs)) <= 1e-12 * np.max(np.abs(rhs))
    d = diagonal(mesh, None, dt, eps_n, eps_t, nh, tol)
    assert np.max(np.abs(d - np.diag(A))) <= 1e-12 * np.max(np.abs(np.diag(A)))


def test_curvature_rhs_of_a_sphere_converges_to_two_over_r():
    """Nodal normals of a sphere centred outside the box, n = (x - c) / |x - c|, have div n = 2 / r:
    the sum of the curvature rhs tends to -int 2 / |x - c| dx (reference integral from a 12-point
    Gauss rule per cell of an 8^3 grid), and the error falls at least 4x per mesh halving."""
    from oracle.reinit import curvature_rhs

    c = np.array([-0.4, 1.3, 0.6])
    xg, wg = np.polynomial.legendre.leggauss(12)
    pts = np.concatenate([(j + 0.5 * (xg + 1.0)) / 8.0 for j in range(8)])
    wts = np.tile(0.5 * wg / 8.0, 8)
    P = np.stack(np.meshgrid(pts, pts, pts, indexing="ij"), axis=-1)
    Wt = np.einsum("a,b,c->abc", wts, wts, wts)
    exact = -np.sum(Wt * 2.0 / np.linalg.norm(P - c, axis=-1))
    err = []
    for m in (2, 4, 8):
        mesh = Mesh(2, (m, m, m))
        X, Y, Z = mesh.coords()
        r = np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2)
        got = curvature_rhs(mesh, None, [(X - c[0]) / r, (Y - c[1]) / r, (Z - c[2]) / r], 1e-12).sum()
        err.append(abs(got - exact))
    assert err[1] <= err[0] / 4 and err[2] <= err[1] / 4 and err[2] <= 1e-5 * abs(exact), (err, exact)


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_wetting_faces_are_the_boundary_flux(degree):
    """With a constant normal, D is constant and for a quadratic u integration by parts gives
    int_boundary (D grad u . n_f) phi = int D grad u . grad phi + tr(D H_u) int phi exactly: the wetting
    tangent on all six faces equals the cell diffusion apply plus tr(D H_u) times the lumped mass."""
    from oracle.reinit import wetting_tangent_apply

    mesh = Mesh(degree, (3, 2, 4), origin=(0.1, -0.2, 0.3), length=(0.6, 0.5, 0.8))
    X, Y, Z = mesh.coords()
    a = np.array([0.3, -0.5, 0.8]) / np.linalg.norm([0.3, -0.5, 0.8])
    normal = [np.full(mesh.ndofs, c) for c in a]
    eps_n, eps_t, tol = 0.05, 0.01, 1e-12
    if degree == 1:  # bilinear terms only: H_u has no diagonal
        u = -0.4 * X * Y + 0.2 * Y * Z + X - 0.5
        H = np.array([[0.0, -0.4, 0.0], [-0.4, 0.0, 0.2], [0.0, 0.2, 0.0]])
    else:
        u = 0.7 * X * X - 0.4 * X * Y + 1.3 * Z * Z + 0.2 * Y * Z + X - 0.5
        H = np.array([[1.4, -0.4, 0.0], [-0.4, 0.0, 0.2], [0.0, 0.2, 2.6]])
    D = eps_t * np.eye(3) + (eps_n - eps_t) * np.outer(a, a)
    Ku = tangent_apply(mesh, None, 1e300, eps_n, eps_t, normal, tol, u)  # the 1/dt mass term vanishes
    M1 = tangent_apply(mesh, None, 1.0, 0.0, 0.0, normal, tol, np.ones(mesh.ndofs))
    ref = Ku + np.sum(D * H) * M1
    got = wetting_tangent_apply(mesh, None, 63, eps_n, eps_t, normal, tol, u)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    # additive over faces
    parts = sum(wetting_tangent_apply(mesh, None, 1 << f, eps_n, eps_t, normal, tol, u) for f in range(6))
    assert np.max(np.abs(parts - got)) <= 1e-13 * np.max(np.abs(got))


def test_wetting_rhs_linearisation_and_compressive_flux():
    from oracle.reinit import wetting_rhs, wetting_tangent_apply

    mesh = Mesh(2, (3, 3, 2), length=(0.9, 0.6, 0.5))
    cmask = mesh.face_mask(0b000100)
    n = radial_normal(mesh)
    eps_n, eps_t, tol = 0.05, 0.01, 1e-12
    faces = 0b110011
    rng = np.random.default_rng(7)
    psi = rng.uniform(-0.9, 0.9, mesh.ndofs)
    du = np.where(cmask == 0, rng.uniform(-1, 1, mesh.ndofs), 0.0)
    # the diffusive part is linear in psi: rhs(psi + du) - rhs(psi) = -tangent(du) + compressive change
    zero_c = lambda p: wetting_rhs(mesh, cmask, faces, eps_n, eps_t, n, tol, p)  # noqa: E731
    e = 1e-6
    fd = (zero_c(psi + e * du) - zero_c(psi - e * du)) / (2 * e)
    tan = wetting_tangent_apply(mesh, cmask, faces, eps_n, eps_t, n, tol, du)
    comp = fd + tan  # what is left is the derivative of the compressive flux, int -psi du n.n_f phi
    assert np.all(comp[cmask != 0] == 0) and np.all(tan[cmask != 0] == 0)
    assert np.max(np.abs(comp)) > 1e-3 * np.max(np.abs(tan))
    # at psi = 0 that derivative vanishes (c'(0) = 0), so the tangent is minus the rhs derivative
    fd0 = (zero_c(e * du) - zero_c(-e * du)) / (2 * e)
    assert np.max(np.abs(fd0 + tan)) <= 1e-8 * np.max(np.abs(tan))
    # a constant psi = p on one face: only c(p) n.n_f is left; its sum is c(p) times the flux of n
    p = 0.3
    a = np.array([0.6, 0.0, 0.8])
    const = [np.full(mesh.ndofs, c) for c in a]
    r = wetting_rhs(mesh, None, 1 << 1, eps_n, eps_t, const, tol, np.full(mesh.ndofs, p))
    assert abs(r.sum() - 0.5 * (1 - p * p) * a[0] * 0.6 * 0.5) <= 1e-14
    r = wetting_rhs(mesh, None, 1 << 4, eps_n, eps_t, const, tol, np.full(mesh.ndofs, p))
    assert abs(r.sum() + 0.5 * (1 - p * p) * a[2] * 0.9 * 0.6) <= 1e-14


def _sub_box(degree, m, length, cells_x):
    """The box of the first cells_x cell layers in x and the lattice indices of its DoFs in the full
    mesh."""
    h = length[0] / m[0]
    sub = Mesh(degree, (cells_x, m[1], m[2]), length=(cells_x * h, length[1], length[2]))
    n_full = [degree * c + 1 for c in m]
    nx = degree * cells_x + 1
    i, j, k = np.meshgrid(np.arange(nx), np.arange(n_full[1]), np.arange(n_full[2]), indexing="ij")
    order = np.argsort((i + nx * (j + n_full[1] * k)).ravel())
    full = (i + n_full[0] * (j + n_full[1] * k)).ravel()[order]
    return sub, full, h


@pytest.mark.parametrize("degree", [1, 2])
def test_narrow_band_is_the_operator_on_the_band(degree):
    """A level set x and a band |x| < 2 h: every Gauss point of the first two cell layers is inside,
    every other one outside, so the masked projection operator and right-hand sides equal the
    unmasked ones of the two-layer box (the C++ oracle's heat operator for M + damping K)."""
    from oracle.reinit import curvature_rhs, normal_rhs, projection_apply

    m, length, damping = (5, 3, 2), (1.0, 0.6, 0.4), 0.02
    mesh = Mesh(degree, m, length=length)
    sub, full, h = _sub_box(degree, m, length, 2)
    X, Y, Z = mesh.coords()
    rng = np.random.default_rng(9)
    u = rng.uniform(-1, 1, mesh.ndofs)
    # without a band the projection operator is the heat operator with rho_cp = dt = 1, k = damping
    cmask = mesh.face_mask(0b001000)
    o = Operator(mesh, "heat", cmask=cmask, rho_cp=1.0, dt=1.0, k=damping)
    ou = o.vmult(u)
    assert np.max(np.abs(projection_apply(mesh, cmask, damping, u) - ou)) <= 1e-12 * np.max(np.abs(ou))
    got = projection_apply(mesh, None, damping, u, level_set=X, narrow_band=2 * h)
    ref = np.zeros(mesh.ndofs)
    ref[full] = Operator(sub, "heat", rho_cp=1.0, dt=1.0, k=damping).vmult(u[full])
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    # the normal rhs of the level set x and the curvature rhs of a smooth normal field, banded by x
    band = 2 * h
    got = normal_rhs(mesh, None, X, narrow_band=band)
    sX = sub.coords()[0]
    for d in range(3):
        ref = np.zeros(mesh.ndofs)
        ref[full] = normal_rhs(sub, None, sX)[d]
        assert np.max(np.abs(got[d] - ref)) <= 1e-13
    normal = [1.0 + 0.2 * Y, Z - 0.3 * X, X * Y + 0.1]
    got = curvature_rhs(mesh, None, normal, 1e-10, level_set=X, narrow_band=band)
    ref = np.zeros(mesh.ndofs)
    ref[full] = curvature_rhs(sub, None, [c[full] for c in normal], 1e-10)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    # a band wider than the level set's range masks nothing
    wide = curvature_rhs(mesh, None, normal, 1e-10, level_set=X, narrow_band=10.0)
    assert np.array_equal(wide, curvature_rhs(mesh, None, normal, 1e-10))
