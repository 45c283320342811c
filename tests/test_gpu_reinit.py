"""Conservative level-set reinitialisation operator (Olsson) on the GPU against oracle/reinit.py,
through the C ABI: vmult (FP64, FP32), create_rhs (overwriting), the inverse diagonal, a CG solve
and the argument checks."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from oracle.reinit import create_rhs, diagonal, tangent_apply
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu

CASES = [(1, (9, 7, 5), 0b000001), (2, (9, 8, 5), 0b010011), (2, (16, 16, 16), 0), (1, (17, 5, 3), 0),
         (3, (5, 4, 3), 0b001100)]
EPS_N, EPS_T, DT, TOL = 0.05, 0.01, 1e-2, 1e-3


def setup(degree, m, faces):
    from meltpooldg_b200.operators import OlssonOperator

    om, gm, cm = meshes(degree, m, faces=faces, length=(1.0, 0.9, 1.1))
    X, Y, Z = om.coords()
    # radial normal field through the domain (zero length at its centre: the tolerance branch)
    normal = [X - 0.5, Y - 0.45, Z - 0.55]
    g = OlssonOperator(gm, dt=DT, eps_normal=EPS_N, eps_tangential=EPS_T, normal_tolerance=TOL)
    nd = [to_gpu(c) for c in normal]
    g.set_normal(*nd)
    return g, om, cm, normal, nd


@pytest.mark.parametrize("degree,m,faces", CASES)
def test_reinit_vmult_matches_oracle(degree, m, faces):
    import torch

    g, om, cm, normal, keep = setup(degree, m, faces)
    x = uniform_dofs(om, seed=1)
    ref = tangent_apply(om, cm, DT, EPS_N, EPS_T, normal, TOL, x)
    xd = to_gpu(x)
    yd = torch.full_like(xd, np.nan)
    g.vmult(yd, xd)
    assert rel_err(yd.cpu().numpy(), ref) <= 1e-12
    y32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.vmult(y32, to_gpu(x, torch.float32))
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6


@pytest.mark.parametrize("degree,m,faces", CASES)
def test_reinit_create_rhs_and_diagonal(degree, m, faces):
    import torch

    g, om, cm, normal, keep = setup(degree, m, faces)
    psi = np.tanh(4.0 * uniform_dofs(om, seed=3))
    ref = create_rhs(om, cm, EPS_N, EPS_T, normal, TOL, psi)
    dst = to_gpu(uniform_dofs(om, seed=4))  # overwritten
    g.create_rhs(dst, to_gpu(psi))
    assert rel_err(dst.cpu().numpy(), ref) <= 1e-12
    d = diagonal(om, cm, DT, EPS_N, EPS_T, normal, TOL)
    if cm is not None:
        d[cm != 0] = 1.0
    linf = max(1.0, np.max(np.abs(d)))
    inv = np.where(np.abs(d) > 1e-14 * linf, 1.0 / d, 1.0)
    dd = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(dd)
    assert rel_err(dd.cpu().numpy(), inv) <= 1e-12


def test_reinit_cg_reaches_the_oracle_residual():
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    g, om, cm, normal, keep = setup(2, (12, 10, 9), 0b010011)
    b = uniform_dofs(om, seed=9)
    b[cm != 0] = 0.0
    x = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    LinearSolver.solve(g, x, to_gpu(b), LinearSolverData("CG", "Diagonal", max_iterations=2000, rel_tolerance=1e-10))
    xs = x.cpu().numpy()
    r = b - tangent_apply(om, cm, DT, EPS_N, EPS_T, normal, TOL, xs)
    assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(b)


def test_reinit_argument_checks():
    import torch

    from meltpooldg_b200._lib import MPDG_ERR_ARG, MPDG_ERR_UNSUPPORTED, MpdgError
    from meltpooldg_b200.operators import Mesh, OlssonOperator

    with pytest.raises(MpdgError) as e:
        OlssonOperator(Mesh(4, (2, 2, 2)), dt=1e-2, eps_normal=0.1, eps_tangential=0.1)
    assert e.value.code == MPDG_ERR_UNSUPPORTED
    g = OlssonOperator(Mesh(1, (4, 4, 4)), dt=1e-2, eps_normal=0.1, eps_tangential=0.1)
    x = torch.zeros(g.n_dofs, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    with pytest.raises(MpdgError) as e:
        g.vmult(y, x)  # no normal field yet
    assert e.value.code == MPDG_ERR_ARG
    g.set_normal(x + 1.0, x, x)
    g.vmult(y, x)


@pytest.mark.parametrize("degree,m,faces", [(1, (9, 7, 5), 0), (2, (9, 8, 5), 0b010011), (2, (16, 16, 16), 0),
                                            (3, (4, 5, 3), 0b000011)])
def test_level_set_rhs_and_normal_projection(degree, m, faces):
    """The normal-vector and curvature right-hand sides against the oracle, and the normal projection
    (M + damping K) n_d = rhs_d solved with a heat operator (rho_cp = dt = 1, k = damping)."""
    import torch

    from meltpooldg_b200.operators import HeatDiffuseOperator, LinearSolver, LinearSolverData
    from oracle.oracle import Operator as OOp
    from oracle.reinit import curvature_rhs, normal_rhs

    om, gm, cm = meshes(degree, m, faces=faces, length=(1.0, 0.9, 1.1))
    X, Y, Z = om.coords()
    dist = np.sqrt((X - 0.5) ** 2 + (Y - 0.45) ** 2 + (Z - 0.55) ** 2) - 0.3
    psi = np.tanh(dist / 0.05)
    damping = 4e-3
    g = HeatDiffuseOperator(gm, rho_cp=1.0, dt=1.0, conductivity=damping)
    # the normalised gradient is checked on a field whose gradient never vanishes: far from the
    # interface the tanh profile's gradient is at the rounding level of psi (and the distance
    # function's interpolant has cells where it cancels by symmetry), so its direction is noise there
    smooth = 0.8 * X - 0.5 * Y + 0.3 * Z + 0.05 * np.sin(3.0 * X) * np.cos(2.0 * Y)
    for normalized, field in ((False, psi), (True, smooth)):
        ref = normal_rhs(om, cm, field, normalized)
        pre = 1e-5 * uniform_dofs(om, seed=11)  # the rhs accumulates (constrained rows keep pre)
        nd = [to_gpu(pre) for _ in range(3)]
        g.level_set_normal_rhs(to_gpu(field), *nd, normalized=normalized)
        for d in range(3):
            assert rel_err(nd[d].cpu().numpy() - pre, ref[d]) <= 1e-11
    # the projection, then the curvature rhs of the projected normal
    o = OOp(om, "heat", cmask=cm, rho_cp=1.0, dt=1.0, k=damping)
    ref = normal_rhs(om, cm, psi)
    normal = []
    for d in range(3):
        b = to_gpu(ref[d])
        x = torch.zeros_like(b)
        LinearSolver.solve(g, x, b, LinearSolverData("CG", "Diagonal", rel_tolerance=1e-12))
        xs = x.cpu().numpy()
        assert np.linalg.norm(ref[d] - o.vmult(xs)) <= 1e-11 * np.linalg.norm(ref[d])
        normal.append(xs)
    c_ref = curvature_rhs(om, cm, normal, 1e-6)
    c = to_gpu(np.full(om.ndofs, 7.0))  # overwritten
    g.level_set_curvature_rhs(c, *[to_gpu(v) for v in normal], normal_tolerance=1e-6)
    assert rel_err(c.cpu().numpy(), c_ref) <= 1e-12


@pytest.mark.parametrize("degree,m,faces", [(1, (9, 7, 5), 0), (2, (8, 7, 6), 0b000011), (3, (5, 4, 4), 0)])
def test_narrow_band_projection_and_rhs(degree, m, faces):
    """Narrow band of the normal-vector / curvature projections (level_set_tools.hpp:357-368) on a
    heat handle used as the projection operator: vmult (FP64, FP32), the inverse diagonal with the
    relative rule, the normal and curvature right-hand sides and a CG solve, against the oracle."""
    import torch

    from meltpooldg_b200.operators import HeatDiffuseOperator, LinearSolver, LinearSolverData
    from oracle.reinit import curvature_rhs, normal_rhs, projection_apply

    om, gm, cm = meshes(degree, m, faces=faces, length=(1.0, 0.9, 1.1))
    X, Y, Z = om.coords()
    psi = np.tanh((np.sqrt((X - 0.5) ** 2 + (Y - 0.45) ** 2 + (Z - 0.55) ** 2) - 0.3) / 0.1)
    band, damping = 0.8, 0.02
    g = HeatDiffuseOperator(gm, rho_cp=1.0, dt=1.0, conductivity=damping)
    psid = to_gpu(psi)
    g.set_narrow_band(psid, band)
    x = uniform_dofs(om, seed=1)
    ref = projection_apply(om, cm, damping, x, level_set=psi, narrow_band=band)
    y = torch.full((om.ndofs,), np.nan, dtype=torch.float64, device="cuda")
    g.vmult(y, to_gpu(x))
    assert rel_err(y.cpu().numpy(), ref) <= 1e-12
    y32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.vmult(y32, to_gpu(x, torch.float32))
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6
    # diagonal by unit vectors of the oracle, relative inversion rule, constrained rows 1
    n = om.ndofs
    dref = np.array([projection_apply(om, cm, damping, np.eye(1, n, i).ravel(), level_set=psi, narrow_band=band)[i]
                     for i in range(n)])
    if cm is not None:
        dref[cm == 1] = 1.0
    thr = 1e-14 * max(1.0, np.max(np.abs(dref)))
    inv = np.where(np.abs(dref) > thr, 1.0 / np.where(dref != 0, dref, 1.0), 1.0)
    d = torch.empty_like(y)
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert rel_err(d.cpu().numpy(), inv) <= 1e-12
    # right-hand sides
    nx, ny, nz = (torch.zeros_like(y) for _ in range(3))
    g.level_set_normal_rhs(psid, nx, ny, nz)
    for got, want in zip((nx, ny, nz), normal_rhs(om, cm, psi, narrow_band=band)):
        assert rel_err(got.cpu().numpy(), want) <= 1e-12
    normal = [X - 0.5, Y - 0.45, Z - 0.55]
    kap = torch.empty_like(y)
    g.level_set_curvature_rhs(kap, *(to_gpu(c) for c in normal), 1e-10)
    assert rel_err(kap.cpu().numpy(), curvature_rhs(om, cm, normal, 1e-10, level_set=psi, narrow_band=band)) <= 1e-12
    # projection solve: the banded operator is only semidefinite (rows outside the band are zero, and
    # cells with few Gauss points in the band add nearly singular terms), so CG converges slowly and
    # amplifies rounding quickly (a 1e-15 perturbation of the right-hand side reaches 1e-3 after 20
    # steps); a fixed number of Jacobi-CG steps (SolverCG's recurrence, restated here on the oracle's
    # operator) must give the same iterate
    from meltpooldg_b200._lib import NoConvergence

    steps = 8
    rhs = nx.clone()
    sol = torch.zeros_like(rhs)
    try:  # a small system may converge within the steps: then compare after as many
        steps = LinearSolver.solve(g, sol, rhs, LinearSolverData("CG", "Diagonal", rel_tolerance=1e-14,
                                                                 max_iterations=steps)).iterations
    except NoConvergence:
        pass
    b = rhs.cpu().numpy()
    xo, r = np.zeros(n), b.copy()
    z = inv * r
    p, rz = z.copy(), float(r @ z)
    for _ in range(steps):
        v = projection_apply(om, cm, damping, p, level_set=psi, narrow_band=band)
        alpha = rz / float(p @ v)
        xo += alpha * p
        r -= alpha * v
        z = inv * r
        rz, rz_old = float(r @ z), rz
        p = z + (rz / rz_old) * p
    assert rel_err(sol.cpu().numpy(), xo) <= 1e-8
    g.set_narrow_band(None, 0.0)
    g.vmult(y, to_gpu(x))
    assert rel_err(y.cpu().numpy(), projection_apply(om, cm, damping, x)) <= 1e-12


@pytest.mark.parametrize("degree,m,faces,wet", [(1, (6, 5, 4), 0, 0b000101), (2, (5, 4, 6), 0b100000, 0b011010),
                                                (2, (7, 6, 5), 0, 0b111111), (3, (4, 3, 4), 0, 0b010110)])
def test_wetting_faces_match_oracle(degree, m, faces, wet):
    """Wetting boundary faces of the reinitialisation operator (olsson_CG_operator.cpp:550-716):
    vmult, create_rhs and the inverse diagonal with the face terms, against oracle/reinit.py."""
    import torch

    from oracle.reinit import wetting_rhs, wetting_tangent_apply

    g, om, cm, normal, keep = setup(degree, m, faces)
    g.set_wetting(wet)
    x = uniform_dofs(om, seed=1)
    ref = tangent_apply(om, cm, DT, EPS_N, EPS_T, normal, TOL, x) + \
        wetting_tangent_apply(om, cm, wet, EPS_N, EPS_T, normal, TOL, x)
    y = torch.full((om.ndofs,), np.nan, dtype=torch.float64, device="cuda")
    g.vmult(y, to_gpu(x))
    assert rel_err(y.cpu().numpy(), ref) <= 1e-12
    psi = np.tanh(uniform_dofs(om, seed=3))
    r = torch.full_like(y, np.nan)
    g.create_rhs(r, to_gpu(psi))
    rref = create_rhs(om, cm, EPS_N, EPS_T, normal, TOL, psi) + wetting_rhs(om, cm, wet, EPS_N, EPS_T, normal, TOL, psi)
    assert rel_err(r.cpu().numpy(), rref) <= 1e-12
    n = om.ndofs
    dw = np.array([wetting_tangent_apply(om, cm, wet, EPS_N, EPS_T, normal, TOL, np.eye(1, n, i).ravel())[i]
                   for i in range(n)])
    dref = diagonal(om, cm, DT, EPS_N, EPS_T, normal, TOL) + dw
    if cm is not None:
        dref[cm == 1] = 1.0
    thr = 1e-14 * max(1.0, np.max(np.abs(dref)))
    inv = np.where(np.abs(dref) > thr, 1.0 / np.where(dref != 0, dref, 1.0), 1.0)
    d = torch.empty_like(y)
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert rel_err(d.cpu().numpy(), inv) <= 1e-12
    g.set_wetting(0)
    g.vmult(y, to_gpu(x))
    assert rel_err(y.cpu().numpy(), tangent_apply(om, cm, DT, EPS_N, EPS_T, normal, TOL, x)) <= 1e-12
