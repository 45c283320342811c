"""SUPG-stabilised advection-diffusion operator on the GPU (C ABI) against the oracle: the cell
oracle plus oracle/supg.py; vmult (FP64, FP32), create_rhs, the inverse diagonal and a GMRES solve."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from oracle.oracle import Operator as OOp
from oracle.supg import supg_apply, supg_diagonal
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu

VEL = [0.1, 0.2, -0.3, 0.0, -1.0, 0.3, 1.0, 0.1, 0.0, 0.2, 0.1, -0.2]
CASES = [(1, (9, 8, 9), 0b010011, 1.0, 1e-3, -1.0), (1, (17, 5, 3), 0, 0.5, 0.0, 0.3),
         (2, (9, 8, 5), 0b010011, 1.0, 1e-3, -1.0), (2, (16, 16, 16), 0b001001, 0.5, 2e-3, 0.25),
         (2, (6, 7, 5), 0, 1.0, 1e-2, -1.0), (3, (5, 4, 3), 0b000011, 1.0, 1e-3, -1.0)]


def supg_pair(degree, m, faces, theta, eps, coef, dt=5e-3):
    from meltpooldg_b200.operators import AdvectionDiffusionOperator

    om, gm, cm = meshes(degree, m, faces=faces, origin=(0.0, 0.1, -0.2), length=(1.0, 0.9, 1.1))
    o = OOp(om, "advdiff", cmask=cm, dt=dt, theta=theta, eps=eps, vel=VEL)
    g = AdvectionDiffusionOperator(gm, dt=dt, theta=theta, diffusivity=eps, velocity=VEL)
    g.set_convection_stabilization("SUPG", coef)
    return o, g, om, cm


@pytest.mark.parametrize("degree,m,faces,theta,eps,coef", CASES)
def test_supg_vmult_matches_oracle(degree, m, faces, theta, eps, coef):
    import torch

    dt = 5e-3
    o, g, om, cm = supg_pair(degree, m, faces, theta, eps, coef, dt)
    x = uniform_dofs(om, seed=11)
    ref = o.vmult(x) + supg_apply(om, cm, VEL, coef, 1.0 / dt, theta, theta * eps, x)
    xd = to_gpu(x)
    yd = torch.full_like(xd, np.nan)
    g.vmult(yd, xd)
    assert rel_err(yd.cpu().numpy(), ref) <= 1e-12
    x32 = to_gpu(x, torch.float32)
    y32 = torch.empty_like(x32)
    g.vmult(y32, x32)
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6
    assert g.device_errors() == 0


@pytest.mark.parametrize("degree,m,faces,theta,eps,coef", CASES)
def test_supg_create_rhs_and_diagonal(degree, m, faces, theta, eps, coef):
    import torch

    dt = 5e-3
    o, g, om, cm = supg_pair(degree, m, faces, theta, eps, coef, dt)
    u_old = uniform_dofs(om, seed=13)
    ref = uniform_dofs(om, seed=14)
    dst = to_gpu(ref)
    o.create_rhs(ref, u_old)
    ref += supg_apply(om, cm, VEL, coef, 1.0 / dt, theta - 1.0, (theta - 1.0) * eps, u_old, plain=True)
    g.create_rhs(dst, to_gpu(u_old))
    assert rel_err(dst.cpu().numpy(), ref) <= 1e-12
    d = o.diagonal() + supg_diagonal(om, cm, VEL, coef, 1.0 / dt, theta, theta * eps)
    linf = max(1.0, np.max(np.abs(d)))
    inv = np.where(np.abs(d) > 1e-14 * linf, 1.0 / d, 1.0)
    dd = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(dd)
    # the SUPG entries are sums over 27 x 27 quadrature terms of both signs
    assert rel_err(dd.cpu().numpy(), inv) <= 1e-11
    d32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(d32)
    assert rel_err(d32.cpu().numpy(), inv) <= 1e-6  # FP64 diagonal rounded once


def test_supg_gmres_reaches_the_oracle_residual():
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    # tau_c = 0.1 h_c: with tau_c = h_c / max |v| this velocity (slow near its rotation axis) and
    # dt = 5e-3 make the symmetric part of the operator indefinite, and Jacobi-GMRES(30) stalls on the
    # oracle's matrix as well
    dt, theta, eps, coef = 5e-3, 1.0, 1e-3, 0.1
    o, g, om, cm = supg_pair(2, (12, 10, 9), 0b010011, theta, eps, coef, dt)
    b = uniform_dofs(om, seed=15)
    b[cm != 0] = 0.0
    x = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    LinearSolver.solve(g, x, to_gpu(b), LinearSolverData("GMRES", "Diagonal", max_iterations=2000, rel_tolerance=1e-10))
    xs = x.cpu().numpy()
    r = b - o.vmult(xs) - supg_apply(om, cm, VEL, coef, 1.0 / dt, theta, theta * eps, xs)
    assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(b)
    # switching the stabilisation off gives back the plain operator
    g.set_convection_stabilization("none")
    y = torch.empty_like(x)
    g.vmult(y, x)
    assert rel_err(y.cpu().numpy(), o.vmult(xs)) <= 1e-12


def test_supg_mixed_precision_solve():
    """FP32 GMRES inside FP64 defect correction on the stabilised operator reaches the oracle residual."""
    import torch

    from meltpooldg_b200.operators import LinearSolver

    dt, theta, eps, coef = 5e-3, 1.0, 1e-3, 0.1
    o, g, om, cm = supg_pair(2, (12, 10, 9), 0b010011, theta, eps, coef, dt)
    b = uniform_dofs(om, seed=16)
    b[cm != 0] = 0.0
    x = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    LinearSolver.solve_mixed(g, x, to_gpu(b), outer_rel_tol=1e-9, inner_rel_tol=1e-3, solver="GMRES")
    xs = x.cpu().numpy()
    r = b - o.vmult(xs) - supg_apply(om, cm, VEL, coef, 1.0 / dt, theta, theta * eps, xs)
    assert np.linalg.norm(r) <= 2e-9 * np.linalg.norm(b)


FIELD_CASES = [(1, (9, 7, 5), 0b010011, 1.0, 1e-3, -1.0), (2, (8, 9, 6), 0b010011, 0.5, 2e-3, -1.0),
               (2, (12, 10, 9), 0, 1.0, 1e-3, 0.3), (3, (5, 4, 3), 0b000011, 1.0, 1e-3, -1.0)]


@pytest.mark.parametrize("degree,m,faces,theta,eps,coef", FIELD_CASES)
def test_supg_with_velocity_field_matches_oracle(degree, m, faces, theta, eps, coef):
    """SUPG with the velocity as a DoF vector (the reference's advection_velocity read plainly per cell,
    advection_diffusion_operator.cpp:461-466, also in tau_c's max_q |v|, :510-520): vmult (FP64, FP32),
    create_rhs, the inverse diagonal and a GMRES solve against oracle/advection_field.py plus
    oracle/supg.py, with a non-affine field."""
    import torch

    from meltpooldg_b200.operators import AdvectionDiffusionOperator, LinearSolver, LinearSolverData
    from oracle import advection_field as AF

    dt = 5e-3
    om, gm, cm = meshes(degree, m, faces=faces, length=(1.0, 0.8, 1.1))
    X, Y, Z = om.coords()
    field = [np.sin(3.0 * Y) * (Z + 0.2) + 0.3, np.cos(2.0 * X) - Z * Z, 0.5 * X * Y - 0.1]
    g = AdvectionDiffusionOperator(gm, dt=dt, theta=theta, diffusivity=eps)
    g.set_velocity_field(*[to_gpu(c) for c in field])
    g.set_convection_stabilization("SUPG", coef)

    def tangent(u, c=coef):
        return AF.tangent_apply(om, cm, field, dt, theta, eps, u) + supg_apply(
            om, cm, None, c, 1.0 / dt, theta, theta * eps, u, field=field)

    u = uniform_dofs(om, seed=15)
    ref = tangent(u)
    y = torch.full((om.ndofs,), np.nan, dtype=torch.float64, device="cuda")
    g.vmult(y, to_gpu(u))
    assert rel_err(y.cpu().numpy(), ref) <= 1e-12
    y32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.vmult(y32, to_gpu(u, torch.float32))
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6
    r = torch.zeros_like(y)
    g.create_rhs(r, to_gpu(u))
    rref = AF.create_rhs(om, cm, field, dt, theta, eps, u) + supg_apply(
        om, cm, None, coef, 1.0 / dt, theta - 1.0, (theta - 1.0) * eps, u, plain=True, field=field)
    assert rel_err(r.cpu().numpy(), rref) <= 1e-12
    d = AF.diagonal(om, cm, field, dt, theta, eps) + supg_diagonal(om, cm, None, coef, 1.0 / dt, theta,
                                                                    theta * eps, field=field)
    linf = max(1.0, np.max(np.abs(d)))
    inv = np.where(np.abs(d) > 1e-14 * linf, 1.0 / d, 1.0)
    dd = torch.empty_like(y)
    g.compute_inverse_diagonal_from_matrixfree(dd)
    assert rel_err(dd.cpu().numpy(), inv) <= 1e-11
    d32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(d32)
    assert rel_err(d32.cpu().numpy(), inv) <= 1e-6
    # the solve with tau_c = 0.1 h_c: with h_c / max |v| (or 0.3 h_c at k = 2) the symmetric part of
    # this operator is indefinite and Jacobi-GMRES(30) stalls on the oracle's matrix as well
    g.set_convection_stabilization("SUPG", 0.1)
    b = uniform_dofs(om, seed=16, cmask=cm)
    x = torch.zeros_like(y)
    LinearSolver.solve(g, x, to_gpu(b), LinearSolverData("GMRES", "Diagonal", max_iterations=2000, rel_tolerance=1e-10))
    res = b - tangent(x.cpu().numpy(), 0.1)
    assert np.linalg.norm(res) <= 2e-10 * np.linalg.norm(b)
    assert g.device_errors() == 0


def test_supg_affine_field_is_the_affine_supg_operator():
    """An affine field sampled at the support points gives the affine SUPG operator on the GPU."""
    import torch

    from meltpooldg_b200.operators import AdvectionDiffusionOperator

    o, ga, om, cm = supg_pair(2, (9, 8, 5), 0b010011, 1.0, 1e-3, -1.0)
    X, Y, Z = om.coords()
    aff = [VEL[k] + VEL[3 + 3 * k] * X + VEL[4 + 3 * k] * Y + VEL[5 + 3 * k] * Z for k in range(3)]
    _, gm, _ = meshes(2, (9, 8, 5), faces=0b010011, origin=(0.0, 0.1, -0.2), length=(1.0, 0.9, 1.1))
    gf = AdvectionDiffusionOperator(gm, dt=5e-3, theta=1.0, diffusivity=1e-3)
    gf.set_velocity_field(*[to_gpu(c) for c in aff])
    gf.set_convection_stabilization("SUPG", -1.0)
    u = to_gpu(uniform_dofs(om, seed=17))
    ya, yf = torch.empty_like(u), torch.empty_like(u)
    ga.vmult(ya, u)
    gf.vmult(yf, u)
    assert rel_err(yf.cpu().numpy(), ya.cpu().numpy()) <= 1e-12
