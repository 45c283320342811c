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
