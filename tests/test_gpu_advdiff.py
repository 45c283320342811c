"""Advection-diffusion operator on the GPU (C ABI) against the CPU oracle."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from oracle.oracle import Operator as OOp
from oracle.oracle import solve as osolve
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu

VEL_ROT = [0.5, -0.5, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0]  # (-(y-.5), x-.5, 0)
VEL_GEN = [0.1, 0.2, -0.3, 0.0, -1.0, 0.3, 1.0, 0.1, 0.0, 0.2, 0.1, -0.2]


def adv_pair(degree, m, faces=0, mask=None, dt=5e-3, theta=1.0, eps=1e-3, vel=VEL_GEN):
    from meltpooldg_b200.operators import AdvectionDiffusionOperator

    om, gm, cm = meshes(degree, m, faces=faces, mask=mask, origin=(0.0, 0.1, -0.2), length=(1.0, 0.9, 1.1))
    o = OOp(om, "advdiff", cmask=cm, dt=dt, theta=theta, eps=eps, vel=vel)
    g = AdvectionDiffusionOperator(gm, dt=dt, theta=theta, diffusivity=eps, velocity=vel)
    return o, g, om, cm


@pytest.mark.parametrize("degree,m", [(1, (9, 8, 9)), (1, (17, 5, 3)), (2, (9, 8, 5)), (2, (16, 16, 16)), (3, (6, 5, 4)),
                                      (3, (9, 8, 3))])
@pytest.mark.parametrize("theta,eps", [(1.0, 1e-3), (0.5, 0.0)])
def test_vmult_matches_oracle(degree, m, theta, eps):
    import torch

    o, g, om, cm = adv_pair(degree, m, faces=0b010011, theta=theta, eps=eps)
    x = uniform_dofs(om, seed=11)
    y_ref = o.vmult(x)
    xd = to_gpu(x)
    yd = torch.empty_like(xd)
    g.vmult(yd, xd)
    assert rel_err(yd.cpu().numpy(), y_ref) <= 1e-12
    xf = to_gpu(x, torch.float32)
    yf = torch.empty_like(xf)
    g.vmult(yf, xf)
    assert rel_err(yf.cpu().numpy(), y_ref) <= 2e-6
    assert g.device_errors() == 0


@pytest.mark.parametrize("degree,m", [(1, (7, 6, 9)), (2, (5, 7, 4)), (3, (5, 4, 6))])
@pytest.mark.parametrize("theta,eps", [(1.0, 1e-3), (0.5, 0.2)])
def test_inverse_diagonal_closed_form(degree, m, theta, eps):
    """The closed-form diagonal (1-D quadrature moments) against the oracle's unit-vector applies."""
    import torch

    o, g, om, cm = adv_pair(degree, m, faces=0b001001, theta=theta, eps=eps)
    d = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert rel_err(d.cpu().numpy(), o.inverse_diagonal()) <= 1e-12


def test_per_dof_mask_and_diagonal():
    import torch

    om, _, _ = meshes(2, (9, 8, 5))
    mask = (uniform_dofs(om, seed=21) > 0.6).astype(np.uint8)
    o, g, om, cm = adv_pair(2, (9, 8, 5), faces=0b100000, mask=mask)
    x = uniform_dofs(om, seed=12)
    xd = to_gpu(x)
    yd = torch.empty_like(xd)
    g.vmult(yd, xd)
    assert rel_err(yd.cpu().numpy(), o.vmult(x)) <= 1e-12
    d = torch.empty_like(xd)
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert rel_err(d.cpu().numpy(), o.inverse_diagonal()) <= 1e-12


@pytest.mark.parametrize("degree,m", [(2, (9, 8, 5)), (3, (5, 6, 4))])
@pytest.mark.parametrize("theta", [1.0, 0.5])
def test_create_rhs(degree, m, theta):
    o, g, om, cm = adv_pair(degree, m, faces=0b000011, theta=theta)
    u_old = uniform_dofs(om, seed=13)
    ref = uniform_dofs(om, seed=14)
    dst = to_gpu(ref)
    o.create_rhs(ref, u_old)
    g.create_rhs(dst, to_gpu(u_old))
    assert rel_err(dst.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("degree,m", [(2, (12, 12, 12)), (3, (7, 6, 8))])
def test_gmres_solve(degree, m):
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    o, g, om, cm = adv_pair(degree, m, vel=VEL_ROT)
    b = uniform_dofs(om, seed=15)
    x_ref = np.zeros(om.ndofs)
    it_ref, _ = osolve(o, x_ref, b, "gmres", inv_diag=o.inverse_diagonal(), rel_tol=1e-10)
    xd = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    st = LinearSolver.solve(g, xd, to_gpu(b), LinearSolverData("GMRES", "Diagonal", rel_tolerance=1e-10))
    assert abs(st.iterations - it_ref) <= 1
    assert rel_err(xd.cpu().numpy(), x_ref) <= 1e-8


@pytest.mark.parametrize("degree,m,faces", [(1, (9, 7, 5), 0), (2, (8, 9, 6), 0b010011), (2, (33, 5, 4), 0),
                                            (3, (5, 4, 3), 0b000011)])
def test_velocity_field_matches_oracle(degree, m, faces):
    """Advection velocity as a DoF vector (advection_diffusion_operator.cpp:461-466, 475-479): vmult
    (FP64, FP32), create_rhs, the inverse diagonal and a GMRES solve against oracle/advection_field.py,
    and a field sampled from the affine velocity reproduces the affine operator."""
    import torch

    from meltpooldg_b200.operators import AdvectionDiffusionOperator, LinearSolver, LinearSolverData
    from oracle import advection_field as AF
    from tests.gpu_util import meshes, rel_err, to_gpu

    om, gm, cm = meshes(degree, m, faces=faces, length=(1.0, 0.8, 1.1))
    X, Y, Z = om.coords()
    field = [np.sin(3.0 * Y) * (Z + 0.2), np.cos(2.0 * X) - Z * Z, 0.5 * X * Y - 0.1]
    dt, theta, eps = 5e-3, 0.5, 2e-3
    g = AdvectionDiffusionOperator(gm, dt=dt, theta=theta, diffusivity=eps)
    fd = [to_gpu(c) for c in field]
    g.set_velocity_field(*fd)
    u = uniform_dofs(om, seed=1)
    ref = AF.tangent_apply(om, cm, field, dt, theta, eps, u)
    y = torch.full((om.ndofs,), np.nan, dtype=torch.float64, device="cuda")
    g.vmult(y, to_gpu(u))
    assert rel_err(y.cpu().numpy(), ref) <= 1e-12
    y32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.vmult(y32, to_gpu(u, torch.float32))
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6
    r = torch.zeros_like(y)
    g.create_rhs(r, to_gpu(u))
    assert rel_err(r.cpu().numpy(), AF.create_rhs(om, cm, field, dt, theta, eps, u)) <= 1e-12
    d = torch.empty_like(y)
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert rel_err(d.cpu().numpy(), AF.inverse_diagonal(om, cm, field, dt, theta, eps)) <= 1e-12
    b = uniform_dofs(om, seed=2, cmask=cm)
    x = torch.zeros_like(y)
    LinearSolver.solve(g, x, to_gpu(b), LinearSolverData("GMRES", "Diagonal", rel_tolerance=1e-10))
    res = b - AF.tangent_apply(om, cm, field, dt, theta, eps, x.cpu().numpy())
    assert np.linalg.norm(res) <= 1.01e-10 * np.linalg.norm(b)
    # an affine field sampled at the support points is the affine operator
    vel = [0.2, -0.1, 0.05, 0.0, -1.0, 0.3, 1.0, 0.0, -0.2, 0.1, 0.2, 0.0]
    aff = [vel[k] + vel[3 + 3 * k] * X + vel[4 + 3 * k] * Y + vel[5 + 3 * k] * Z for k in range(3)]
    om0 = om
    ga = AdvectionDiffusionOperator(gm, dt=dt, theta=theta, diffusivity=eps, velocity=vel)
    gf = AdvectionDiffusionOperator(gm, dt=dt, theta=theta, diffusivity=eps)
    af = [to_gpu(c) for c in aff]
    gf.set_velocity_field(*af)
    ya, yf = torch.empty_like(y), torch.empty_like(y)
    ga.vmult(ya, to_gpu(u))
    gf.vmult(yf, to_gpu(u))
    assert rel_err(yf.cpu().numpy(), ya.cpu().numpy()) <= 1e-12
    assert om0.ndofs == om.ndofs and g.device_errors() == 0
