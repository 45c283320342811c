"""Heat operator on the GPU (C ABI) against the CPU oracle."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import normal_cells, uniform_dofs
from oracle.oracle import Operator as OOp
from oracle.oracle import solve as osolve
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu

CASES = [(1, (5, 3, 4)), (1, (17, 9, 9)), (2, (9, 8, 5)), (2, (16, 16, 16)), (3, (5, 4, 6)),
         (4, (5, 6, 4)), (4, (8, 8, 8))]


def heat_pair(degree, m, faces=0b111111, kfield=True, rho_cp=1.3, dt=1e-2, k=1.0, length=(1, 1, 1)):
    from meltpooldg_b200.operators import HeatDiffuseOperator

    om, gm, cm = meshes(degree, m, faces=faces, length=length)
    kc = np.exp(normal_cells(om, seed=2, sigma=0.5)) if kfield else None
    o = OOp(om, "heat", cmask=cm, rho_cp=rho_cp, dt=dt, k=k, k_cell=kc)
    g = HeatDiffuseOperator(gm, rho_cp=rho_cp, dt=dt, conductivity=k, conductivity_cells=kc)
    return o, g, om, cm


@pytest.mark.parametrize("degree,m", CASES)
def test_vmult_fp64_matches_oracle(degree, m):
    import torch

    o, g, om, cm = heat_pair(degree, m, length=(1.0, 0.8, 1.2))
    x = uniform_dofs(om, seed=1)
    y_ref = o.vmult(x)
    xd = to_gpu(x)
    yd = torch.full_like(xd, np.nan)
    g.vmult(yd, xd)
    torch.cuda.synchronize()
    assert rel_err(yd.cpu().numpy(), y_ref) <= 1e-12
    # twice in a row (tickets, flags and epochs reset correctly)
    g.vmult(yd, xd)
    assert rel_err(yd.cpu().numpy(), y_ref) <= 1e-12
    assert g.device_errors() == 0


@pytest.mark.parametrize("degree,m", CASES)
def test_vmult_fp32_matches_oracle(degree, m):
    import torch

    o, g, om, cm = heat_pair(degree, m)
    x = uniform_dofs(om, seed=3)
    y_ref = o.vmult(x)
    xd = to_gpu(x, torch.float32)
    yd = torch.empty_like(xd)
    g.vmult(yd, xd)
    assert rel_err(yd.cpu().numpy(), y_ref) <= 2e-6


@pytest.mark.parametrize("faces", [0, 0b000001, 0b101010, 0b111111])
def test_constraint_faces(faces):
    import torch

    o, g, om, cm = heat_pair(2, (9, 8, 5), faces=faces)
    x = uniform_dofs(om, seed=5)
    xd = to_gpu(x)
    yd = torch.empty_like(xd)
    g.vmult(yd, xd)
    assert rel_err(yd.cpu().numpy(), o.vmult(x)) <= 1e-12
    if cm is not None:
        assert np.all(yd.cpu().numpy()[cm == 1] == 0.0)


@pytest.mark.parametrize("degree,m", [(1, (6, 5, 4)), (2, (9, 8, 5)), (3, (5, 4, 6)), (4, (5, 6, 4))])
def test_inverse_diagonal(degree, m):
    import torch

    o, g, om, cm = heat_pair(degree, m)
    d = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert rel_err(d.cpu().numpy(), o.inverse_diagonal()) <= 1e-12


def test_vmult_add_and_residual():
    import torch

    o, g, om, cm = heat_pair(2, (9, 8, 5))
    x, b = uniform_dofs(om, seed=1), uniform_dofs(om, seed=2)
    Ax = o.vmult(x)
    xd, bd = to_gpu(x), to_gpu(b)
    acc = bd.clone()
    g.vmult_add(acc, xd, -0.5)
    ref = b - 0.5 * Ax  # constrained rows untouched
    assert rel_err(acc.cpu().numpy(), ref) <= 1e-12
    r = torch.empty_like(xd)
    g.residual(r, bd, xd)
    assert rel_err(r.cpu().numpy(), b - Ax) <= 1e-12
    r2 = bd.clone()
    g.residual(r2, r2, xd)  # in place on b
    assert rel_err(r2.cpu().numpy(), b - Ax) <= 1e-12


@pytest.mark.parametrize("degree", [1, 2, 4])
def test_create_rhs(degree):
    o, g, om, cm = heat_pair(degree, (6, 5, 4))
    T, To, q = (uniform_dofs(om, seed=s) for s in (1, 2, 3))
    ref = uniform_dofs(om, seed=4)
    dst = to_gpu(ref)
    o.create_rhs(ref, T, To, q)
    g.create_rhs(dst, to_gpu(T), to_gpu(To), to_gpu(q))
    assert rel_err(dst.cpu().numpy(), ref) <= 1e-12


def test_zero_time_increment_raises():
    from meltpooldg_b200.operators import ZeroTimeIncrement

    o, g, om, cm = heat_pair(2, (4, 4, 4))
    with pytest.raises(ZeroTimeIncrement):
        g.reset_time_increment(0.0)


@pytest.mark.parametrize("solver", ["CG", "GMRES"])
def test_solve_config1(solver):
    """C1: 16^3 Q2, dt 1e-2, k 1, rho c_p 1, homogeneous Dirichlet, Jacobi, rel 1e-10."""
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    o, g, om, cm = heat_pair(2, (16, 16, 16), kfield=False, rho_cp=1.0, dt=1e-2, k=1.0)
    b = uniform_dofs(om, seed=1, cmask=cm)
    x_ref = np.zeros(om.ndofs)
    it_ref, _ = osolve(o, x_ref, b, solver.lower(), inv_diag=o.inverse_diagonal(), rel_tol=1e-10)
    xd = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    st = LinearSolver.solve(g, xd, to_gpu(b), LinearSolverData(solver, "Diagonal", rel_tolerance=1e-10),
                            history=True)
    assert abs(st.iterations - it_ref) <= 1
    assert rel_err(xd.cpu().numpy(), x_ref) <= 1e-8
    assert st.history[-1] <= 1e-10 * st.history[0]


def test_cg_not_converged_raises():
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData, NoConvergence

    o, g, om, cm = heat_pair(2, (8, 8, 8))
    b = uniform_dofs(om, seed=1, cmask=cm)
    xd = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    with pytest.raises(NoConvergence):
        LinearSolver.solve(g, xd, to_gpu(b), LinearSolverData("CG", "Diagonal", max_iterations=3))


def test_mixed_precision_matches_fp64_oracle():
    import torch

    from meltpooldg_b200.operators import LinearSolver

    o, g, om, cm = heat_pair(2, (16, 16, 16), dt=1e-3)
    b = uniform_dofs(om, seed=3, cmask=cm)
    x_ref = np.zeros(om.ndofs)
    osolve(o, x_ref, b, "cg", inv_diag=o.inverse_diagonal(), rel_tol=1e-12)
    xd = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    st = LinearSolver.solve_mixed(g, xd, to_gpu(b), outer_rel_tol=1e-8, inner_rel_tol=1e-4)
    assert st.final_residual <= 1e-8 * np.linalg.norm(b)
    assert np.linalg.norm(xd.cpu().numpy() - x_ref) <= 1e-7 * np.linalg.norm(x_ref)


def test_vmult_host_buffers():
    o, g, om, cm = heat_pair(4, (5, 6, 4))
    x = uniform_dofs(om, seed=8)
    y = np.zeros_like(x)
    g.vmult_host(y, x)
    assert rel_err(y, o.vmult(x)) <= 1e-12


@pytest.mark.parametrize("zero_out", [True, False])
def test_create_rhs_and_apply_dirichlet(zero_out):
    """rhs = -A_noBC x_D + create_rhs(T, T_old, q) on free rows, 0 on constrained rows."""
    o, g, om, cm = heat_pair(2, (9, 8, 5), faces=0b100111)
    T, To, q, xd = (uniform_dofs(om, seed=s) for s in (41, 42, 43, 44))
    x_D = np.where(cm == 1, xd, 0.0)
    ref = -o.with_(cmask=None).vmult(x_D)
    o.with_(cmask=None).create_rhs(ref, T, To, q)
    start = uniform_dofs(om, seed=45)
    if not zero_out:
        ref = ref + start
    ref[cm == 1] = 0.0
    rhs = to_gpu(start)
    g.create_rhs_and_apply_dirichlet(rhs, to_gpu(T), to_gpu(xd), b=to_gpu(To), c=to_gpu(q), zero_out=zero_out)
    assert rel_err(rhs.cpu().numpy(), ref) <= 1e-12
