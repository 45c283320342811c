"""Parity at the full size of every benchmark workload, against the oracle.

  * heat apply, 64^3 cells FE_Q(4), k = exp(N(0, 0.5^2)) (seed 2), dt 1e-3: vmult to 1e-12;
  * heat solve, 128^3 cells FE_Q(2), k seed 3, b = U[-1,1] seed 3: Jacobi-CG to 1e-8 (iteration count
    within one of the oracle's), and the FP64 CG and the mixed-precision solve run to the tolerance the
    benchmark uses, each compared with the oracle's CG solution to 1e-12;
  * level-set advection-diffusion, 96^3 cells FE_Q(2), 10 implicit-Euler steps of Jacobi-GMRES(30),
    FP64 and FP32-inner / FP64-outer, against 10 oracle GMRES steps;
  * transient heat adjoint, 48^3 cells FE_Q(2), 20 steps, checkpoints every 5: the gradient against
    the oracle's adjoint (every state kept, no checkpointing) and against central differences on 20
    random directions with h = 1e-6.
Inputs are the benchmark's seeded inputs (meltpooldg_b200.inputs), so CPU and GPU see identical
vectors.  The workloads are sized as in the benchmark; the oracle runs on all host threads.
"""
import numpy as np
import pytest

from meltpooldg_b200.inputs import lattice_coords, moving_gaussian, normal_cells, uniform_dofs, unit_directions
from oracle import adjoint as OA
from oracle.oracle import Mesh as OMesh
from oracle.oracle import Operator as OOp
from oracle.oracle import solve as osolve
from tests.gpu_util import rel_err, to_gpu

pytestmark = pytest.mark.gpu

# stopping tolerance of both arms of the 128^3 solve comparison: relative residual 1e-8 bounds the
# error only up to the condition number, so both arms run to the residual that keeps their error
# against the oracle's solution at or below 1e-8
SOLVE_TOL = 5e-10
INNER_TOL = 1e-5  # the inner reduction of the benchmarked mixed solve


def rel2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_heat_apply_q4_64cube():
    import torch

    from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh

    om = OMesh(4, (64, 64, 64))
    kc = np.exp(normal_cells(om, seed=2, sigma=0.5))
    src = uniform_dofs(om, seed=1)
    ref = OOp(om, "heat", cmask=om.face_mask(63), rho_cp=1.0, dt=1e-3, k_cell=kc).vmult(src)
    op = HeatDiffuseOperator(Mesh(4, (64, 64, 64), dirichlet_faces=63), rho_cp=1.0, dt=1e-3, conductivity_cells=kc)
    y = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    op.vmult(y, to_gpu(src))
    assert rel_err(y.cpu().numpy(), ref) <= 1e-12
    y32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    op.vmult(y32, to_gpu(src, torch.float32))
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6
    assert op.device_errors() == 0


@pytest.fixture(scope="module")
def heat_solve_case():
    om = OMesh(2, (128, 128, 128))
    cm = om.face_mask(63)
    kc = np.exp(normal_cells(om, seed=3, sigma=0.5))
    b = uniform_dofs(om, seed=3, cmask=cm)
    orc = OOp(om, "heat", cmask=cm, rho_cp=1.0, dt=1e-3, k_cell=kc)
    x = np.zeros(om.ndofs)
    it, hist = osolve(orc, x, b, "cg", orc.inverse_diagonal(), rel_tol=1e-12, history=True)
    it_1e8 = int(np.argmax(hist <= 1e-8 * hist[0]))
    return dict(mesh=om, kc=kc, b=b, x=x, it_1e8=it_1e8)


def _heat_op(c):
    from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh

    return HeatDiffuseOperator(Mesh(2, (128, 128, 128), dirichlet_faces=63), rho_cp=1.0, dt=1e-3,
                               conductivity_cells=c["kc"])


def test_heat_cg_q2_128cube_iterations(heat_solve_case):
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    c = heat_solve_case
    op = _heat_op(c)
    x = torch.zeros(c["mesh"].ndofs, dtype=torch.float64, device="cuda")
    st = LinearSolver.solve(op, x, to_gpu(c["b"]), LinearSolverData("CG", "Diagonal", rel_tolerance=1e-8))
    assert abs(st.iterations - c["it_1e8"]) <= 1
    assert st.final_residual <= 1e-8 * st.initial_residual
    # a residual of 1e-8 bounds the error by the condition number (about 15 here)
    assert rel2(x.cpu().numpy(), c["x"]) <= 5e-7
    assert op.device_errors() == 0


def test_heat_cg_and_mixed_q2_128cube_error(heat_solve_case):
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    c = heat_solve_case
    op = _heat_op(c)
    bd = to_gpu(c["b"])
    x64 = torch.zeros_like(bd)
    LinearSolver.solve(op, x64, bd, LinearSolverData("CG", "Diagonal", rel_tolerance=SOLVE_TOL))
    xm = torch.zeros_like(bd)
    st = LinearSolver.solve_mixed(op, xm, bd, outer_rel_tol=SOLVE_TOL, inner_rel_tol=1e-4)
    assert st.final_residual <= SOLVE_TOL * st.initial_residual
    e64, em = rel2(x64.cpu().numpy(), c["x"]), rel2(xm.cpu().numpy(), c["x"])
    # the benchmarked arm: inner CG to 1e-5, the last inner solve only as far as the outer tolerance asks
    xi = torch.zeros_like(bd)
    st = LinearSolver.solve_mixed(op, xi, bd, outer_rel_tol=SOLVE_TOL, inner_rel_tol=INNER_TOL, inexact_last=True)
    assert st.final_residual <= SOLVE_TOL * st.initial_residual
    ei = rel2(xi.cpu().numpy(), c["x"])
    print(f"error vs oracle: FP64 CG {e64:.3e}, mixed {em:.3e}, mixed inexact {ei:.3e}")
    assert e64 <= 1e-8 and em <= 1e-8 and ei <= 1e-8
    assert op.device_errors() == 0


def _advection_setup(om):
    X, Y, Z = lattice_coords(om)
    phi0 = 0.5 * (1.0 - np.tanh((np.sqrt((X - 0.5) ** 2 + (Y - 0.75) ** 2 + (Z - 0.5) ** 2) - 0.25) / 0.01))
    vel = [0.5, -0.5, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0]
    return phi0, vel


def test_advection_q2_96cube_10_steps():
    import torch

    from meltpooldg_b200.operators import AdvectionDiffusionOperator, LinearSolver, LinearSolverData, Mesh

    om = OMesh(2, (96, 96, 96))
    phi0, vel = _advection_setup(om)
    orc = OOp(om, "advdiff", rho_cp=1.0, dt=5e-3, theta=1.0, eps=1e-3, vel=vel)
    inv = orc.inverse_diagonal()
    phi = phi0.copy()
    its_orc = []
    for _ in range(10):
        rhs = np.zeros(om.ndofs)
        orc.create_rhs(rhs, phi)
        x = phi.copy()
        it, _ = osolve(orc, x, rhs, "gmres", inv, rel_tol=1e-10)
        its_orc.append(it)
        phi = x
    op = AdvectionDiffusionOperator(Mesh(2, (96, 96, 96)), dt=5e-3, theta=1.0, diffusivity=1e-3, velocity=vel)
    for mode in ("fp64", "mixed"):
        p = to_gpu(phi0)
        rhs = torch.empty_like(p)
        its = []
        for _ in range(10):
            rhs.zero_()
            op.create_rhs(rhs, p)
            x = p.clone()
            if mode == "fp64":
                st = LinearSolver.solve(op, x, rhs, LinearSolverData("GMRES", "Diagonal", rel_tolerance=1e-10))
                its.append(st.iterations)
            else:
                LinearSolver.solve_mixed(op, x, rhs, outer_rel_tol=1e-10, inner_rel_tol=1e-4, solver="GMRES")
            p = x
        err = rel2(p.cpu().numpy(), phi)
        print(f"advection {mode}: error vs oracle after 10 steps {err:.3e}")
        assert err <= 1e-9
        if mode == "fp64":
            assert all(abs(a - b) <= 1 for a, b in zip(its, its_orc)), (its, its_orc)
    assert op.device_errors() == 0


def test_adjoint_q2_48cube_gradient():
    import torch

    from meltpooldg_b200.adjoint import TransientHeatAdjoint
    from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh

    om = OMesh(2, (48, 48, 48))
    cm = om.face_mask(63)
    steps, dt, amp = 20, 1e-3, 100.0
    qhat = moving_gaussian(om, steps, dt)
    z = normal_cells(om, seed=5, sigma=0.3)
    zt = normal_cells(om, seed=6, sigma=0.3)
    op = HeatDiffuseOperator(Mesh(2, (48, 48, 48), dirichlet_faces=63), rho_cp=1.0, dt=dt, conductivity=1.0)
    adj = TransientHeatAdjoint(op, steps, checkpoint_every=5, cg_rel_tol=1e-12)
    qd = to_gpu(qhat)
    target = torch.empty((steps, om.ndofs), dtype=torch.float64, device="cuda")
    adj.forward(to_gpu(zt), qd, amp, target)
    grad = torch.empty(om.ncells, dtype=torch.float64, device="cuda")
    zd = to_gpu(z)
    J, gA, _ = adj.objective_and_gradient(zd, qd, amp, target, grad)
    g = grad.cpu().numpy()
    # the oracle's adjoint with the same target states
    J_o, gz_o, gA_o = OA.gradient(om, cm, 1.0, dt, z, qhat, amp, target.cpu().numpy(), rel_tol=1e-12)
    assert abs(J - J_o) <= 1e-9 * abs(J_o)
    assert rel2(g, gz_o) <= 1e-7
    assert abs(gA - gA_o) <= 1e-7 * abs(gA_o)
    # central differences, h = 1e-6, 20 random unit directions (seed 7)
    h, worst = 1e-6, 0.0
    for d in unit_directions(om.ncells, 20, seed=7):
        dd = to_gpu(d)
        jp, _, _ = adj.objective_and_gradient(zd + h * dd, qd, amp, target)
        jm, _, _ = adj.objective_and_gradient(zd - h * dd, qd, amp, target)
        fd = (jp - jm) / (2 * h)
        worst = max(worst, abs(fd - float(g @ d)) / max(abs(fd), 1e-300))
    print(f"adjoint: central differences on 20 directions, worst relative difference {worst:.3e}")
    assert worst <= 1e-5
    assert op.device_errors() == 0
