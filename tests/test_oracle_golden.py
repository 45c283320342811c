"""The CPU oracle reproduces the reference's own golden application logs."""
import json
import os

import numpy as np

from oracle.oracle import Operator, inflow_dofs, solve
from tests.cases import heat_unidirectional, vortex, vortex_inflow, vortex_supg

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_logs.json")))


def test_heat_unidirectional_log():
    """Newton + GMRES(Jacobi) time loop; norms printed to 6 digits must agree exactly."""
    mesh, T = heat_unidirectional()
    op = Operator(mesh, "heat", rho_cp=1.0, dt=1e-4, k=1.0)
    zero = np.zeros(mesh.ndofs)
    got = []
    for _ in range(5):
        T_old = T.copy()
        for _newton in range(10):  # NewtonRaphsonSolver::solve, newton_raphson_solver.cpp:22-80
            rhs = np.zeros(mesh.ndofs)
            op.create_rhs(rhs, T, T_old, zero)
            d = np.zeros(mesh.ndofs)
            solve(op, d, rhs, "gmres", inv_diag=op.inverse_diagonal(), rel_tol=1e-12)
            if np.linalg.norm(rhs) < 5e-9 and np.linalg.norm(d) < 1e-10:
                break
            T += d
        got.append("%.5e" % op.l2_norm(T))
    assert got == GOLD["heat_unidirectional_2d_q1"]["values"]


def _vortex_norms(dim):
    mesh, phi, mask, vel = vortex(dim)
    op = Operator(mesh, "advdiff", cmask=mask, dt=0.01, theta=0.5, eps=0.0, vel=vel)
    nobc = op.with_(cmask=None)
    out = []
    for _ in range(5):
        old = phi.copy()
        bc = np.where(mask == 1, -1.0, 0.0)  # create_rhs_and_apply_dirichlet_matrixfree
        rhs = -nobc.vmult(bc)
        nobc.create_rhs(rhs, old)
        rhs[mask == 1] = 0.0
        x = old.copy()
        solve(op, x, rhs, "gmres", inv_diag=op.inverse_diagonal(), rel_tol=1e-12)
        x[mask == 1] = -1.0
        phi = x
        out.append(op.l2_norm(phi))
    return np.array(out)


# The logs print 11 digits, but the reference computes the norm from per-cell values stored in
# single precision: MeltPoolDG::VectorTools::compute_global_error_norm collects
# dealii::VectorTools::integrate_difference into a dealii::Vector<float>
# (source/utilities/vector_tools.cpp:151-165) and dealii::VectorTools::compute_global_error sums
# their squares in that vector's type.  Its last printed digits therefore carry float rounding of a
# few 1e-8 relative, in an order set by the MPI partition and the summation tree of the machine that
# wrote the logs; the restatement computes the norm in double and agrees to that float noise.
FLOAT_NORM_NOISE = 5e-8


def test_vortex_logs():
    """Reproduced to the float rounding of the reference's norm (see FLOAT_NORM_NOISE); a dense
    direct solve of the same discrete system agrees with GMRES here to 11 digits, so the solution
    itself is not the source of the remaining difference."""
    for dim, key in ((3, "advdiff_vortex_mf_3d_q1"), (2, "advdiff_vortex_mf_2d_q1")):
        ref = np.array([float(v) for v in GOLD[key]["values"]])
        got = _vortex_norms(dim)
        assert np.max(np.abs(got - ref) / ref) < FLOAT_NORM_NOISE, (got, ref)


def _vortex_inflow_norms(dim):
    """AdvectionDiffusionOperation::solve with inflow/outflow constraints
    (source/level_set/advection_diffusion_operation.cpp:243-296): Dirichlet lifting with the inflow
    values as additional inhomogeneous constraints and the operator's pre/post hooks off, rhs zero
    on the inflow rows, GMRES on the operator with identity inflow rows, then the inflow values set."""
    mesh, phi, vel, faces = vortex_inflow(dim)
    inflow = inflow_dofs(mesh, vel, faces)
    op = Operator(mesh, "advdiff", dt=0.01, theta=0.5, eps=0.0, vel=vel, imask=inflow)
    nobc = op.with_(imask=None)
    out = []
    for _ in range(5):
        old = phi.copy()
        bc = np.where(inflow == 1, -1.0, 0.0)
        rhs = -nobc.vmult(bc)
        nobc.create_rhs(rhs, old)
        rhs[inflow == 1] = 0.0
        x = old.copy()
        solve(op, x, rhs, "gmres", inv_diag=op.inverse_diagonal(), rel_tol=1e-12)
        x[inflow == 1] = -1.0
        phi = x
        out.append(op.l2_norm(phi))
    return np.array(out)


def test_vortex_inflow_outflow_logs():
    for dim, key in ((3, "advdiff_vortex_mf_inflow_outflow_3d_q1"), (2, "advdiff_vortex_mf_inflow_outflow_2d_q1")):
        ref = np.array([float(v) for v in GOLD[key]["values"]])
        got = _vortex_inflow_norms(dim)
        assert np.max(np.abs(got - ref) / ref) < FLOAT_NORM_NOISE, (dim, got, ref)


def supg_vortex_norms(steps=5):
    """The SUPG vortex case restated: the oracle's affine advection operator plus oracle/supg.py, the
    Dirichlet lifting (utilities_matrixfree.hpp:39-100) and right-preconditioned GMRES(30) to 1e-12
    (scipy, the same Krylov space); norms of the 2-D field."""
    import scipy.sparse.linalg as spla

    from oracle import supg as S

    mesh, phi, mask, vel, h = vortex_supg()
    dt, theta, coef = 0.01, 0.5, -1.0
    op = Operator(mesh, "advdiff", cmask=mask, dt=dt, theta=theta, eps=0.0, vel=vel)
    nobc = op.with_(cmask=None)
    n = mesh.ndofs

    def A(u):
        return op.vmult(u) + S.supg_apply(mesh, mask, vel, coef, 1.0 / dt, theta, 0.0, u)

    d = op.diagonal() + S.supg_diagonal(mesh, mask, vel, coef, 1.0 / dt, theta, 0.0)
    d[mask == 1] = 1.0
    thr = 1e-14 * max(1.0, np.max(np.abs(d)))
    inv = np.where(np.abs(d) > thr, 1.0 / d, 1.0)
    out = []
    for _ in range(steps):
        old = phi.copy()
        bc = np.where(mask == 1, -1.0, 0.0)
        rhs = -(nobc.vmult(bc) + S.supg_apply(mesh, None, vel, coef, 1.0 / dt, theta, 0.0, bc))
        nobc.create_rhs(rhs, old)
        rhs += S.supg_apply(mesh, None, vel, coef, 1.0 / dt, theta - 1.0, 0.0, old, plain=True)
        rhs[mask == 1] = 0.0
        Aop = spla.LinearOperator((n, n), matvec=lambda v: A(inv * v))  # right preconditioning
        y, info = spla.gmres(Aop, rhs - A(old), rtol=1e-13, atol=0.0, restart=30, maxiter=1000)
        assert info == 0
        x = old + inv * y
        x[mask == 1] = -1.0
        phi = x
        out.append(op.l2_norm(phi) / np.sqrt(h))
    return np.array(out)


def test_vortex_supg_log():
    """advection_diffusion_vortex_mf_supg.mpirun=4.output: SUPG pinned on the reference's log."""
    ref = np.array([float(v) for v in GOLD["advdiff_vortex_supg_2d_q1"]["values"]])
    got = supg_vortex_norms()
    assert np.max(np.abs(got - ref) / ref) < FLOAT_NORM_NOISE, (got, ref)
