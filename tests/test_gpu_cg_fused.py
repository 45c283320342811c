"""The one-sweep PCG iteration (fused vector updates, preconditioner, apply and dot products) against
the three-pass iteration and the oracle's SolverCG restatement.

Meshes cover whole and partial tiles (32 cells in x, 8 in y), a single cell, thin slabs, Dirichlet on
some faces only, and FP32; iteration counts must agree with the oracle within one and the solutions
with the oracle's to the accuracy the tolerance allows.
"""
import numpy as np
import pytest

from meltpooldg_b200.inputs import normal_cells, uniform_dofs
from oracle.oracle import Operator as OOp
from oracle.oracle import solve as osolve
from tests.gpu_util import meshes, to_gpu

pytestmark = pytest.mark.gpu

CASES = [((16, 16, 16), 63), ((40, 20, 12), 63), ((33, 9, 5), 0b010101), ((1, 1, 1), 63), ((64, 17, 3), 0b111100),
         ((7, 40, 18), 0b001111), ((32, 8, 9), 63)]


def _solve(op, b, fused, dtype, tol, precond="Diagonal"):
    import torch

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    assert L.lib().mpdg_op_set_cg_variant(op._h, 1 if fused else 0) == L.MPDG_OK
    x = torch.zeros(b.numel(), dtype=dtype, device="cuda")
    st = LinearSolver.solve(op, x, b.to(dtype), LinearSolverData("CG", precond, rel_tolerance=tol), history=True)
    return x.double().cpu().numpy(), st


@pytest.mark.parametrize("m,faces", CASES)
def test_fused_cg_matches_three_pass_and_oracle(m, faces):
    from meltpooldg_b200.operators import HeatDiffuseOperator

    import torch

    om, gm, cm = meshes(2, m, faces=faces, length=(1.0, 0.8, 1.3))
    kc = np.exp(normal_cells(om, seed=3, sigma=0.5))
    b = uniform_dofs(om, seed=3, cmask=cm)
    if not np.any(b):
        pytest.skip("every DoF constrained")
    orc = OOp(om, "heat", cmask=cm, rho_cp=1.0, dt=1e-3, k_cell=kc)
    xo = np.zeros(om.ndofs)
    it_o, _ = osolve(orc, xo, b, "cg", orc.inverse_diagonal(), rel_tol=1e-10)
    op = HeatDiffuseOperator(gm, rho_cp=1.0, dt=1e-3, conductivity_cells=kc)
    bd = to_gpu(b)
    xf, sf = _solve(op, bd, True, torch.float64, 1e-10)
    x3, s3 = _solve(op, bd, False, torch.float64, 1e-10)
    assert abs(sf.iterations - it_o) <= 1 and abs(s3.iterations - it_o) <= 1, (sf.iterations, s3.iterations, it_o)
    scale = np.linalg.norm(xo)
    assert np.linalg.norm(xf - xo) <= 1e-8 * scale
    assert np.linalg.norm(xf - x3) <= 1e-8 * scale
    # the residual history is SolverCG's |r_k|
    n = min(len(sf.history), len(s3.history))
    assert np.allclose(sf.history[:n], s3.history[:n], rtol=1e-6, atol=1e-14 * sf.history[0])
    # FP32: same iteration count within a few, solution to FP32 accuracy
    x32, s32 = _solve(op, bd, True, torch.float32, 1e-5)
    assert np.linalg.norm(x32 - xo) <= 1e-4 * scale
    assert op.device_errors() == 0


def test_fused_cg_identity_preconditioner_and_nonzero_guess():
    import torch

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200.operators import HeatDiffuseOperator, LinearSolver, LinearSolverData

    om, gm, cm = meshes(2, (20, 12, 10), faces=63)
    b = uniform_dofs(om, seed=4, cmask=cm)
    orc = OOp(om, "heat", cmask=cm, rho_cp=2.0, dt=1e-2, k=0.5)
    xo = np.zeros(om.ndofs)
    it_o, _ = osolve(orc, xo, b, "cg", None, rel_tol=1e-9)
    op = HeatDiffuseOperator(gm, rho_cp=2.0, dt=1e-2, conductivity=0.5)
    x, st = _solve(op, to_gpu(b), True, torch.float64, 1e-9, precond="Identity")
    assert abs(st.iterations - it_o) <= 1
    assert np.linalg.norm(x - xo) <= 1e-7 * np.linalg.norm(xo)
    # a nonzero initial guess: the residual b - A x0 starts the iteration
    x0 = uniform_dofs(om, seed=5, cmask=cm) * 0.1
    xg = to_gpu(x0)
    L.lib().mpdg_op_set_cg_variant(op._h, 1)
    st2 = LinearSolver.solve(op, xg, to_gpu(b), LinearSolverData("CG", "Diagonal", rel_tolerance=1e-10))
    r = b - orc.vmult(xg.cpu().numpy())
    assert np.linalg.norm(r) <= 1.01e-10 * st2.initial_residual
