"""Degenerate and ragged inputs on the GPU against the oracle: one-cell meshes and meshes one cell
thick for every apply kernel, fully constrained and zero right-hand sides in the solvers, and the
argument checks of mpdg_op_create (degree, cell counts, lengths, time increment, size limit)."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import normal_cells, uniform_dofs
from oracle.oracle import Operator as OOp
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu

THIN = [(1, 1, 1), (2, 1, 1), (1, 3, 1), (1, 1, 4), (33, 1, 2)]


@pytest.mark.parametrize("degree", [1, 2, 3, 4])
@pytest.mark.parametrize("m", THIN)
@pytest.mark.parametrize("faces", [0, 0b111111, 0b011010])
def test_heat_vmult_on_thin_meshes(degree, m, faces):
    import torch

    from meltpooldg_b200.operators import HeatDiffuseOperator

    om, gm, cm = meshes(degree, m, faces=faces, length=(0.3, 0.5, 0.7))
    kc = np.exp(normal_cells(om, seed=2, sigma=0.5))
    o = OOp(om, "heat", cmask=cm, rho_cp=1.3, dt=1e-2, k=0.8, k_cell=kc)
    g = HeatDiffuseOperator(gm, rho_cp=1.3, dt=1e-2, conductivity=0.8, conductivity_cells=kc)
    x = uniform_dofs(om, seed=1)
    ref = o.vmult(x)
    y = torch.full((om.ndofs,), np.nan, dtype=torch.float64, device="cuda")
    g.vmult(y, to_gpu(x))
    if faces == 0b111111 and max(m) == 1 and degree == 1:
        assert np.all(y.cpu().numpy() == 0)  # every DoF constrained
    else:
        assert rel_err(y.cpu().numpy(), ref) <= 1e-12
    d = torch.empty_like(y)
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert rel_err(d.cpu().numpy(), o.inverse_diagonal()) <= 1e-12
    assert g.device_errors() == 0


@pytest.mark.parametrize("degree", [1, 2])
@pytest.mark.parametrize("m", THIN)
def test_advection_vmult_on_thin_meshes(degree, m):
    import torch

    from meltpooldg_b200.operators import AdvectionDiffusionOperator

    vel = [0.1, 0.2, -0.3, 0.0, -1.0, 0.3, 1.0, 0.1, 0.0, 0.2, 0.1, -0.2]
    om, gm, cm = meshes(degree, m, faces=0b000101, length=(0.3, 0.5, 0.7))
    o = OOp(om, "advdiff", cmask=cm, dt=5e-3, theta=0.5, eps=1e-3, vel=vel)
    g = AdvectionDiffusionOperator(gm, dt=5e-3, theta=0.5, diffusivity=1e-3, velocity=vel)
    x = uniform_dofs(om, seed=3)
    y = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    g.vmult(y, to_gpu(x))
    assert rel_err(y.cpu().numpy(), o.vmult(x)) <= 1e-12


@pytest.mark.parametrize("solver", ["CG", "GMRES"])
def test_solvers_with_nothing_to_solve(solver):
    """A fully constrained mesh (every DoF on a Dirichlet face) and a zero right-hand side: the
    initial residual is 0, so ReductionControl stops at step 0 with x untouched."""
    import torch

    from meltpooldg_b200.operators import HeatDiffuseOperator, LinearSolver, LinearSolverData, Mesh

    for mesh in (Mesh(1, (1, 1, 1), dirichlet_faces=63), Mesh(2, (4, 3, 5))):
        op = HeatDiffuseOperator(mesh, dt=1e-2)
        b = torch.zeros(mesh.ndofs, dtype=torch.float64, device="cuda")
        x = torch.zeros_like(b)
        st = LinearSolver.solve(op, x, b, LinearSolverData(solver, "Diagonal"))
        assert st.iterations == 0
        assert torch.count_nonzero(x).item() == 0
        st = LinearSolver.solve_mixed(op, x, b)
        assert torch.count_nonzero(x).item() == 0


def test_op_create_argument_checks():
    import ctypes as C

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200.operators import AdvectionDiffusionOperator, HeatDiffuseOperator, Mesh

    def code(fn):
        with pytest.raises(L.MpdgError) as e:
            fn()
        return e.value.code

    assert code(lambda: HeatDiffuseOperator(Mesh(5, (2, 2, 2)), dt=1e-2)) == L.MPDG_ERR_UNSUPPORTED
    assert code(lambda: HeatDiffuseOperator(Mesh(0, (2, 2, 2)), dt=1e-2)) == L.MPDG_ERR_UNSUPPORTED
    assert code(lambda: AdvectionDiffusionOperator(Mesh(4, (2, 2, 2)), dt=1e-2)) == L.MPDG_ERR_UNSUPPORTED
    assert code(lambda: HeatDiffuseOperator(Mesh(2, (2, 0, 2)), dt=1e-2)) == L.MPDG_ERR_ARG
    assert code(lambda: HeatDiffuseOperator(Mesh(2, (2, 2, 2), length=(1, -1, 1)), dt=1e-2)) == L.MPDG_ERR_ARG
    assert code(lambda: HeatDiffuseOperator(Mesh(2, (2, 2, 2)), dt=0.0)) == L.MPDG_ERR_ZERO_DT
    # (2 * 1000 + 1)^3 > 2^31 DoFs: refused before any allocation
    assert code(lambda: HeatDiffuseOperator(Mesh(2, (1000, 1000, 1000)), dt=1e-2)) == L.MPDG_ERR_UNSUPPORTED
    assert L.lib().mpdg_op_create(None, None, None) == L.MPDG_ERR_ARG
    assert L.lib().mpdg_op_destroy(None) in (L.MPDG_OK, L.MPDG_ERR_ARG)
    _ = C
