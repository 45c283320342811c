"""Failure detection of the brick handshake, driven on purpose without faulting or hanging the GPU.

The apply kernels take bricks from a ticket counter and wait, bounded, for the flags their lower
neighbour bricks publish.  A ticket counter left at a stale value (as after an aborted launch) makes
the first bricks of a launch go unprocessed, so their upper neighbours' waits run out: the kernel
must return, record its error word, reset the counter for the next launch, and the solvers must
report MPDG_ERR_TIMEOUT.  The waits are shortened for these launches only.
"""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs

SHORT = 4096  # sleeps of about 32 ns: a few hundred microseconds per wait that gives up


def _op(degree, cells):
    from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh

    mesh = Mesh(degree, cells, dirichlet_faces=63)
    return mesh, HeatDiffuseOperator(mesh, rho_cp=1.0, dt=1e-2, conductivity=1.0)


# (degree, cells): two bricks along x (32 cells per brick row for both the column-marching and the
# pencil kernels), so the second brick waits for the first one
CASES = [(2, (64, 4, 8)), (1, (64, 4, 16)), (4, (64, 2, 4))]


@pytest.mark.gpu
@pytest.mark.parametrize("degree,cells", CASES)
def test_stale_ticket_makes_the_wait_give_up(degree, cells):
    import torch

    from meltpooldg_b200 import _lib as L

    mesh, op = _op(degree, cells)
    lib = L.lib()
    assert lib.mpdg_op_n_bricks(op._h) == 2
    x = torch.tensor(uniform_dofs(mesh, seed=1), device="cuda")
    y = torch.empty_like(x)
    ref = torch.empty_like(x)
    op.vmult(ref, x)
    torch.cuda.synchronize()
    assert op.device_errors() == 0
    assert lib.mpdg_op_test_set_wait_limit(op._h, SHORT) == L.MPDG_OK
    assert lib.mpdg_op_test_set_ticket(op._h, 1) == L.MPDG_OK
    op.vmult(y, x)  # brick 1 waits for brick 0, which no CTA takes
    torch.cuda.synchronize()
    code = op.device_errors()
    assert code > 0, "the wait for a flag nothing sets must give up and record its error word"
    assert op.device_errors() == 0  # read and reset
    # the last CTA reset the counter: the next launch is normal again
    assert lib.mpdg_op_test_set_wait_limit(op._h, 0) == L.MPDG_OK
    op.vmult(y, x)
    torch.cuda.synchronize()
    assert op.device_errors() == 0
    # brick faces are summed with atomics, so repeated applies agree to rounding, not bit for bit
    assert torch.max(torch.abs(y - ref)).item() <= 1e-13 * torch.max(torch.abs(ref)).item()


@pytest.mark.gpu
def test_solver_reports_timeout_after_a_wait_gave_up():
    import torch

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    mesh, op = _op(2, (64, 4, 8))
    lib = L.lib()
    from oracle.oracle import Mesh as OMesh

    cm = OMesh(2, (64, 4, 8)).face_mask(63)  # right-hand side zero on the Dirichlet rows
    b = torch.tensor(uniform_dofs(mesh, seed=3, cmask=cm), device="cuda")
    x = torch.zeros_like(b)
    assert lib.mpdg_op_test_set_wait_limit(op._h, SHORT) == L.MPDG_OK
    assert lib.mpdg_op_test_set_ticket(op._h, 1) == L.MPDG_OK
    with pytest.raises(L.MpdgError) as exc:
        LinearSolver.solve(op, x, b, LinearSolverData("CG", "Diagonal", rel_tolerance=1e-8, max_iterations=200))
    assert exc.value.code == L.MPDG_ERR_TIMEOUT
    assert b"bounded device wait" in lib.mpdg_last_error()
    # the handle stays usable: a clean solve afterwards converges without errors
    assert lib.mpdg_op_test_set_wait_limit(op._h, 0) == L.MPDG_OK
    op.device_errors()
    x.zero_()
    st = LinearSolver.solve(op, x, b, LinearSolverData("CG", "Diagonal", rel_tolerance=1e-8))
    assert st.final_residual <= 1e-8 * st.initial_residual
    assert op.device_errors() == 0
    # the wait limit hook rejects a null handle
    assert lib.mpdg_op_test_set_wait_limit(None, 1) == L.MPDG_ERR_ARG
    assert np.isfinite(st.final_residual)
