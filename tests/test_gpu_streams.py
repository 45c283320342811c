"""The C ABI on a non-blocking stream: every host read of device results (norms, solver state,
error words, the inflow detection's copies) is ordered on the operator's stream, so results do not
depend on how far the stream's earlier work has run.  A spin kernel queued on the stream just
before each call keeps that work in flight while the host issues the call."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from tests.gpu_util import meshes

pytestmark = pytest.mark.gpu

SPIN = 20_000_000  # cycles of torch.cuda._sleep: about 10 ms


def test_mixed_and_cg_solves_on_a_busy_non_blocking_stream():
    import torch

    from meltpooldg_b200.operators import HeatDiffuseOperator, LinearSolver, LinearSolverData

    s = torch.cuda.Stream()  # created non-blocking
    om, gm, cm = meshes(2, (48, 40, 36), faces=0b111111)
    b = uniform_dofs(om, seed=41, cmask=cm)
    with torch.cuda.stream(s):
        g = HeatDiffuseOperator(gm, rho_cp=1.0, dt=1e-3, conductivity=1.0, stream=s.cuda_stream)
        bd = torch.tensor(b, device="cuda")
        xs = []
        for _ in range(3):
            x = torch.zeros_like(bd)
            torch.cuda._sleep(SPIN)
            st = LinearSolver.solve_mixed(g, x, bd, outer_rel_tol=1e-10, inner_rel_tol=1e-4, inexact_last=True)
            assert st.history[0] == pytest.approx(np.linalg.norm(b), rel=1e-12)
            xs.append(x.clone())
        for x in xs[1:]:
            assert torch.linalg.norm(x - xs[0]).item() <= 1e-9 * torch.linalg.norm(xs[0]).item()
        r = torch.empty_like(bd)
        g.residual(r, bd, xs[-1])
        s.synchronize()
        assert torch.linalg.norm(r).item() <= 1.01e-10 * np.linalg.norm(b)
        for _ in range(2):
            x = torch.zeros_like(bd)
            torch.cuda._sleep(SPIN)
            st = LinearSolver.solve(g, x, bd, LinearSolverData("CG", "Diagonal", rel_tolerance=1e-10))
            assert st.initial_residual == pytest.approx(np.linalg.norm(b), rel=1e-12)
        torch.cuda._sleep(SPIN)
        assert g.device_errors() == 0
