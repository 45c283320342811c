"""CPU checks of the Python mirror's host logic (meltpooldg_b200/operators.py, adjoint.py) against a
recording stand-in for the C ABI: every wrapper passes vectors of the right length and type through
to the one entry point it forwards to, and refuses short or mistyped vectors before any call."""
import pytest
import torch

from meltpooldg_b200 import adjoint as A
from meltpooldg_b200 import operators as O

PTR = 4096


class FakeCuda:
    """Duck-typed CUDA tensor: only what the wrappers read."""

    is_cuda = True

    def __init__(self, n, dtype=torch.float64):
        self.n, self.dtype = n, dtype

    def is_contiguous(self):
        return True

    def numel(self):
        return self.n

    def data_ptr(self):
        return PTR


class RecordingLib:
    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        def fn(*args):
            self.calls.append((name, args))
            return 0

        return fn


@pytest.fixture
def rec(monkeypatch):
    r = RecordingLib()
    monkeypatch.setattr(O, "lib", lambda: r)
    monkeypatch.setattr(A, "lib", lambda: r)
    return r


def test_every_wrapper_forwards_checked_vectors(rec):
    mesh = O.Mesh(2, (3, 4, 5))
    n, nc = mesh.ndofs, mesh.ncells
    v = lambda dt=torch.float64: FakeCuda(n, dt)  # noqa: E731
    heat = O.HeatDiffuseOperator(mesh, dt=1e-2)
    adv = O.AdvectionDiffusionOperator(mesh, dt=1e-2)
    ols = O.OlssonOperator(mesh, dt=1e-2, eps_normal=0.1, eps_tangential=0.05)
    rec.calls.clear()
    heat.vmult(v(), v())
    heat.vmult(v(torch.float32), v(torch.float32))
    heat.vmult_add(v(), v(), 0.5)
    heat.residual(v(), v(), v())
    heat.compute_inverse_diagonal_from_matrixfree(v())
    heat.compute_inverse_diagonal_from_matrixfree(v(torch.float32))
    heat.create_rhs(v(), v(), v(), None)
    heat.create_rhs_and_apply_dirichlet(v(), v(), v())
    heat.level_set_normal_rhs(v(), v(), v(), v(), normalized=True)
    heat.level_set_curvature_rhs(v(), v(), v(), v(), 1e-10)
    heat.set_conductivity(FakeCuda(nc))
    heat.set_temperature(v())
    heat.set_old_temperature(v())
    adv.create_rhs(v(), v())
    ols.set_normal(v(), v(), v())
    O.LinearSolver.solve(heat, v(), v(), O.LinearSolverData("CG", "Diagonal"))
    O.LinearSolver.solve(heat, v(torch.float32), v(torch.float32), O.LinearSolverData("CG", "Diagonal"))
    O.LinearSolver.solve_mixed(heat, v(), v())
    adj = A.TransientHeatAdjoint(heat, 3)
    adj.forward(FakeCuda(nc), FakeCuda(3 * n), 1.0, FakeCuda(3 * n))
    adj.objective_and_gradient(FakeCuda(nc), FakeCuda(3 * n), 1.0, FakeCuda(3 * n), FakeCuda(nc))
    A.cell_stiffness_form(heat, v(), v(), FakeCuda(nc))
    names = [c[0] for c in rec.calls if not c[0].startswith("mpdg_last")]
    assert names == [
        "mpdg_op_vmult", "mpdg_op_vmult_f32", "mpdg_op_vmult_add", "mpdg_op_residual",
        "mpdg_op_compute_inverse_diagonal", "mpdg_op_compute_inverse_diagonal_f32", "mpdg_op_create_rhs",
        "mpdg_op_create_rhs_and_apply_dirichlet", "mpdg_level_set_normal_rhs", "mpdg_level_set_curvature_rhs",
        "mpdg_op_set_conductivity", "mpdg_op_set_temperature", "mpdg_op_set_old_temperature",
        "mpdg_op_create_rhs", "mpdg_op_set_reinit", "mpdg_solve", "mpdg_solve_f32", "mpdg_solve_mixed",
        "mpdg_heat_forward", "mpdg_adjoint_heat", "mpdg_heat_cell_stiffness_form"]
    # every vector argument arrived as its device address (None stays None)
    for name, args in rec.calls:
        ptrs = [a for a in args if isinstance(a, int) and a == PTR]
        assert ptrs or name.startswith("mpdg_last"), name


def test_short_or_mistyped_vectors_never_reach_the_library(rec):
    mesh = O.Mesh(1, (4, 4, 4))
    n, nc = mesh.ndofs, mesh.ncells
    heat = O.HeatDiffuseOperator(mesh, dt=1e-2)
    rec.calls.clear()
    bad = [
        (ValueError, lambda: heat.vmult(FakeCuda(n - 1), FakeCuda(n))),
        (TypeError, lambda: heat.vmult(FakeCuda(n, torch.float32), FakeCuda(n))),
        (TypeError, lambda: heat.vmult(FakeCuda(n), FakeCuda(n, torch.float16))),
        (TypeError, lambda: heat.compute_inverse_diagonal_from_matrixfree(FakeCuda(n, torch.float16))),
        (ValueError, lambda: heat.create_rhs(FakeCuda(n), FakeCuda(n), FakeCuda(n // 2))),
        (ValueError, lambda: heat.set_conductivity(FakeCuda(nc - 1))),
        (TypeError, lambda: heat.set_temperature(FakeCuda(n, torch.float32))),
        (TypeError, lambda: O.LinearSolver.solve(heat, FakeCuda(n), FakeCuda(n, torch.float32), O.LinearSolverData())),
        (TypeError, lambda: O.LinearSolver.solve(heat, FakeCuda(n, torch.int64), FakeCuda(n), O.LinearSolverData())),
        (ValueError, lambda: A.TransientHeatAdjoint(heat, 2).forward(FakeCuda(nc), FakeCuda(n), 1.0, FakeCuda(2 * n))),
        (ValueError, lambda: A.cell_stiffness_form(heat, FakeCuda(n), FakeCuda(n), FakeCuda(nc - 1))),
    ]
    for exc, call in bad:
        with pytest.raises(exc):
            call()
    assert rec.calls == []
