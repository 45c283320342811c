"""Transient heat adjoint on the GPU (C ABI) against the oracle's adjoint and central differences."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import normal_cells, uniform_dofs, unit_directions
from oracle import adjoint as OA
from oracle.oracle import Operator as OOp
from tests.adjoint_case import small_case
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu


def gpu_problem(c, n_steps, checkpoint_every, rel_tol=1e-13):
    from meltpooldg_b200.adjoint import TransientHeatAdjoint
    from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh

    om = c["mesh"]
    gm = Mesh(om.degree, om.m, dirichlet_faces=c["faces"])
    op = HeatDiffuseOperator(gm, rho_cp=c["rho_cp"], dt=c["dt"], conductivity=1.0)
    return op, TransientHeatAdjoint(op, n_steps, checkpoint_every, cg_rel_tol=rel_tol)


@pytest.mark.parametrize("degree,m,faces", [(1, (6, 5, 7), 0b111111), (2, (5, 6, 4), 0b111111),
                                            (2, (9, 4, 3), 0), (1, (33, 5, 3), 0b010101)])
def test_cell_stiffness_form_matches_oracle(degree, m, faces):
    import torch

    from meltpooldg_b200.adjoint import cell_stiffness_form
    from meltpooldg_b200.operators import HeatDiffuseOperator

    om, gm, cm = meshes(degree, m, faces=faces, length=(1.0, 0.7, 1.3))
    lam, T = uniform_dofs(om, seed=11), uniform_dofs(om, seed=12)
    ref = OOp(om, "heat", cmask=cm).cell_stiffness_form(lam, T)
    g = HeatDiffuseOperator(gm)
    out = torch.full((om.ncells,), np.nan, dtype=torch.float64, device="cuda")
    cell_stiffness_form(g, to_gpu(lam), to_gpu(T), out)
    assert rel_err(out.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("degree,rho_cp", [(1, 1.0), (2, 1.0), (2, 2.5)])
def test_forward_states_match_oracle(degree, rho_cp):
    import torch

    c = small_case(degree=degree, m=(5, 4, 6), n_steps=4, rho_cp=rho_cp)
    ref = OA.forward(c["mesh"], c["cmask"], c["rho_cp"], c["dt"], c["z"], c["qhat"], c["amplitude"])
    op, adj = gpu_problem(c, 4, 2)
    T = torch.full((4, c["mesh"].ndofs), np.nan, dtype=torch.float64, device="cuda")
    adj.forward(to_gpu(c["z"]), to_gpu(c["qhat"]), c["amplitude"], T)
    assert rel_err(T.cpu().numpy(), ref) <= 1e-10


@pytest.mark.parametrize("degree,n_steps,every", [(2, 6, 5), (2, 5, 2), (1, 4, 1), (2, 3, 7)])
def test_gradient_matches_oracle_adjoint(degree, n_steps, every):
    import torch

    c = small_case(degree=degree, m=(6, 5, 4), n_steps=n_steps)
    args = (c["mesh"], c["cmask"], c["rho_cp"], c["dt"])
    target = OA.forward(*args, c["z_target"], c["qhat"], c["amplitude"])
    J, gz, gA = OA.gradient(*args, c["z"], c["qhat"], c["amplitude"], target)
    op, adj = gpu_problem(c, n_steps, every)
    grad = torch.full((c["mesh"].ncells,), np.nan, dtype=torch.float64, device="cuda")
    Jg, gAg, st = adj.objective_and_gradient(to_gpu(c["z"]), to_gpu(c["qhat"]), c["amplitude"], to_gpu(target),
                                             grad)
    assert abs(Jg - J) <= 1e-9 * J
    assert rel_err(grad.cpu().numpy(), gz) <= 1e-8
    assert abs(gAg - gA) <= 1e-8 * abs(gA)
    n_seg = -(-n_steps // min(every, n_steps))
    assert st.adjoint_solves == n_steps
    assert st.forward_solves == 2 * n_steps  # one sweep, then every segment recomputed once
    assert n_seg >= 1 and op.device_errors() == 0


def test_gradient_matches_central_differences():
    import torch

    c = small_case(degree=2, m=(6, 6, 6), n_steps=6)
    op, adj = gpu_problem(c, 6, 5)
    zt, q = to_gpu(c["z_target"]), to_gpu(c["qhat"])
    target = torch.empty((6, c["mesh"].ndofs), dtype=torch.float64, device="cuda")
    adj.forward(zt, q, c["amplitude"], target)
    z = to_gpu(c["z"])
    grad = torch.empty(c["mesh"].ncells, dtype=torch.float64, device="cuda")
    J, gA, _ = adj.objective_and_gradient(z, q, c["amplitude"], target, grad)
    g = grad.cpu().numpy()
    h = 1e-6
    for d in unit_directions(c["mesh"].ncells, 5, seed=7):
        dd = to_gpu(d)
        jp, _, _ = adj.objective_and_gradient(z + h * dd, q, c["amplitude"], target)
        jm, _, _ = adj.objective_and_gradient(z - h * dd, q, c["amplitude"], target)
        fd = (jp - jm) / (2 * h)
        assert abs(fd - g @ d) <= 1e-6 * max(abs(fd), 1e-3 * np.linalg.norm(g))
    A = c["amplitude"]
    jp, _, _ = adj.objective_and_gradient(z, q, A * (1 + 1e-6), target)
    jm, _, _ = adj.objective_and_gradient(z, q, A * (1 - 1e-6), target)
    assert abs((jp - jm) / (2e-6 * A) - gA) <= 1e-6 * abs(gA)


def test_adjoint_argument_errors():
    import torch

    from meltpooldg_b200._lib import MpdgError
    from meltpooldg_b200.adjoint import TransientHeatAdjoint
    from meltpooldg_b200.operators import AdvectionDiffusionOperator, HeatDiffuseOperator, Mesh

    m = Mesh(3, (3, 3, 3))
    z = torch.zeros(27, dtype=torch.float64, device="cuda")
    q = torch.zeros((2, m.ndofs), dtype=torch.float64, device="cuda")
    with pytest.raises(MpdgError):
        TransientHeatAdjoint(HeatDiffuseOperator(m), 2).forward(z, q, 1.0, q.clone())
    with pytest.raises(MpdgError):
        m2 = Mesh(2, (3, 3, 3))
        a = AdvectionDiffusionOperator(m2, dt=1.0)
        q2 = torch.zeros((2, m2.ndofs), dtype=torch.float64, device="cuda")
        TransientHeatAdjoint(a, 2).objective_and_gradient(z, q2, 1.0, q2, None)
