"""The reference's golden application logs reproduced through the GPU operators."""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Operator as OOp
from tests.cases import heat_unidirectional, vortex, vortex_inflow, vortex_supg
from tests.gpu_util import to_gpu

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_logs.json")))


def test_heat_unidirectional_log_gpu():
    import torch

    from meltpooldg_b200.operators import HeatDiffuseOperator, LinearSolver, LinearSolverData, Mesh

    om, T0 = heat_unidirectional()
    g = HeatDiffuseOperator(Mesh(1, om.m, om.origin, om.length), rho_cp=1.0, dt=1e-4, conductivity=1.0)
    norm = OOp(om, "heat", dt=1e-4)  # L2 norm of the GPU result (post-processing only)
    T = to_gpu(T0)
    zero = torch.zeros_like(T)
    got = []
    data = LinearSolverData("GMRES", "Diagonal", rel_tolerance=1e-12)
    for _ in range(5):
        T_old = T.clone()
        for _newton in range(10):
            rhs = torch.zeros_like(T)
            g.create_rhs(rhs, T, T_old, zero)
            d = torch.zeros_like(T)
            LinearSolver.solve(g, d, rhs, data)
            if torch.linalg.norm(rhs).item() < 5e-9 and torch.linalg.norm(d).item() < 1e-10:
                break
            T += d
        got.append("%.5e" % norm.l2_norm(T.cpu().numpy()))
    assert got == GOLD["heat_unidirectional_2d_q1"]["values"]


@pytest.mark.parametrize("dim,key", [(3, "advdiff_vortex_mf_3d_q1"), (2, "advdiff_vortex_mf_2d_q1")])
def test_vortex_log_gpu(dim, key):
    import torch

    from meltpooldg_b200.operators import AdvectionDiffusionOperator, LinearSolver, LinearSolverData, Mesh

    om, phi0, mask, vel = vortex(dim)
    gm = Mesh(1, om.m, om.origin, om.length, dirichlet_mask=mask)
    g = AdvectionDiffusionOperator(gm, dt=0.01, theta=0.5, diffusivity=0.0, velocity=vel)
    norm = OOp(om, "heat")
    ref = np.array([float(v) for v in GOLD[key]["values"]])
    phi = to_gpu(phi0)
    mask_t = torch.tensor(mask, device="cuda").bool()
    dirichlet_minus_one = torch.full_like(phi, -1.0)
    data = LinearSolverData("GMRES", "Diagonal", rel_tolerance=1e-12)
    out = []
    for _ in range(5):
        old = phi.clone()
        # create_rhs_and_apply_dirichlet_matrixfree (utilities_matrixfree.hpp:39-100), Dirichlet -1
        rhs = torch.empty_like(phi)
        g.create_rhs_and_apply_dirichlet(rhs, old, dirichlet_minus_one)
        x = old.clone()
        LinearSolver.solve(g, x, rhs, data)
        x[mask_t] = -1.0
        phi = x
        out.append(norm.l2_norm(phi.cpu().numpy()))
    assert np.max(np.abs(np.array(out) - ref) / ref) < 5e-8


@pytest.mark.parametrize("dim,key", [(3, "advdiff_vortex_mf_inflow_outflow_3d_q1"),
                                     (2, "advdiff_vortex_mf_inflow_outflow_2d_q1")])
def test_vortex_inflow_outflow_log_gpu(dim, key):
    """AdvectionDiffusionOperation::solve with the inflow/outflow condition
    (source/level_set/advection_diffusion_operation.cpp:243-296) through the GPU operator: lifting with
    the inflow values, GMRES with identity inflow rows, the values distributed after the solve.
    Checked against the reference's log (to its float-rounded norm, see test_oracle_golden.py) and
    step by step against the oracle's fields."""
    import torch

    from meltpooldg_b200.operators import AdvectionDiffusionOperator, LinearSolver, LinearSolverData, Mesh
    from oracle.oracle import inflow_dofs
    from oracle.oracle import solve as osolve

    om, phi0, vel, faces = vortex_inflow(dim)
    g = AdvectionDiffusionOperator(Mesh(1, om.m, om.origin, om.length), dt=0.01, theta=0.5, diffusivity=0.0,
                                   velocity=vel)
    values = torch.full((om.ndofs,), -1.0, dtype=torch.float64, device="cuda")
    inflow = inflow_dofs(om, vel, faces)
    assert g.set_inflow_outflow_bc(faces, values) == int(inflow.sum())
    orc = OOp(om, "advdiff", dt=0.01, theta=0.5, eps=0.0, vel=vel, imask=inflow)
    # vmult and the inverse diagonal with identity inflow rows
    x = np.sin(np.arange(om.ndofs) * 0.37)
    y = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    g.vmult(y, to_gpu(x))
    assert np.max(np.abs(y.cpu().numpy() - orc.vmult(x))) <= 1e-12 * np.max(np.abs(orc.vmult(x)))
    d = torch.empty_like(y)
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert np.max(np.abs(d.cpu().numpy() - orc.inverse_diagonal())) <= 1e-12 * np.max(np.abs(orc.inverse_diagonal()))
    ref = np.array([float(v) for v in GOLD[key]["values"]])
    phi = to_gpu(phi0)
    phi_o = phi0.copy()
    nobc = orc.with_(imask=None)
    zero = torch.zeros_like(phi)
    data = LinearSolverData("GMRES", "Diagonal", rel_tolerance=1e-12)
    out = []
    for _ in range(5):
        old = phi.clone()
        rhs = torch.empty_like(phi)
        g.create_rhs_and_apply_dirichlet(rhs, old, zero)
        x = old.clone()
        LinearSolver.solve(g, x, rhs, data)
        g.distribute_inflow(x)
        phi = x
        out.append(orc.l2_norm(phi.cpu().numpy()))
        # the oracle's step
        bc = np.where(inflow == 1, -1.0, 0.0)
        r_o = -nobc.vmult(bc)
        nobc.create_rhs(r_o, phi_o)
        r_o[inflow == 1] = 0.0
        x_o = phi_o.copy()
        osolve(orc, x_o, r_o, "gmres", inv_diag=orc.inverse_diagonal(), rel_tol=1e-12)
        x_o[inflow == 1] = -1.0
        phi_o = x_o
        assert np.max(np.abs(phi.cpu().numpy() - phi_o)) <= 1e-10
    assert np.max(np.abs(np.array(out) - ref) / ref) < 5e-8
    assert g.device_errors() == 0


def test_vortex_supg_log_gpu():
    """advection_diffusion_vortex_mf_supg.mpirun=4.output through the GPU operator with SUPG
    (coefficient -1): Dirichlet lifting, GMRES(30) with the Jacobi preconditioner, 5 steps."""
    import torch

    from meltpooldg_b200.operators import AdvectionDiffusionOperator, LinearSolver, LinearSolverData, Mesh

    om, phi0, mask, vel, h = vortex_supg()
    gm = Mesh(1, om.m, om.origin, om.length, dirichlet_mask=mask)
    g = AdvectionDiffusionOperator(gm, dt=0.01, theta=0.5, diffusivity=0.0, velocity=vel)
    g.set_convection_stabilization("SUPG", -1.0)
    norm = OOp(om, "heat")
    ref = np.array([float(v) for v in GOLD["advdiff_vortex_supg_2d_q1"]["values"]])
    phi = to_gpu(phi0)
    mask_t = torch.tensor(mask, device="cuda").bool()
    minus_one = torch.full_like(phi, -1.0)
    data = LinearSolverData("GMRES", "Diagonal", rel_tolerance=1e-12)
    out = []
    for _ in range(5):
        old = phi.clone()
        rhs = torch.empty_like(phi)
        g.create_rhs_and_apply_dirichlet(rhs, old, minus_one)
        x = old.clone()
        LinearSolver.solve(g, x, rhs, data)
        x[mask_t] = -1.0
        phi = x
        out.append(norm.l2_norm(phi.cpu().numpy()) / np.sqrt(h))
    assert np.max(np.abs(np.array(out) - ref) / ref) < 5e-8
    assert g.device_errors() == 0
