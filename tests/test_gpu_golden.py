"""The reference's golden application logs reproduced through the GPU operators."""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Operator as OOp
from tests.cases import heat_unidirectional, vortex
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
