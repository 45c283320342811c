"""Heat operator with temperature-dependent material (solidification tangent) on the GPU against
oracle/solidification.py, through the C ABI: vmult (FP64, FP32), create_rhs, the inverse diagonal,
the argument checks and a GMRES solve of the (nonsymmetric) tangent system."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from oracle.oracle import Operator as OOp
from oracle.solidification import SolidLiquid, diagonal, residual, tangent_apply
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu

LIQ, SOL, TL, TS = (7.4, 0.8, 30.0), (7.9, 0.6, 20.0), 1700.0, 1600.0
CASES = [(1, (9, 7, 5), 0b000001, False, False), (2, (9, 8, 5), 0b010011, False, False),
         (2, (16, 16, 16), 0, False, False), (2, (6, 5, 7), 0b000001, True, False),
         (1, (5, 6, 4), 0b100000, False, True), (2, (7, 4, 6), 0, False, True),
         (3, (5, 4, 3), 0b000101, False, False), (3, (4, 3, 5), 0b000001, True, True)]


def setup(degree, m, faces, use_mask, sharp, dt=1e-3):
    from meltpooldg_b200.operators import HeatDiffuseOperator

    length = (0.7, 0.9, 0.5)
    if use_mask:
        from oracle.oracle import Mesh as OMesh

        mask = OMesh(degree, m, length=length).face_mask(faces)
        om, gm, cm = meshes(degree, m, faces=0, mask=mask, length=length)
    else:
        om, gm, cm = meshes(degree, m, faces=faces, length=length)
    g = HeatDiffuseOperator(gm, rho_cp=1.0, dt=dt, conductivity=1.0)
    g.set_solidification(LIQ, SOL, TL, TS, sharp=sharp)
    mat = SolidLiquid(LIQ, SOL, TL, TS, sharp)
    T = 1650.0 + 90.0 * uniform_dofs(om, seed=5)
    Told = T - 4.0 * (uniform_dofs(om, seed=6) + 1.0)
    Td, Tod = to_gpu(T), to_gpu(Told)
    g.set_temperature(Td)
    g.set_old_temperature(Tod)
    return g, om, cm, mat, T, Told, (Td, Tod)


@pytest.mark.parametrize("degree,m,faces,use_mask,sharp", CASES)
def test_solid_vmult_matches_oracle(degree, m, faces, use_mask, sharp):
    import torch

    dt = 1e-3
    g, om, cm, mat, T, Told, keep = setup(degree, m, faces, use_mask, sharp, dt)
    x = uniform_dofs(om, seed=1)
    ref = tangent_apply(om, cm, mat, dt, T, Told, x)
    xd = to_gpu(x)
    yd = torch.full_like(xd, np.nan)
    g.vmult(yd, xd)
    assert rel_err(yd.cpu().numpy(), ref) <= 1e-12
    y32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.vmult(y32, to_gpu(x, torch.float32))
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-5  # material evaluated at FP32 temperatures
    assert g.device_errors() == 0


@pytest.mark.parametrize("degree,m,faces,use_mask,sharp", CASES)
def test_solid_create_rhs_and_diagonal(degree, m, faces, use_mask, sharp):
    import torch

    dt = 1e-3
    g, om, cm, mat, T, Told, (Td, Tod) = setup(degree, m, faces, use_mask, sharp, dt)
    q = 1e4 * uniform_dofs(om, seed=7)
    dst0 = uniform_dofs(om, seed=8)
    ref = dst0.copy()
    mass = OOp(om, "heat", cmask=cm, rho_cp=1.0, dt=1.0, k=1.0)  # create_rhs(0, 0, q) = int q phi
    mass.create_rhs(ref, np.zeros(om.ndofs), np.zeros(om.ndofs), q)
    ref += residual(om, cm, mat, dt, T, Told)
    dst = to_gpu(dst0)
    g.create_rhs(dst, Td, Tod, to_gpu(q))
    assert rel_err(dst.cpu().numpy(), ref) <= 1e-12
    d = diagonal(om, cm, mat, dt, T, Told)
    if cm is not None:
        d[cm != 0] = 1.0
    inv = np.where(np.abs(d) > 1e-10, 1.0 / d, 1.0)
    dd = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(dd)
    assert rel_err(dd.cpu().numpy(), inv) <= 1e-12


def test_solid_gmres_reaches_the_oracle_residual():
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    dt = 1e-3
    g, om, cm, mat, T, Told, keep = setup(2, (12, 10, 9), 0b010011, False, False, dt)
    b = uniform_dofs(om, seed=9)
    b[cm != 0] = 0.0
    x = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    LinearSolver.solve(g, x, to_gpu(b), LinearSolverData("GMRES", "Diagonal", max_iterations=2000, rel_tolerance=1e-10))
    xs = x.cpu().numpy()
    r = b - tangent_apply(om, cm, mat, dt, T, Told, xs)
    assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(b)


def test_solid_argument_checks():
    import torch

    from meltpooldg_b200._lib import MPDG_ERR_ARG, MPDG_ERR_UNSUPPORTED, MpdgError
    from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh

    g = HeatDiffuseOperator(Mesh(4, (2, 2, 2)), dt=1e-3)
    with pytest.raises(MpdgError) as e:
        g.set_solidification(LIQ, SOL, TL, TS)
    assert e.value.code == MPDG_ERR_UNSUPPORTED
    g = HeatDiffuseOperator(Mesh(2, (4, 4, 4)), dt=1e-3)
    with pytest.raises(MpdgError) as e:
        g.set_solidification(LIQ, SOL, 1500.0, 1600.0)  # liquidus below solidus
    assert e.value.code == MPDG_ERR_ARG
    g.set_solidification(LIQ, SOL, TL, TS)
    x = torch.zeros(g.n_dofs, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    with pytest.raises(MpdgError) as e:
        g.vmult(y, x)  # no temperatures yet
    assert e.value.code == MPDG_ERR_ARG
    T = x + 1650.0
    g.set_temperature(T)
    g.set_old_temperature(T)
    g.vmult(y, x)
    g.set_solidification(enabled=False)
    g.vmult(y, x)


@pytest.mark.parametrize("degree,capacity", [(1, "qlq"), (2, "qlq"), (2, "poly4_bell"), (2, "constant"), (3, "qlq")])
def test_solid_latent_heat_matches_oracle(degree, capacity):
    """Latent heat of fusion as the reference's apparent capacity (material.templates.hpp:561-614):
    vmult, the residual part of create_rhs and the inverse diagonal against the oracle, with the
    temperatures spread over the mushy zone and both pure phases."""
    import torch

    from meltpooldg_b200.operators import HeatDiffuseOperator

    dt, L = 1e-3, 2.7e5
    om, gm, cm = meshes(degree, (9, 8, 6), faces=0b000011, length=(0.7, 0.9, 0.5))
    g = HeatDiffuseOperator(gm, rho_cp=1.0, dt=dt, conductivity=1.0)
    g.set_solidification(LIQ, SOL, TL, TS, latent_heat=L, capacity_type=capacity)
    mat = SolidLiquid(LIQ, SOL, TL, TS, False, latent_heat=L, capacity_type=capacity)
    T = 1650.0 + 90.0 * uniform_dofs(om, seed=5)
    Told = T - 4.0 * (uniform_dofs(om, seed=6) + 1.0)
    Td, Tod = to_gpu(T), to_gpu(Told)
    g.set_temperature(Td)
    g.set_old_temperature(Tod)
    x = uniform_dofs(om, seed=1)
    ref = tangent_apply(om, cm, mat, dt, T, Told, x)
    yd = torch.full((om.ndofs,), np.nan, dtype=torch.float64, device="cuda")
    g.vmult(yd, to_gpu(x))
    assert rel_err(yd.cpu().numpy(), ref) <= 1e-12
    rhs = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    g.create_rhs(rhs, Td, Tod)
    assert rel_err(rhs.cpu().numpy(), residual(om, cm, mat, dt, T, Told)) <= 1e-12
    d = torch.empty_like(rhs)
    g.compute_inverse_diagonal_from_matrixfree(d)
    dref = diagonal(om, cm, mat, dt, T, Told)
    inv = np.where(np.abs(dref) > 1e-10, 1.0 / np.where(dref != 0, dref, 1.0), 1.0)
    if cm is not None:
        inv[cm == 1] = 1.0
    assert rel_err(d.cpu().numpy(), inv) <= 1e-12
    assert g.device_errors() == 0
