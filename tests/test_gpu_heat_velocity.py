"""Convection velocity of the heat operator (heat_diffuse_operator.cpp:448-453, 499-500, 1038-1041)
on the GPU against the oracle: the heat operator (oracle C++ restatement) plus the velocity term of
oracle/advection_field.py, for vmult (FP64 and FP32), create_rhs, the inverse diagonal and a GMRES
solve, with a non-affine DoF-vector velocity."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from oracle import advection_field as AF
from oracle.oracle import Operator as OOp
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu

RHO_CP, DT, K = 1.3, 1e-2, 0.7


def setup(degree, m, faces):
    from meltpooldg_b200.operators import HeatDiffuseOperator

    om, gm, cm = meshes(degree, m, faces=faces, length=(1.0, 0.8, 1.2))
    X, Y, Z = om.coords()
    field = [np.sin(2.0 * Y) + 0.3 * Z, np.cos(1.5 * X) - Z * Z, 0.4 * X * Y - 0.2]
    o = OOp(om, "heat", cmask=cm, rho_cp=RHO_CP, dt=DT, k=K)
    g = HeatDiffuseOperator(gm, rho_cp=RHO_CP, dt=DT, conductivity=K)
    fd = [to_gpu(c) for c in field]
    g.set_velocity_field(*fd)
    return o, g, om, cm, field, fd


def velocity_term(om, cm, field, u, plain):
    """int rho c_p (v . grad u) phi on the free rows (constrained entries of u read as 0 unless plain)."""
    return AF._form(om, cm, field, 0.0, RHO_CP, 0.0, u, plain=plain)


@pytest.mark.parametrize("degree,m,faces", [(1, (9, 7, 5), 0b111111), (2, (9, 8, 5), 0b010011), (2, (12, 10, 9), 0),
                                            (3, (5, 4, 4), 0b000011)])
def test_heat_velocity_vmult_rhs_diagonal(degree, m, faces):
    import torch

    o, g, om, cm, field, fd = setup(degree, m, faces)
    u = uniform_dofs(om, seed=21)
    ref = o.vmult(u) + velocity_term(om, cm, field, u, plain=False)
    y = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    g.vmult(y, to_gpu(u))
    assert rel_err(y.cpu().numpy(), ref) <= 1e-12
    y32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.vmult(y32, to_gpu(u, torch.float32))
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6
    # create_rhs: dst += M (rho c_p / dt (T_old - T) + q) - K T - int rho c_p (v . grad T) phi
    T, To, q = (uniform_dofs(om, seed=s) for s in (22, 23, 24))
    ref_rhs = uniform_dofs(om, seed=25)
    dst = to_gpu(ref_rhs)
    o.create_rhs(ref_rhs, T, To, q)
    ref_rhs -= velocity_term(om, cm, field, T, plain=True)
    g.create_rhs(dst, to_gpu(T), to_gpu(To), to_gpu(q))
    assert rel_err(dst.cpu().numpy(), ref_rhs) <= 1e-12
    # inverse diagonal of the whole tangent, heat rule (|d| > 1e-10 ? 1/d : 1, constrained rows 1)
    dfull = RHO_CP * AF.diagonal(om, cm, field, DT, 1.0, K / RHO_CP)
    if cm is not None:
        dfull[np.asarray(cm) != 0] = 1.0
    inv = np.where(np.abs(dfull) > 1e-10, 1.0 / np.where(dfull != 0, dfull, 1.0), 1.0)
    d = torch.empty_like(y)
    g.compute_inverse_diagonal_from_matrixfree(d)
    assert rel_err(d.cpu().numpy(), inv) <= 1e-12
    assert g.device_errors() == 0


def test_heat_velocity_gmres_solve():
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    o, g, om, cm, field, fd = setup(2, (10, 9, 8), 0b111111)
    b = uniform_dofs(om, seed=26, cmask=cm)
    # the GPU GMRES must reach its tolerance measured with the oracle's operator
    xg = torch.zeros(om.ndofs, dtype=torch.float64, device="cuda")
    st = LinearSolver.solve(g, xg, to_gpu(b), LinearSolverData("GMRES", "Diagonal", rel_tolerance=1e-10))
    x = xg.cpu().numpy()
    r = b - (o.vmult(x) + velocity_term(om, cm, field, x, plain=False))
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b)
    assert st.iterations > 0


def test_heat_velocity_restrictions():
    import torch

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200.operators import HeatDiffuseOperator

    o, g, om, cm, field, fd = setup(2, (4, 4, 4), 0)
    with pytest.raises(L.MpdgError) as exc:
        g.set_solidification((7.4, 0.8, 30.0), (7.9, 0.6, 20.0), 1700.0, 1600.0)
    assert exc.value.code == L.MPDG_ERR_UNSUPPORTED
    om4, gm4, _ = meshes(4, (2, 2, 2))
    g4 = HeatDiffuseOperator(gm4, rho_cp=RHO_CP, dt=DT, conductivity=K)
    v = torch.zeros(om4.ndofs, dtype=torch.float64, device="cuda")
    with pytest.raises(L.MpdgError) as exc:
        g4.set_velocity_field(v, v, v)
    assert exc.value.code == L.MPDG_ERR_UNSUPPORTED
