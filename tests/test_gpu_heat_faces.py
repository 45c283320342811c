"""Boundary-face terms of the heat operator (convection, radiation, Neumann flux) on the GPU against
the oracle: the cell oracle plus oracle/faces.py, through the C ABI.  Covers every apply kernel
(column march k <= 2, pencil k = 3, 4, brick kernel with a per-DoF Dirichlet mask), FP64 and FP32,
the inverse diagonal, create_rhs, CG and the mixed-precision solve, and the argument checks."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import normal_cells, uniform_dofs
from oracle.faces import HeatBC, face_diagonal, face_rhs, face_tangent
from oracle.oracle import Operator as OOp
from tests.gpu_util import meshes, rel_err, to_gpu

pytestmark = pytest.mark.gpu

RAD = dict(emissivity=0.7, radiation_temperature_infinity=350.0)
CONV = dict(convection_coefficient=3.0, convection_temperature_infinity=300.0)
# (degree, cells, Dirichlet faces, per-DoF mask, boundary-face terms)
CASES = [
    (1, (9, 7, 5), 0b000001, False, dict(convection_faces=0b000010, radiation_faces=0b111100, **CONV, **RAD)),
    (2, (16, 16, 16), 0b010000, False, dict(convection_faces=0b100000, radiation_faces=0b001111, **CONV, **RAD)),
    (2, (9, 8, 5), 0, False, dict(radiation_faces=0b111111, **RAD)),
    (2, (6, 5, 7), 0b000001, True, dict(convection_faces=0b111110, **CONV)),
    (3, (5, 4, 6), 0b000011, False, dict(convection_faces=0b111100, **CONV)),
    (4, (5, 6, 4), 0b110000, False, dict(radiation_faces=0b001111, **RAD)),
    (4, (8, 8, 8), 0, False, dict(convection_faces=0b111111, **CONV)),
    (2, (7, 6, 5), 0b000001, False, dict(convection_faces=0b000010, neumann_faces=0b111100,
                                         neumann_flux=[0, 0, 2.0, -1.5, 0.5, 3.0], **CONV)),
    (3, (4, 5, 3), 0, False, dict(radiation_faces=0b000011, neumann_faces=0b110000,
                                  neumann_flux=[0, 0, 0, 0, -4.0, 1.0], **RAD)),
]


def setup(degree, m, faces, use_mask, bcargs, rho_cp=1.3, dt=1e-2, k=0.8):
    from meltpooldg_b200.operators import HeatDiffuseOperator

    length = (1.0, 0.8, 1.2)
    if use_mask:
        from oracle.oracle import Mesh as OMesh

        mask = OMesh(degree, m, length=length).face_mask(faces)
        om, gm, cm = meshes(degree, m, faces=0, mask=mask, length=length)
    else:
        om, gm, cm = meshes(degree, m, faces=faces, length=length)
    kc = np.exp(normal_cells(om, seed=2, sigma=0.5))
    o = OOp(om, "heat", cmask=cm, rho_cp=rho_cp, dt=dt, k=k, k_cell=kc)
    g = HeatDiffuseOperator(gm, rho_cp=rho_cp, dt=dt, conductivity=k, conductivity_cells=kc)
    bc = HeatBC(**bcargs)
    g.set_boundary_conditions(**bcargs)
    T = 300.0 + 300.0 * (uniform_dofs(om, seed=5) + 1.0)
    Td = to_gpu(T)
    g.set_temperature(Td)
    return o, g, om, cm, bc, T, Td


@pytest.mark.parametrize("degree,m,faces,use_mask,bcargs", CASES)
def test_vmult_with_faces_matches_oracle(degree, m, faces, use_mask, bcargs):
    import torch

    o, g, om, cm, bc, T, Td = setup(degree, m, faces, use_mask, bcargs)
    x = uniform_dofs(om, seed=1)
    ref = o.vmult(x) + face_tangent(om, cm, bc, T, x)
    xd = to_gpu(x)
    yd = torch.full_like(xd, np.nan)
    g.vmult(yd, xd)
    torch.cuda.synchronize()
    assert rel_err(yd.cpu().numpy(), ref) <= 1e-12
    x32 = to_gpu(x, torch.float32)
    y32 = torch.empty_like(x32)
    g.vmult(y32, x32)
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6
    assert g.device_errors() == 0


@pytest.mark.parametrize("degree,m,faces,use_mask,bcargs", CASES)
def test_inverse_diagonal_with_faces(degree, m, faces, use_mask, bcargs):
    import torch

    o, g, om, cm, bc, T, Td = setup(degree, m, faces, use_mask, bcargs)
    d = o.diagonal() + face_diagonal(om, cm, bc, T)
    ref = np.where(np.abs(d) > 1e-10, 1.0 / d, 1.0)
    dd = torch.empty(om.ndofs, dtype=torch.float64, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(dd)
    assert rel_err(dd.cpu().numpy(), ref) <= 1e-12
    d32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.compute_inverse_diagonal_from_matrixfree(d32)
    assert rel_err(d32.cpu().numpy(), ref) <= 1e-6


@pytest.mark.parametrize("degree,m,faces,use_mask,bcargs", CASES)
def test_create_rhs_with_faces(degree, m, faces, use_mask, bcargs):
    o, g, om, cm, bc, T, Td = setup(degree, m, faces, use_mask, bcargs)
    T_old = T - 20.0 * (uniform_dofs(om, seed=6) + 1.0)
    q = 1e3 * uniform_dofs(om, seed=7)
    dst0 = uniform_dofs(om, seed=8)
    ref = dst0.copy()
    o.create_rhs(ref, T, T_old, q)
    ref += face_rhs(om, cm, bc, T)
    dst = to_gpu(dst0)
    g.create_rhs(dst, Td, to_gpu(T_old), to_gpu(q))
    assert rel_err(dst.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("degree,m,faces,use_mask,bcargs", [CASES[1], CASES[3], CASES[5]])
def test_solves_with_faces_reach_the_oracle_residual(degree, m, faces, use_mask, bcargs):
    import torch

    from meltpooldg_b200.operators import LinearSolver, LinearSolverData

    o, g, om, cm, bc, T, Td = setup(degree, m, faces, use_mask, bcargs)
    b = uniform_dofs(om, seed=9)
    if cm is not None:
        b[cm != 0] = 0.0
    bd = to_gpu(b)

    def oracle_residual(x):
        return np.linalg.norm(b - o.vmult(x) - face_tangent(om, cm, bc, T, x)) / np.linalg.norm(b)

    x = torch.zeros_like(bd)
    LinearSolver.solve(g, x, bd, LinearSolverData("CG", "Diagonal", rel_tolerance=1e-10))
    assert oracle_residual(x.cpu().numpy()) <= 2e-10
    x = torch.zeros_like(bd)
    LinearSolver.solve_mixed(g, x, bd, outer_rel_tol=1e-9, inner_rel_tol=1e-3)
    assert oracle_residual(x.cpu().numpy()) <= 2e-9
    assert g.device_errors() == 0


def test_face_argument_checks():
    import ctypes as C

    import torch

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200._lib import MPDG_ERR_ARG, MpdgError
    from meltpooldg_b200.operators import AdvectionDiffusionOperator, HeatDiffuseOperator, Mesh

    g = HeatDiffuseOperator(Mesh(2, (4, 4, 4), dirichlet_faces=0b000001), dt=1e-2)
    for kw in (dict(convection_faces=0b000001),                          # a Dirichlet face
               dict(convection_faces=0b000010, neumann_faces=0b000010),  # Neumann and convection
               dict(radiation_faces=64)):                                 # not a face
        with pytest.raises(MpdgError) as e:
            g.set_boundary_conditions(**kw)
        assert e.value.code == MPDG_ERR_ARG
    g.set_boundary_conditions(radiation_faces=0b000010, emissivity=0.5)
    x = torch.zeros(g.n_dofs, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    with pytest.raises(MpdgError) as e:
        g.vmult(y, x)  # radiation without a linearisation temperature
    assert e.value.code == MPDG_ERR_ARG
    T = x + 400.0
    g.set_temperature(T)
    g.vmult(y, x)
    # the advection-diffusion operator has no heat faces
    a = AdvectionDiffusionOperator(Mesh(1, (4, 4, 4)), dt=1e-2)
    bc = L.HeatBC()
    bc.convection_faces = 1
    assert L.lib().mpdg_op_set_heat_bc(a._h, C.byref(bc)) == MPDG_ERR_ARG


def test_host_buffer_vmult_with_faces():
    """mpdg_op_vmult_host on an operator with face terms (large enough for the slab pipeline, which
    the face terms switch off) equals the device vmult."""
    import torch

    o, g, om, cm, bc, T, Td = setup(2, (80, 80, 82), 0b000001, False,
                                    dict(convection_faces=0b000010, radiation_faces=0b111100, **CONV, **RAD))
    x = uniform_dofs(om, seed=4)
    xd = to_gpu(x)
    yd = torch.empty_like(xd)
    g.vmult(yd, xd)
    yh = np.empty_like(x)
    g.vmult_host(yh, np.ascontiguousarray(x))
    # the same kernels; atomics on shared points may add in another order
    assert rel_err(yh, yd.cpu().numpy()) <= 1e-14
