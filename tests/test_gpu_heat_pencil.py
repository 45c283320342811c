"""Degree 3 and 4 heat applies (pencil-marching kernel) on bricks of every fill: full 32-cell rows
in x (the last x point of the row is processed cooperatively), partial rows, partial y rows and z
layers, all output modes and Dirichlet face patterns, against the oracle."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from tests.gpu_util import rel_err, to_gpu
from tests.test_gpu_heat import heat_pair

pytestmark = pytest.mark.gpu

MESHES = [(4, (32, 3, 5)), (4, (65, 2, 9)), (3, (64, 5, 4)), (3, (33, 1, 1)), (4, (1, 7, 3)), (4, (40, 4, 8))]


@pytest.mark.parametrize("degree,m", MESHES)
@pytest.mark.parametrize("faces", [0b111111, 0, 0b010110])
def test_vmult_matches_oracle(degree, m, faces):
    import torch

    o, g, om, cm = heat_pair(degree, m, faces=faces, length=(1.3, 0.9, 1.1))
    x = uniform_dofs(om, seed=7)
    ref = o.vmult(x)
    xd = to_gpu(x)
    for _ in range(2):
        yd = torch.full_like(xd, np.nan)
        g.vmult(yd, xd)
        assert rel_err(yd.cpu().numpy(), ref) <= 1e-12
    if cm is not None:
        assert np.all(yd.cpu().numpy()[cm == 1] == 0.0)
    y32 = torch.empty(om.ndofs, dtype=torch.float32, device="cuda")
    g.vmult(y32, to_gpu(x, torch.float32))
    assert rel_err(y32.cpu().numpy(), ref) <= 2e-6
    assert g.device_errors() == 0


@pytest.mark.parametrize("degree,m", [(4, (33, 3, 5)), (3, (64, 2, 3))])
def test_modes_and_plain_reads(degree, m):
    o, g, om, cm = heat_pair(degree, m)
    x, b = uniform_dofs(om, seed=1), uniform_dofs(om, seed=2)
    Ax = o.vmult(x)
    xd, bd = to_gpu(x), to_gpu(b)
    acc = bd.clone()
    g.vmult_add(acc, xd, -0.5)
    assert rel_err(acc.cpu().numpy(), b - 0.5 * Ax) <= 1e-12
    r = bd.clone()
    g.residual(r, r, xd)
    assert rel_err(r.cpu().numpy(), b - Ax) <= 1e-12
    T, To, q = (uniform_dofs(om, seed=s) for s in (3, 4, 5))
    ref = uniform_dofs(om, seed=6)
    dst = to_gpu(ref)
    o.create_rhs(ref, T, To, q)
    g.create_rhs(dst, to_gpu(T), to_gpu(To), to_gpu(q))
    assert rel_err(dst.cpu().numpy(), ref) <= 1e-12
