"""Degree 1 and 2 heat applies (column-marching kernel) on meshes with full 32-cell columns, where
interior layers are staged with 16-byte copies, with and without Dirichlet faces, with vectors at
offsets that are not 16-byte aligned, against the oracle."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from tests.gpu_util import rel_err, to_gpu
from tests.test_gpu_heat import heat_pair

pytestmark = pytest.mark.gpu

MESHES = [(2, (64, 8, 16)), (2, (33, 5, 9)), (1, (64, 8, 33)), (1, (96, 4, 16))]


@pytest.mark.parametrize("degree,m", MESHES)
@pytest.mark.parametrize("faces", [0, 0b111111, 0b101010])
def test_vmult_full_columns(degree, m, faces):
    import torch

    o, g, om, cm = heat_pair(degree, m, faces=faces, length=(1.2, 0.8, 1.0))
    x = uniform_dofs(om, seed=9)
    ref = o.vmult(x)
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 2e-6)):
        xd = to_gpu(x, dt)
        yd = torch.full_like(xd, float("nan"))
        g.vmult(yd, xd)
        assert rel_err(yd.cpu().numpy(), ref) <= tol
    assert g.device_errors() == 0


@pytest.mark.parametrize("degree,m", [(2, (64, 8, 16)), (1, (64, 8, 33)), (4, (33, 3, 5))])
@pytest.mark.parametrize("offset", [1, 3])
def test_vmult_unaligned_vectors(degree, m, offset):
    """src and dst that start `offset` elements into their allocations (not 16-byte aligned)."""
    import torch

    o, g, om, cm = heat_pair(degree, m, faces=0)
    x = uniform_dofs(om, seed=10)
    ref = o.vmult(x)
    for dt, tol in ((torch.float64, 1e-12), (torch.float32, 2e-6)):
        xs = torch.zeros(om.ndofs + offset, dtype=dt, device="cuda")
        ys = torch.full((om.ndofs + offset,), float("nan"), dtype=dt, device="cuda")
        xs[offset:] = to_gpu(x, dt)
        g.vmult(ys[offset:], xs[offset:])
        assert rel_err(ys[offset:].cpu().numpy(), ref) <= tol
