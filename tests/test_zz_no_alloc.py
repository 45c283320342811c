"""Allocation-free heat vmult (mpdg_heat_vmult_noalloc) against the allocating mpdg_op_vmult.

Callers that reserve all of their device memory themselves, or that cannot afford a device-wide
synchronisation from cudaMalloc / cudaFree inside a time loop, use this entry point.  The file is
collected last on purpose: the test must pass in a fresh process (the first call on a device does
the set-up) and after every other test has run on the same device.
"""
import ctypes as C

import numpy as np
import pytest

from meltpooldg_b200.inputs import normal_cells, uniform_dofs

CASES = [(1, (17, 9, 9), 0b111111, True), (2, (16, 16, 16), 0b111111, True), (2, (9, 8, 5), 0b101010, False),
         (3, (5, 4, 6), 0b111111, True), (4, (8, 8, 8), 0b111111, True), (4, (5, 6, 4), 0, False)]


def descs(degree, cells, faces, rho_cp=1.3, dt=1e-2, k=0.7, length=(1.0, 0.8, 1.2)):
    from meltpooldg_b200 import _lib as L

    m = L.MeshDesc()
    m.degree = degree
    for d in range(3):
        m.cells[d], m.length[d], m.origin[d] = cells[d], length[d], 0.0
    m.dirichlet_faces = faces
    m.dirichlet_mask = None
    p = L.OpParams()
    p.kind, p.rho_cp, p.dt, p.conductivity = L.MPDG_HEAT, rho_cp, dt, k
    p.conductivity_cells = None
    return m, p


def call_noalloc(m, p, k_dev, dst, src, stream=None):
    from meltpooldg_b200 import _lib as L

    return L.lib().mpdg_heat_vmult_noalloc(C.byref(m), C.byref(p), None if k_dev is None else k_dev.data_ptr(),
                                           None if dst is None else dst.data_ptr(),
                                           None if src is None else src.data_ptr(), stream)


@pytest.mark.gpu
@pytest.mark.parametrize("degree,cells,faces,kfield", CASES)
def test_noalloc_vmult_matches_vmult_twice(degree, cells, faces, kfield):
    import torch

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh

    mesh = Mesh(degree, cells, length=(1.0, 0.8, 1.2), dirichlet_faces=faces)
    kc = np.exp(normal_cells(mesh, seed=2, sigma=0.5)) if kfield else None
    op = HeatDiffuseOperator(mesh, rho_cp=1.3, dt=1e-2, conductivity=0.7, conductivity_cells=kc)
    src = torch.tensor(uniform_dofs(mesh, seed=1), dtype=torch.float64, device="cuda")
    ref = torch.empty_like(src)
    op.vmult(ref, src)
    torch.cuda.synchronize()
    ref = ref.cpu().numpy()
    m, p = descs(degree, cells, faces)
    k_dev = None if kc is None else torch.tensor(kc, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    scale = np.max(np.abs(ref))
    for _ in range(2):  # the second call finds the first call's contents in the shared scratch
        dst = torch.full_like(src, np.nan)
        rc = call_noalloc(m, p, k_dev, dst, src, stream)
        assert rc == L.MPDG_OK, L.lib().mpdg_last_error()
        torch.cuda.synchronize()
        assert np.max(np.abs(dst.cpu().numpy() - ref)) <= 1e-13 * scale


@pytest.mark.gpu
def test_noalloc_rejects_oversized_and_unsupported_inputs():
    """Every rejected call returns before any GPU work.  The oversized mesh is passed without
    vectors: the size check comes before the vector check, so no outcome of this call can launch."""
    import torch

    from meltpooldg_b200 import _lib as L

    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    y = torch.zeros(8, dtype=torch.float64, device="cuda")
    # 1280^3 cells of degree 1 (< 2^31 DoFs) need far more than MPDG_NOALLOC_MAX_BRICKS (65472) brick
    # flags for any brick of fewer than 32768 cells
    m, p = descs(1, (1280, 1280, 1280), 0b111111)
    assert call_noalloc(m, p, None, None, None) == L.MPDG_ERR_UNSUPPORTED
    assert b"brick flags" in L.lib().mpdg_last_error()
    m, p = descs(5, (4, 4, 4), 0b111111)
    assert call_noalloc(m, p, None, y, x) == L.MPDG_ERR_UNSUPPORTED
    m, p = descs(2, (4, 4, 4), 0)
    assert call_noalloc(m, p, None, x, x) == L.MPDG_ERR_ARG
    p.dt = 0.0
    assert call_noalloc(m, p, None, y, x) == L.MPDG_ERR_ZERO_DT
    m, p = descs(2, (4, 4, 4), 0)
    mask = np.zeros(9 ** 3, dtype=np.uint8)
    m.dirichlet_mask = mask.ctypes.data
    assert call_noalloc(m, p, None, y, x) == L.MPDG_ERR_UNSUPPORTED
    m, p = descs(2, (4, 4, 4), 0)
    p.kind = L.MPDG_ADVDIFF
    assert call_noalloc(m, p, None, y, x) == L.MPDG_ERR_ARG
