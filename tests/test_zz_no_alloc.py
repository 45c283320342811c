"""Allocation-free heat vmult (mpdg_heat_vmult_noalloc) against the allocating mpdg_op_vmult and the
oracle.

Callers that reserve all of their device memory themselves, or that cannot afford a device-wide
synchronisation from cudaMalloc / cudaFree inside a time loop, use this entry point.  The file is
collected last on purpose, so that it runs after every other test on the same device;
test_noalloc_in_a_fresh_process runs the entry point's first call on a device (its set-up) in a new
Python process.
"""
import ctypes as C
import os
import subprocess
import sys

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


def error_word(stream=None):
    from meltpooldg_b200 import _lib as L

    w = C.c_int(-1)
    assert L.lib().mpdg_heat_vmult_noalloc_errors(stream, C.byref(w)) == L.MPDG_OK, L.lib().mpdg_last_error()
    return w.value


@pytest.mark.gpu
@pytest.mark.parametrize("degree,cells,faces,kfield", CASES)
def test_noalloc_vmult_matches_vmult_twice(degree, cells, faces, kfield):
    import torch

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh
    from oracle.oracle import Mesh as OMesh
    from oracle.oracle import Operator as OOp

    mesh = Mesh(degree, cells, length=(1.0, 0.8, 1.2), dirichlet_faces=faces)
    kc = np.exp(normal_cells(mesh, seed=2, sigma=0.5)) if kfield else None
    op = HeatDiffuseOperator(mesh, rho_cp=1.3, dt=1e-2, conductivity=0.7, conductivity_cells=kc)
    src = torch.tensor(uniform_dofs(mesh, seed=1), dtype=torch.float64, device="cuda")
    ref = torch.empty_like(src)
    op.vmult(ref, src)
    torch.cuda.synchronize()
    ref = ref.cpu().numpy()
    om = OMesh(degree, cells, length=(1.0, 0.8, 1.2))
    orc = OOp(om, "heat", cmask=om.face_mask(faces) if faces else None, rho_cp=1.3, dt=1e-2, k=0.7, k_cell=kc)
    y_orc = orc.vmult(src.cpu().numpy())
    m, p = descs(degree, cells, faces)
    k_dev = None if kc is None else torch.tensor(kc, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    scale = np.max(np.abs(ref))
    for _ in range(2):  # the second call finds the first call's contents in the shared scratch
        dst = torch.full_like(src, np.nan)
        rc = call_noalloc(m, p, k_dev, dst, src, stream)
        assert rc == L.MPDG_OK, L.lib().mpdg_last_error()
        assert error_word(stream) == 0
        torch.cuda.synchronize()
        y = dst.cpu().numpy()
        assert np.max(np.abs(y - ref)) <= 1e-13 * scale
        assert np.max(np.abs(y - y_orc)) <= 1e-12 * np.max(np.abs(y_orc))


FRESH = r"""
import ctypes as C, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from test_zz_no_alloc import call_noalloc, descs, error_word
from meltpooldg_b200 import _lib as L
from meltpooldg_b200.inputs import uniform_dofs
from oracle.oracle import Mesh as OMesh, Operator as OOp
om = OMesh(2, (16, 16, 16), length=(1.0, 0.8, 1.2))
x = uniform_dofs(om, seed=1)
src = torch.tensor(x, device="cuda")
stream = torch.cuda.current_stream().cuda_stream
y_orc = OOp(om, "heat", cmask=om.face_mask(63), rho_cp=1.3, dt=1e-2, k=0.7).vmult(x)
m, p = descs(2, (16, 16, 16), 63)
for _ in range(2):
    dst = torch.full_like(src, float("nan"))
    assert call_noalloc(m, p, None, dst, src, stream) == L.MPDG_OK, L.lib().mpdg_last_error()
    assert error_word(stream) == 0
    err = np.max(np.abs(dst.cpu().numpy() - y_orc)) / np.max(np.abs(y_orc))
    assert err <= 1e-12, err
print("fresh ok")
"""


@pytest.mark.gpu
def test_noalloc_in_a_fresh_process():
    """The first call of the process on the device (the set-up) and a second call, against the oracle."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", FRESH, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "fresh ok" in r.stdout, r.stdout + r.stderr


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
