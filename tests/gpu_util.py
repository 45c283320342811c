"""Helpers shared by the GPU parity tests (oracle = checker only)."""
import numpy as np

from oracle.oracle import Mesh as OMesh
from oracle.oracle import Operator as OOp
from meltpooldg_b200.operators import Mesh


def meshes(degree, m, faces=0, mask=None, origin=(0, 0, 0), length=(1, 1, 1)):
    om = OMesh(degree, m, origin=origin, length=length)
    cm = om.face_mask(faces) if faces else None
    if mask is not None:
        cm = mask if cm is None else np.maximum(cm, mask)
    gm = Mesh(degree, m, origin=origin, length=length, dirichlet_faces=faces, dirichlet_mask=mask)
    return om, gm, cm


def to_gpu(x, dtype=None):
    import torch

    return torch.tensor(np.asarray(x), dtype=dtype or torch.float64, device="cuda")


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
