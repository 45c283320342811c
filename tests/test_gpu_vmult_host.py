"""Host-buffer apply (mpdg_op_vmult_host) on meshes large enough for the z-slab pipeline (copies in
both directions overlapped with the slab applies), against the oracle."""
import numpy as np
import pytest

from meltpooldg_b200.inputs import uniform_dofs
from tests.gpu_util import rel_err
from tests.test_gpu_heat import heat_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("degree,m,faces", [(2, (64, 64, 128), 0b111111), (4, (32, 32, 64), 0b110011),
                                            (1, (128, 128, 256), 0), (3, (48, 47, 73), 0b111111)])
def test_vmult_host_slab_pipeline(degree, m, faces):
    import torch

    o, g, om, cm = heat_pair(degree, m, faces=faces, length=(1.0, 1.1, 0.9))
    assert om.ndofs >= 1 << 22 and m[2] >= 16  # the pipelined path
    x = uniform_dofs(om, seed=31)
    ref = o.vmult(x)
    src = torch.tensor(x).pin_memory()
    for _ in range(2):
        dst = torch.full_like(src, np.nan).pin_memory()
        g.vmult_host(dst.numpy(), src.numpy())
        assert rel_err(dst.numpy(), ref) <= 1e-12
    assert g.device_errors() == 0
