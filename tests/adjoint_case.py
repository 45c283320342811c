"""Small instance of the transient heat adjoint workload (moving Gaussian source, seeded fields)."""
import numpy as np

from meltpooldg_b200.inputs import moving_gaussian, normal_cells


def small_case(degree=2, m=(4, 4, 4), n_steps=6, dt=1e-3, amplitude=100.0, faces=0b111111, rho_cp=1.0):
    from oracle.oracle import Mesh as OMesh

    om = OMesh(degree, m)
    cm = om.face_mask(faces) if faces else None
    z = normal_cells(om, seed=5, sigma=0.3)
    zt = normal_cells(om, seed=6, sigma=0.3)
    qhat = moving_gaussian(om, n_steps, dt)
    return dict(mesh=om, cmask=cm, rho_cp=rho_cp, dt=dt, z=z, z_target=zt, qhat=qhat, amplitude=amplitude,
                faces=faces)
