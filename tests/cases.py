"""The reference's golden application cases, restated on a structured 3-D lattice.

* heat_unidirectional: applications/mp-heat-transfer/cases/unidirectional_heat_transfer/
  unidirectional_heat_transfer.cpp:26-48 (LinearTemp 0 -> 0.1 on [0,0.1]), :160-175 (hyper
  rectangle [0,0.1]^2, 5 global refinements), tests/unidirectional_heat_transfer.json (Q1, dt 1e-4,
  5 steps, rho = c_p = k = 1, no boundary condition: adiabatic).  The 2-D problem is solved as a
  32 x 32 x 1 hexahedral mesh of depth 1: its z-independent solution is the 2-D one and the L2
  norm over depth 1 equals the 2-D norm.
* vortex: applications/mp-advec-diff/cases/advection_diffusion_vortex.hpp (tanh sphere at
  (0,0,0.5) / (0,0.5), r 0.25, eps = 0.5 min_cell_diameter / sqrt(dim); velocity
  (4 y, -4 x) with y = p[dim-1]; Dirichlet -1 on the inflow half-faces, :176-206),
  tests/advection_diffusion_vortex_mf[_3d].json (Q1, [-1,1]^dim, 3 / 5 refinements, dt 0.01,
  Crank-Nicolson, diffusivity 0, GMRES + Jacobi).
"""
import numpy as np

from oracle.oracle import Mesh


def heat_unidirectional():
    mesh = Mesh(degree=1, m=(32, 32, 1), origin=(0, 0, 0), length=(0.1, 0.1, 1.0))
    X, _, _ = mesh.coords()
    return mesh, X.copy()


def vortex(dim: int):
    if dim == 3:
        m, h = 8, 0.25
        mesh = Mesh(1, (m, m, m), origin=(-1, -1, -1), length=(2, 2, 2))
        X, Y, Z = mesh.coords()
        sd = 0.25 - np.sqrt(X ** 2 + Y ** 2 + (Z - 0.5) ** 2)
        eps = 0.5 * (h * np.sqrt(3)) / np.sqrt(3)
        vel = [0, 0, 0, 0, 0, 4, 0, 0, 0, -4, 0, 0]  # (4 z, 0, -4 x)
        a_dim, b_dim = 0, 2  # in-plane coordinates: x and z
    else:
        m, h = 32, 2.0 / 32
        mesh = Mesh(1, (m, m, 1), origin=(-1, -1, 0), length=(2, 2, 1))
        X, Y, Z = mesh.coords()
        sd = 0.25 - np.sqrt(X ** 2 + (Y - 0.5) ** 2)
        eps = 0.5 * (h * np.sqrt(2)) / np.sqrt(2)
        vel = [0, 0, 0, 0, 4, 0, -4, 0, 0, 0, 0, 0]  # (4 y, -4 x)
        a_dim, b_dim = 0, 1
    phi = np.tanh(sd / (2 * eps))
    nx, ny, nz = mesh.n
    mask = np.zeros((nz, ny, nx), np.uint8)

    def sl(d, lo_hi, a=None):
        idx = [slice(None)] * 3
        axis = 2 - d  # array axes are (z, y, x)
        idx[axis] = 0 if lo_hi == 0 else -1
        return idx

    # boundary faces of the a_dim / b_dim planes; face-centre rules of advection_diffusion_vortex.hpp
    for c in range(m):
        centre = -1 + (c + 0.5) * h
        rng = slice(c, c + 2)
        for (d, side, other, cond) in (
            (a_dim, 0, b_dim, centre >= 0),   # x = -1, y>=0
            (a_dim, 1, b_dim, centre <= 0),   # x = +1, y<=0
            (b_dim, 1, a_dim, centre >= 0),   # y = +1, x>=0
            (b_dim, 0, a_dim, centre <= 0),   # y = -1, x<=0
        ):
            if not cond:
                continue
            idx = sl(d, side)
            idx[2 - other] = rng
            mask[tuple(idx)] = 1
    mask = mask.ravel()
    phi[mask == 1] = -1.0
    return mesh, phi, mask, vel


def vortex_inflow(dim: int):
    """applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_inflow_outflow[_3d].json:
    the vortex case with the inflow/outflow condition (value -1) on every boundary face of the
    domain (advection_diffusion_vortex.hpp:159-166 attaches it to both boundary ids), no Dirichlet
    constraints, so the initial field keeps its interpolated boundary values.  Returns the mesh, the
    initial field, the velocity and the box faces that carry the condition (the z faces of the
    depth-1 extrusion are not boundaries of the 2-D problem)."""
    mesh, _, _, vel = vortex(dim)
    X, Y, Z = mesh.coords()
    if dim == 3:
        sd = 0.25 - np.sqrt(X ** 2 + Y ** 2 + (Z - 0.5) ** 2)
        eps = 0.5 * (0.25 * np.sqrt(3)) / np.sqrt(3)
        faces = 0b111111
    else:
        h = 2.0 / 32
        sd = 0.25 - np.sqrt(X ** 2 + (Y - 0.5) ** 2)
        eps = 0.5 * (h * np.sqrt(2)) / np.sqrt(2)
        faces = 0b001111
    return mesh, np.tanh(sd / (2 * eps)), vel, faces


def vortex_supg():
    """applications/mp-advec-diff/cases/tests/advection_diffusion_vortex_mf_supg.json: the 2-D vortex
    case (matrix-free by default) with SUPG, coefficient -1 (tau_c = h_c / max |v|).  The SUPG cell
    size is the cell diameter / sqrt(dim) (source/core/scratch_data.cpp:262-277), h for the 2-D
    squares; the extrusion here is one cube cell deep (depth h), whose diameter / sqrt(3) is the same
    h.  Every term then scales with the depth, so the solution is the 2-D one and the 2-D L2 norm is
    the 3-D norm divided by sqrt(h).  Returns the mesh, the initial field, the Dirichlet mask, the
    velocity and h."""
    m, h = 32, 2.0 / 32
    mesh0, phi0, mask0, vel = vortex(2)
    mesh = Mesh(1, (m, m, 1), origin=(-1, -1, 0), length=(2, 2, h))
    assert mesh.ndofs == mesh0.ndofs  # the same lattice, only the depth differs
    return mesh, phi0, mask0, vel, h
