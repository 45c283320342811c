"""Seeded synthetic inputs keyed on lattice coordinates.

Every value is a pure function of ``(seed, index)`` where ``index`` is the lexicographic lattice
index of a DoF (``i + n_x (j + n_y l)``) or of a cell (``c_x + m_x (c_y + m_y c_z)``).  The same
inputs therefore arise for any DoF numbering (deal.II's global numbering is not lexicographic), on
the CPU and on the GPU.  The generator is splitmix64 (Steele, Lea, Flood, "Fast splittable
pseudorandom number generators", OOPSLA 2014).
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        z = x
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _unit(seed: int, index: np.ndarray) -> np.ndarray:
    """Uniform [0, 1) doubles from (seed, index)."""
    base = _splitmix64(np.array([seed], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        bits = _splitmix64(index.astype(np.uint64) + base)
    return (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform_dofs(mesh, seed: int, lo: float = -1.0, hi: float = 1.0, cmask=None) -> np.ndarray:
    """i.i.d. U[lo, hi] per DoF; constrained entries (cmask != 0) are set to 0."""
    idx = np.arange(mesh.ndofs, dtype=np.uint64)
    x = lo + (hi - lo) * _unit(seed, idx)
    if cmask is not None:
        x[np.asarray(cmask) != 0] = 0.0
    return x


def normal_cells(mesh, seed: int, sigma: float) -> np.ndarray:
    """i.i.d. N(0, sigma^2) per cell (Box-Muller on two streams of the same seed)."""
    c = np.arange(mesh.ncells, dtype=np.uint64)
    u1 = 1.0 - _unit(seed, np.uint64(2) * c)  # (0, 1]
    u2 = _unit(seed, np.uint64(2) * c + np.uint64(1))
    return sigma * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def unit_directions(n: int, count: int, seed: int) -> np.ndarray:
    """``count`` random unit vectors of length n (finite-difference directions)."""
    out = np.empty((count, n))
    for k in range(count):
        g = normal_cells(_Flat(n), seed * 1000003 + k, 1.0)
        out[k] = g / np.linalg.norm(g)
    return out


class _Flat:
    def __init__(self, n: int):
        self.ncells = n


def gauss_lobatto_nodes(degree: int) -> np.ndarray:
    """Support points of FE_Q(degree) on [0, 1] (Gauss-Lobatto nodes, degree <= 4)."""
    s5, s37 = 1.0 / np.sqrt(5.0), np.sqrt(3.0 / 7.0)
    table = {1: [-1.0, 1.0], 2: [-1.0, 0.0, 1.0], 3: [-1.0, -s5, s5, 1.0], 4: [-1.0, -s37, 0.0, s37, 1.0]}
    return 0.5 * (np.asarray(table[degree]) + 1.0)


def lattice_coords(mesh):
    """Support-point coordinates (X, Y, Z) of every DoF in lexicographic order (x fastest)."""
    cells = getattr(mesh, "cells", None) or mesh.m
    nodes = gauss_lobatto_nodes(mesh.degree)
    axes = []
    for d in range(3):
        h = mesh.length[d] / cells[d]
        x = np.empty(mesh.degree * cells[d] + 1)
        for c in range(cells[d]):
            x[c * mesh.degree:(c + 1) * mesh.degree + 1] = mesh.origin[d] + h * (c + nodes)
        axes.append(x)
    Z, Y, X = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return X.ravel(), Y.ravel(), Z.ravel()


def moving_gaussian(mesh, n_steps: int, dt: float, start=(0.2, 0.5, 0.95), velocity=(30.0, 0.0, 0.0),
                    width: float = 0.05) -> np.ndarray:
    """Unit-amplitude moving heat source qhat_n(x) = exp(-2 |x - x0(t_n)|^2 / width^2), t_n = n dt,
    x0(t) = start + velocity t, sampled at the support points; shape (n_steps, n_dofs)."""
    X, Y, Z = lattice_coords(mesh)
    out = np.empty((n_steps, X.size))
    for s in range(n_steps):
        t = (s + 1) * dt
        c = [start[d] + velocity[d] * t for d in range(3)]
        out[s] = np.exp(-2.0 * ((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) / width ** 2)
    return out
