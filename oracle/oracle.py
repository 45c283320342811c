"""CPU ORACLE (test infrastructure only) -- ctypes front end of oracle/liborc.so.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import this module.
The product library never calls it.

The C++ restatement it wraps (``oracle/mpdg_oracle.cpp``) follows MeltPoolDG's matrix-free heat
operator (source/heat/heat_diffuse_operator.cpp:179-197, 271-284, 393-529, 955-1086), its
advection-diffusion operator (source/level_set/advection_diffusion_operator.cpp:236-495) and the
SolverCG / right-preconditioned SolverGMRES calls of
include/meltpooldg/linear_algebra/linear_solver.hpp:26-134.

Parity pins (see tests/test_oracle_*.py): an independently assembled sparse matrix
(tests/assembled.py), analytic identities, and the reference's own golden logs
(applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/
unidirectional_heat_transfer.mpirun=4.output and applications/mp-advec-diff/cases/tests/
advection_diffusion_vortex_mf_3d.mpirun=4.output) reproduced in tests/test_oracle_golden.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc.so")


def build() -> str:
    """Compile oracle/liborc.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class OrcOp(C.Structure):
    _fields_ = [
        ("degree", C.c_int32),
        ("m", C.c_int32 * 3),
        ("origin", C.c_double * 3),
        ("length", C.c_double * 3),
        ("cmask", C.c_void_p),
        ("kind", C.c_int32),
        ("pad_", C.c_int32),
        ("rho_cp", C.c_double),
        ("dt", C.c_double),
        ("k_const", C.c_double),
        ("k_cell", C.c_void_p),
        ("theta", C.c_double),
        ("eps", C.c_double),
        ("vel", C.c_double * 12),
        ("imask", C.c_void_p),
    ]


_lib = None


def use_native_build() -> str:
    """Switch this process to liborc_native.so (-march=native, built here on first use), for the timed
    CPU baseline; must run before the first oracle call.  Returns the library path."""
    global _LIB_PATH
    if _lib is not None:
        raise RuntimeError("the oracle library is already loaded")
    # always rebuilt: a copy built on another host may use instructions this one lacks
    native = os.path.join(_HERE, "liborc_native.so")
    if os.path.exists(native):
        os.remove(native)
    subprocess.run(["make", "-s", "-C", _HERE, "native"], check=True)
    _LIB_PATH = native
    return native


def host_cpu() -> dict:
    """Host CPU description for the baseline record: logical CPUs, physical cores, model name."""
    info = {"logical_cpus": os.cpu_count()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=20).stdout
        kv = {}
        for ln in out.splitlines():
            if ":" in ln:
                k, v = ln.split(":", 1)
                kv[k.strip()] = v.strip()
        info["model"] = kv.get("Model name")
        tpc, cps, sockets = (int(kv.get(k, "0") or 0) for k in ("Thread(s) per core", "Core(s) per socket", "Socket(s)"))
        if cps and sockets:
            info["physical_cores"] = cps * sockets
        info["threads_per_core"] = tpc
    except Exception:
        pass
    return info


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.POINTER(OrcOp)
        dp = C.c_void_p
        for name, args, res in [
            ("orc_apply", [P, dp, dp], C.c_int),
            ("orc_apply_add", [P, dp, dp], C.c_int),
            ("orc_apply_batched", [P, dp, dp], C.c_int),
            ("orc_create_rhs", [P, dp, dp, dp, dp], C.c_int),
            ("orc_diagonal", [P, dp], C.c_int),
            ("orc_inverse_diagonal", [P, dp], C.c_int),
            ("orc_cell_stiffness_form", [P, dp, dp, dp], C.c_int),
            ("orc_l2_norm", [P, dp], C.c_double),
            ("orc_dot", [dp, dp, C.c_int64], C.c_double),
            ("orc_n_dofs", [P], C.c_int64),
            ("orc_basis", [C.c_int, dp, dp, dp, dp, dp], C.c_int),
            ("orc_cg", [P, dp, dp, dp, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_int), dp], C.c_int),
            ("orc_gmres", [P, dp, dp, dp, C.c_int, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_int), dp], C.c_int),
            ("orc_num_threads", [], C.c_int),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


@dataclass
class Mesh:
    """Structured box of m[0] x m[1] x m[2] axis-aligned hexahedra, FE_Q(degree)."""

    degree: int
    m: Sequence[int]
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    length: Sequence[float] = (1.0, 1.0, 1.0)

    @property
    def n(self):
        return tuple(self.degree * mi + 1 for mi in self.m)

    @property
    def ndofs(self) -> int:
        a, b, c = self.n
        return a * b * c

    @property
    def ncells(self) -> int:
        return int(np.prod(self.m))

    def basis(self):
        return basis(self.degree)

    def coords_1d(self, d: int) -> np.ndarray:
        nodes = basis(self.degree)[0]
        h = self.length[d] / self.m[d]
        x = np.empty(self.n[d])
        for c in range(self.m[d]):
            x[c * self.degree:(c + 1) * self.degree + 1] = self.origin[d] + h * (c + nodes)
        x[-1] = self.origin[d] + self.length[d]
        return x

    def coords(self):
        """Support-point coordinates (X, Y, Z) of every DoF, lexicographic (x fastest)."""
        x, y, z = (self.coords_1d(d) for d in range(3))
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        return X.ravel(), Y.ravel(), Z.ravel()

    def face_mask(self, faces: int) -> np.ndarray:
        """uint8 Dirichlet flags for whole box faces; bit 2d = low face of dim d, bit 2d+1 = high."""
        nx, ny, nz = self.n
        mask = np.zeros((nz, ny, nx), dtype=np.uint8)
        if faces & 1:
            mask[:, :, 0] = 1
        if faces & 2:
            mask[:, :, -1] = 1
        if faces & 4:
            mask[:, 0, :] = 1
        if faces & 8:
            mask[:, -1, :] = 1
        if faces & 16:
            mask[0, :, :] = 1
        if faces & 32:
            mask[-1, :, :] = 1
        return mask.ravel()


def basis(degree: int):
    n = degree + 1
    nodes, qp, qw = np.zeros(n), np.zeros(n), np.zeros(n)
    B, G = np.zeros(n * n), np.zeros(n * n)
    rc = lib().orc_basis(degree, _ptr(nodes), _ptr(qp), _ptr(qw), _ptr(B), _ptr(G))
    if rc:
        raise ValueError("unsupported degree")
    return nodes, qp, qw, B.reshape(n, n), G.reshape(n, n)


@dataclass
class Operator:
    """Oracle operator: kind 'heat' (rho_cp/dt M + div k grad) or 'advdiff'."""

    mesh: Mesh
    kind: str = "heat"
    cmask: Optional[np.ndarray] = None
    rho_cp: float = 1.0
    dt: float = 1.0
    k: float = 1.0
    k_cell: Optional[np.ndarray] = None
    theta: float = 1.0
    eps: float = 0.0
    vel: Sequence[float] = field(default_factory=lambda: [0.0] * 12)
    imask: Optional[np.ndarray] = None  # advection inflow DoFs: identity rows (do_pre/post_vmult)

    def _struct(self) -> OrcOp:
        s = OrcOp()
        s.degree = self.mesh.degree
        for d in range(3):
            s.m[d] = int(self.mesh.m[d])
            s.origin[d] = float(self.mesh.origin[d])
            s.length[d] = float(self.mesh.length[d])
        if self.cmask is not None:
            self._cm = np.ascontiguousarray(self.cmask, dtype=np.uint8)
            assert self._cm.size == self.mesh.ndofs
            s.cmask = self._cm.ctypes.data
        else:
            s.cmask = None
        s.kind = 0 if self.kind == "heat" else 1
        s.rho_cp, s.dt, s.k_const = self.rho_cp, self.dt, self.k
        if self.k_cell is not None:
            self._kc = np.ascontiguousarray(self.k_cell, dtype=np.float64)
            assert self._kc.size == self.mesh.ncells
            s.k_cell = self._kc.ctypes.data
        else:
            s.k_cell = None
        s.theta, s.eps = self.theta, self.eps
        for i in range(12):
            s.vel[i] = float(self.vel[i])
        if self.imask is not None:
            self._im = np.ascontiguousarray(self.imask, dtype=np.uint8)
            assert self._im.size == self.mesh.ndofs
            s.imask = self._im.ctypes.data
        else:
            s.imask = None
        return s

    def with_(self, **kw) -> "Operator":
        d = dict(self.__dict__)
        d = {k: v for k, v in d.items() if not k.startswith("_")}
        d.update(kw)
        return Operator(**d)

    # -- OperatorMatrixFree-shaped methods -------------------------------------------------------
    def vmult(self, src: np.ndarray) -> np.ndarray:
        s = self._struct()
        src = np.ascontiguousarray(src, dtype=np.float64)
        dst = np.zeros(self.mesh.ndofs)
        lib().orc_apply(C.byref(s), _ptr(src), _ptr(dst))
        return dst

    def vmult_batched(self, src: np.ndarray) -> np.ndarray:
        """Heat vmult by cell-batched SIMD sum factorisation (the timed CPU baseline)."""
        s = self._struct()
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = np.empty(self.mesh.ndofs)
        if lib().orc_apply_batched(C.byref(s), _ptr(src), _ptr(out)) != 0:
            raise ValueError("the batched apply covers the heat operator only")
        return out

    def vmult_add(self, dst: np.ndarray, src: np.ndarray) -> None:
        s = self._struct()
        src = np.ascontiguousarray(src, dtype=np.float64)
        lib().orc_apply_add(C.byref(s), _ptr(src), _ptr(dst))

    def create_rhs(self, dst: np.ndarray, a, b=None, c=None) -> None:
        """Accumulating RHS; heat: (T, T_old, q), advection: (u_old,)."""
        s = self._struct()
        arrs = [None if v is None else np.ascontiguousarray(v, dtype=np.float64) for v in (a, b, c)]
        lib().orc_create_rhs(C.byref(s), _ptr(dst), *[_ptr(v) for v in arrs])

    def diagonal(self) -> np.ndarray:
        s = self._struct()
        d = np.zeros(self.mesh.ndofs)
        lib().orc_diagonal(C.byref(s), _ptr(d))
        return d

    def inverse_diagonal(self) -> np.ndarray:
        s = self._struct()
        d = np.zeros(self.mesh.ndofs)
        lib().orc_inverse_diagonal(C.byref(s), _ptr(d))
        return d

    def cell_stiffness_form(self, lam: np.ndarray, T: np.ndarray) -> np.ndarray:
        s = self._struct()
        out = np.zeros(self.mesh.ncells)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        lib().orc_cell_stiffness_form(C.byref(s), _ptr(lam), _ptr(T), _ptr(out))
        return out

    def l2_norm(self, u: np.ndarray) -> float:
        s = self._struct()
        u = np.ascontiguousarray(u, dtype=np.float64)
        return lib().orc_l2_norm(C.byref(s), _ptr(u))


def inflow_dofs(mesh: Mesh, vel, faces: int = 63) -> np.ndarray:
    """uint8 flags of the inflow DoFs of an inflow/outflow condition on the box faces in `faces`
    (bit 2d low / 2d+1 high face of dim d): every support point of such a face where the outward
    normal n and the velocity v (affine, vel[0..2] + G x) satisfy n . v <= 0, as
    AdvectionDiffusionOperation::create_inflow_outflow_constraints
    (source/level_set/advection_diffusion_operation.cpp:369-499) collects them face by face."""
    X, Y, Z = mesh.coords()
    P = np.stack([X, Y, Z])
    v = np.asarray(vel[:3], dtype=np.float64)[:, None] + np.asarray(vel[3:12], dtype=np.float64).reshape(3, 3) @ P
    nx, ny, nz = mesh.n
    I = np.tile(np.arange(nx), ny * nz)
    J = np.tile(np.repeat(np.arange(ny), nx), nz)
    K = np.repeat(np.arange(nz), nx * ny)
    lat = (I, J, K)
    flags = np.zeros(mesh.ndofs, dtype=np.uint8)
    for f in range(6):
        if not (faces >> f) & 1:
            continue
        d, side = f // 2, f % 2
        on = lat[d] == (mesh.n[d] - 1 if side else 0)
        nv = v[d] if side else -v[d]
        flags[on & (nv <= 0.0)] = 1
    return flags


class NoConvergence(RuntimeError):
    pass


def solve(op: Operator, x: np.ndarray, b: np.ndarray, solver: str = "cg", inv_diag=None,
          max_it: int = 10000, abs_tol: float = 1e-20, rel_tol: float = 1e-12, restart: int = 30,
          history: bool = False):
    """LinearSolver::solve restated: returns (iterations, residual history or None).

    Raises NoConvergence like SolverControl::NoConvergence (linear_solver.hpp:124-129)."""
    s = op._struct()
    b = np.ascontiguousarray(b, dtype=np.float64)
    assert x.dtype == np.float64 and x.flags["C_CONTIGUOUS"]
    it = C.c_int(0)
    hist = np.zeros(max_it + 2) if history else None
    inv = None if inv_diag is None else np.ascontiguousarray(inv_diag, dtype=np.float64)
    if solver == "cg":
        rc = lib().orc_cg(C.byref(s), _ptr(inv), _ptr(x), _ptr(b), max_it, abs_tol, rel_tol,
                          C.byref(it), _ptr(hist))
    elif solver == "gmres":
        rc = lib().orc_gmres(C.byref(s), _ptr(inv), _ptr(x), _ptr(b), max_it, abs_tol, rel_tol,
                             restart, C.byref(it), _ptr(hist))
    else:
        raise ValueError(solver)
    if rc != 0:
        raise NoConvergence(f"{solver} did not converge in {it.value} iterations")
    return it.value, (hist[: it.value + 1] if history else None)


def num_threads() -> int:
    return lib().orc_num_threads()
