"""The C++ host layer (include/mpdg/mpdg.hpp) over the C ABI: it compiles and links here (no GPU),
and on the GPU it reproduces the reference's unidirectional heat log through its Newton /
time-step classes (the same values as tests/test_gpu_golden.py gets through the Python layer)."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "meltpooldg_b200")
CUDA = "/usr/local/cuda"


def build_program(tmp_path, name="heat_newton"):
    exe = str(tmp_path / name)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
           "-o", exe, "-L", LIBDIR, "-lmpdg_b200", "-Wl,-rpath," + LIBDIR, "-L", os.path.join(CUDA, "lib64"),
           "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_host_layer_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libmpdg_b200.so")):
        pytest.skip("library not built")
    build_program(tmp_path)
    build_program(tmp_path, "heat_radiation")
    build_program(tmp_path, "heat_predictor")
    build_program(tmp_path, "heat_solidification")
    build_program(tmp_path, "level_set_step")


@pytest.mark.gpu
def test_cpp_newton_time_steps_reproduce_reference_log(tmp_path):
    from oracle.oracle import Operator as OOp
    from tests.cases import heat_unidirectional

    exe = build_program(tmp_path)
    out = str(tmp_path / "T.bin")
    r = subprocess.run([exe, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    om, _ = heat_unidirectional()
    T = np.fromfile(out, dtype=np.float64).reshape(5, om.ndofs)
    norm = OOp(om, "heat", dt=1e-4)
    got = ["%.5e" % norm.l2_norm(T[s]) for s in range(5)]
    gold = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_logs.json")))
    assert got == gold["heat_unidirectional_2d_q1"]["values"]


def oracle_radiation_steps():
    """The time steps of tests/cpp/heat_radiation.cpp on the oracle: Newton on the cell oracle plus
    oracle/faces.py, each linear step solved by Jacobi-CG (scipy) to 1e-14, to a correction below
    1e-12 of the temperature."""
    from scipy.sparse.linalg import LinearOperator, cg

    from oracle.faces import HeatBC, face_diagonal, face_rhs, face_tangent
    from oracle.oracle import Mesh as OMesh
    from oracle.oracle import Operator as OOp

    om = OMesh(2, (8, 8, 8))
    o = OOp(om, "heat", rho_cp=1.0, dt=1e-2, k=1.0)
    bc = HeatBC(convection_faces=0b000011, convection_coefficient=10.0, convection_temperature_infinity=300.0,
                radiation_faces=0b111100, emissivity=0.6, radiation_temperature_infinity=300.0)
    n = om.ndofs
    X, _, _ = om.coords()
    T = 1000.0 - 300.0 * X
    steps = []
    cell_diag = o.diagonal()
    for _ in range(3):
        T_old = T.copy()
        for _ in range(30):
            r = np.zeros(n)
            o.create_rhs(r, T, T_old, None)
            r += face_rhs(om, None, bc, T)
            Tl = T.copy()
            J = LinearOperator((n, n), matvec=lambda v, Tl=Tl: o.vmult(v) + face_tangent(om, None, bc, Tl, v))
            P = 1.0 / (cell_diag + face_diagonal(om, None, bc, Tl))
            d, info = cg(J, r, rtol=1e-14, atol=0.0, maxiter=10000, M=LinearOperator((n, n), matvec=lambda v: P * v))
            assert info == 0
            T = T + d
            if np.linalg.norm(d) <= 1e-12 * np.linalg.norm(T):
                break
        steps.append(T.copy())
    return np.array(steps)


@pytest.mark.gpu
def test_cpp_newton_with_radiation_faces_matches_oracle(tmp_path):
    exe = build_program(tmp_path, "heat_radiation")
    out = str(tmp_path / "T.bin")
    r = subprocess.run([exe, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ref = oracle_radiation_steps()
    got = np.fromfile(out, dtype=np.float64).reshape(ref.shape)
    for s in range(ref.shape[0]):
        assert np.max(np.abs(got[s] - ref[s])) <= 1e-9 * np.max(np.abs(ref[s]))
    # the radiation and convection faces cool the block
    assert ref[-1].mean() < (1000.0 - 150.0)


@pytest.mark.gpu
def test_cpp_predictors_match_oracle(tmp_path):
    """Each predicted temperature of tests/cpp/heat_predictor.cpp equals the oracle's predictor applied
    to the same solution history (the program's own converged solutions), and all predictors reach
    the same solutions."""
    from oracle.faces import HeatBC, face_rhs, face_tangent
    from oracle.oracle import Mesh as OMesh
    from oracle.oracle import Operator as OOp
    from oracle.predictor import least_squares_projection, linear_extrapolation

    exe = build_program(tmp_path, "heat_predictor")
    prefix = str(tmp_path / "pred")
    r = subprocess.run([exe, prefix], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    om = OMesh(2, (8, 8, 8))
    cm = om.face_mask(0b000001)
    bc = HeatBC(convection_faces=0b000010, convection_coefficient=10.0, convection_temperature_infinity=300.0,
                radiation_faces=0b111100, emissivity=0.6, radiation_temperature_infinity=300.0)
    n = om.ndofs
    X, _, _ = om.coords()
    T0 = 1000.0 - 300.0 * X
    dts = [1e-2, 1e-2, 2e-2, 1e-2, 1.5e-2]
    finals = {}
    for kind in ("none", "zero", "linear_extrapolation", "least_squares_projection"):
        data = np.fromfile(prefix + "_" + kind + ".bin", dtype=np.float64).reshape(len(dts), 2, n)
        hist = [T0, T0, T0]  # max(n_old_solution_vectors = 3, 2) vectors, all the initial solution
        for k, dt in enumerate(dts):
            pred, sol = data[k]
            s0, s1 = hist[0], hist[1]
            tol = 1e-13
            if kind == "none":
                ref = s0.copy()
            elif kind == "zero":
                ref = np.zeros(n)
            elif kind == "linear_extrapolation":
                ref = linear_extrapolation(s0, s1, dt, dts[k - 1] if k else dt)
            elif k >= 3:
                o = OOp(om, "heat", cmask=cm, rho_cp=1.0, dt=dt, k=1.0)
                rhs = np.zeros(n)
                o.create_rhs(rhs, s0, s0, None)
                rhs += face_rhs(om, cm, bc, s0)
                ref = least_squares_projection(lambda v: o.vmult(v) + face_tangent(om, cm, bc, s0, v), rhs, hist)
                tol = 1e-8
            else:
                ref = s0.copy()
            ref = np.where(cm != 0, s0, ref)  # Dirichlet values of the previous solution
            assert np.max(np.abs(pred - ref)) <= tol * np.max(np.abs(ref)), (kind, k)
            hist = [sol] + hist[:-1]
        finals[kind] = data[-1, 1]
    for kind, T in finals.items():
        assert np.max(np.abs(T - finals["none"])) <= 1e-9 * np.max(np.abs(T)), kind


def oracle_solidification_steps():
    """The time steps of tests/cpp/heat_solidification.cpp on the oracle: Newton on
    oracle/solidification.py, each linear step by Jacobi-GMRES (scipy) to 1e-13, to a correction
    below 1e-12 of the temperature."""
    from scipy.sparse.linalg import LinearOperator, gmres

    from oracle.oracle import Mesh as OMesh
    from oracle.solidification import SolidLiquid, diagonal, residual, tangent_apply

    om = OMesh(2, (8, 8, 8))
    cm = om.face_mask(0b000001)
    mat = SolidLiquid((7.4, 0.8, 30.0), (7.9, 0.6, 20.0), 1700.0, 1600.0)
    n, dt = om.ndofs, 2e-3
    X, _, _ = om.coords()
    T = 1500.0 + 250.0 * X
    steps = []
    for _ in range(3):
        T_old = T.copy()
        for _ in range(30):
            r = residual(om, cm, mat, dt, T, T_old)
            Tl = T.copy()
            A = LinearOperator((n, n), matvec=lambda v, Tl=Tl: tangent_apply(om, cm, mat, dt, Tl, T_old, v)
                               + np.where(cm != 0, v, 0.0))
            d = diagonal(om, cm, mat, dt, Tl, T_old)
            d[cm != 0] = 1.0
            dT, info = gmres(A, r, rtol=1e-13, atol=0.0, restart=60, maxiter=200,
                             M=LinearOperator((n, n), matvec=lambda v, d=d: v / d))
            assert info == 0
            T = T + np.where(cm != 0, 0.0, dT)
            if np.linalg.norm(dT) <= 1e-12 * np.linalg.norm(T):
                break
        steps.append(T.copy())
    return np.array(steps)


@pytest.mark.gpu
def test_cpp_newton_with_solidification_matches_oracle(tmp_path):
    exe = build_program(tmp_path, "heat_solidification")
    out = str(tmp_path / "T.bin")
    r = subprocess.run([exe, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ref = oracle_solidification_steps()
    got = np.fromfile(out, dtype=np.float64).reshape(ref.shape)
    for s in range(ref.shape[0]):
        assert np.max(np.abs(got[s] - ref[s])) <= 1e-9 * np.max(np.abs(ref[s]))
    # part of the block crosses the mushy zone
    assert np.any((ref[-1] > 1600.0) & (ref[-1] < 1700.0))


def oracle_level_set_step():
    """The chain of tests/cpp/level_set_step.cpp restated with the oracle: SUPG advection (GMRES to
    1e-13 on the oracle operator plus oracle/supg.py), the normal and curvature projections
    (M + h^2 K, oracle CG) and three Olsson steps (oracle/reinit.py, CG to 1e-13)."""
    import scipy.sparse.linalg as spla

    from oracle import reinit as R
    from oracle import supg as S
    from oracle.oracle import Mesh as OMesh
    from oracle.oracle import Operator as OOp
    from oracle.oracle import solve as osolve

    m, k = 12, 2
    h = 1.0 / m
    mesh = OMesh(k, (m, m, m))
    X, Y, Z = mesh.coords()
    r = np.sqrt((X - 0.5) ** 2 + (Y - 0.6) ** 2 + (Z - 0.5) ** 2)
    psi0 = 0.5 * (1.0 - np.tanh((r - 0.25) / 0.04))
    vel = [0.5, -0.5, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0]
    dt, theta, eps, tau = 5e-3, 1.0, 1e-3, 0.1
    adv = OOp(mesh, "advdiff", dt=dt, theta=theta, eps=eps, vel=vel)
    n = mesh.ndofs

    def A(u):
        return adv.vmult(u) + S.supg_apply(mesh, None, vel, tau, 1.0 / dt, theta, theta * eps, u)

    rhs = np.zeros(n)
    adv.create_rhs(rhs, psi0)
    rhs += S.supg_apply(mesh, None, vel, tau, 1.0 / dt, theta - 1.0, (theta - 1.0) * eps, psi0, plain=True)
    d = adv.diagonal() + S.supg_diagonal(mesh, None, vel, tau, 1.0 / dt, theta, theta * eps)
    Aop = spla.LinearOperator((n, n), matvec=A)
    Pop = spla.LinearOperator((n, n), matvec=lambda v: v / d)
    psi, info = spla.gmres(Aop, rhs, x0=psi0.copy(), M=Pop, rtol=1e-13, atol=0.0, restart=60, maxiter=2000)
    assert info == 0
    proj = OOp(mesh, "heat", rho_cp=1.0, dt=1.0, k=h * h)
    inv = proj.inverse_diagonal()
    normal = []
    for c in R.normal_rhs(mesh, None, psi):
        x = np.zeros(n)
        osolve(proj, x, c, "cg", inv, rel_tol=1e-13)
        normal.append(x)
    tol = 1e-10
    kappa = np.zeros(n)
    osolve(proj, kappa, R.curvature_rhs(mesh, None, normal, tol), "cg", inv, rel_tol=1e-13)
    rdt, eps_n, eps_t = 0.25 * h, 0.5 * h, 0.0
    dr = R.diagonal(mesh, None, rdt, eps_n, eps_t, normal, tol)
    Rop = spla.LinearOperator((n, n), matvec=lambda u: R.tangent_apply(mesh, None, rdt, eps_n, eps_t, normal, tol, u))
    Dop = spla.LinearOperator((n, n), matvec=lambda v: v / dr)
    psi_r = psi.copy()
    for _ in range(3):
        b = R.create_rhs(mesh, None, eps_n, eps_t, normal, tol, psi_r)
        dpsi, info = spla.cg(Rop, b, M=Dop, rtol=1e-13, atol=0.0, maxiter=5000)
        assert info == 0
        psi_r = psi_r + dpsi
    return np.array([psi, normal[0], normal[1], normal[2], kappa, psi_r])


@pytest.mark.gpu
def test_cpp_level_set_step_matches_oracle_chain(tmp_path):
    """tests/cpp/level_set_step.cpp (LevelSetOperation::solve's order, source/level_set/
    level_set_operation.cpp:364-387) on the GPU through the C++ host layer, field by field against
    the oracle's chain: each output within 1e-8 of the oracle's (relative to its largest entry)."""
    exe = build_program(tmp_path, "level_set_step")
    out = str(tmp_path / "ls.bin")
    r = subprocess.run([exe, out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    its = json.loads(r.stdout.strip().splitlines()[-1])
    assert its["advection_iterations"] > 0 and its["reinit_iterations"] > 0
    ref = oracle_level_set_step()
    got = np.fromfile(out, dtype=np.float64).reshape(ref.shape)
    for f, name in enumerate(["psi (advected)", "n_x", "n_y", "n_z", "curvature", "psi (reinitialised)"]):
        err = np.max(np.abs(got[f] - ref[f])) / np.max(np.abs(ref[f]))
        assert err <= 1e-8, (name, err)
