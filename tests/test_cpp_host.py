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


def build_program(tmp_path):
    exe = str(tmp_path / "heat_newton")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "heat_newton.cpp"),
           "-o", exe, "-L", LIBDIR, "-lmpdg_b200", "-Wl,-rpath," + LIBDIR, "-L", os.path.join(CUDA, "lib64"),
           "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_host_layer_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libmpdg_b200.so")):
        pytest.skip("library not built")
    build_program(tmp_path)


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
