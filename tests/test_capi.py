"""CPU checks of the C ABI library: it loads and exports every declared entry point."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            txt = open(os.path.join(inc, fn)).read()
            names |= set(re.findall(r"MPDG_API\s+[\w\s\*]+?\b(mpdg_\w+)\s*\(", txt))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "mpdg_op_vmult" in names and "mpdg_solve" in names and len(names) >= 20


def test_library_loads_and_exports_every_symbol():
    from meltpooldg_b200 import _lib
    from meltpooldg_b200.build import build

    build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_signatures_cover_header():
    from meltpooldg_b200 import _lib

    bound = {n for n, _, _ in _lib.SIGNATURES + _lib.OPTIONAL}
    assert declared_symbols() <= bound


def test_invalid_arguments_rejected_without_gpu():
    """Argument checks run before any CUDA call."""
    from meltpooldg_b200 import _lib

    L = _lib.lib()
    h = ctypes.c_void_p()
    mesh = _lib.MeshDesc()
    mesh.degree = 7
    for d in range(3):
        mesh.cells[d] = 2
        mesh.length[d] = 1.0
    p = _lib.OpParams()
    p.kind = _lib.MPDG_HEAT
    p.dt = 1.0
    assert L.mpdg_op_create(ctypes.byref(mesh), ctypes.byref(p), ctypes.byref(h)) == _lib.MPDG_ERR_UNSUPPORTED
    mesh.degree = 2
    p.dt = 0.0
    assert L.mpdg_op_create(ctypes.byref(mesh), ctypes.byref(p), ctypes.byref(h)) == _lib.MPDG_ERR_ZERO_DT
    assert b"ExcZeroTimeIncrement" in L.mpdg_last_error()
    assert L.mpdg_op_vmult(None, None, None) == _lib.MPDG_ERR_ARG


def test_header_compiles_as_c_and_cpp(tmp_path):
    """include/mpdg_gpu.h is plain C (C99) and C++; include/mpdg/mpdg.hpp is C++17."""
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src_c = tmp_path / "h.c"
    src_c.write_text('#include "mpdg_gpu.h"\nint main(void) { return MPDG_OK; }\n')
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I",
                        os.path.join(root, "include"), str(src_c)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    src_cc = tmp_path / "h.cc"
    src_cc.write_text('#include "mpdg/mpdg.hpp"\nint main() { mpdg::LinearSolverData d; return d.restart == 30 ? 0 : 1; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I",
                        os.path.join(root, "include"), str(src_cc)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes structures of meltpooldg_b200/_lib.py have the sizes and field offsets of the C
    structures in include/mpdg_gpu.h (compiled with the host C compiler)."""
    import ctypes as C
    import subprocess

    from meltpooldg_b200 import _lib as L

    structs = {"mpdg_mesh_desc": L.MeshDesc, "mpdg_op_params": L.OpParams, "mpdg_heat_bc": L.HeatBC,
               "mpdg_solid_liquid": L.SolidLiquid, "mpdg_solver_params": L.SolverParams,
               "mpdg_solve_info": L.SolveInfo, "mpdg_mixed_params": L.MixedParams,
               "mpdg_adjoint_params": L.AdjointParams, "mpdg_adjoint_result": L.AdjointResult}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mpdg_gpu.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = str(tmp_path / "layout")
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_missing_library_fails_loudly(tmp_path):
    """Without the CUDA library the Python operators raise instead of falling back to the CPU."""
    import subprocess
    import sys

    code = (
        "from meltpooldg_b200.operators import HeatDiffuseOperator, Mesh\n"
        "try:\n"
        "    HeatDiffuseOperator(Mesh(2, (2, 2, 2)), rho_cp=1.0, dt=1e-3)\n"
        "except ImportError as e:\n"
        "    print('ImportError', e)\n"
        "else:\n"
        "    print('no error')\n"
    )
    env = dict(os.environ, MPDG_LIB_PATH=str(tmp_path / "absent.so"))
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ImportError") and "absent.so" in r.stdout, r.stdout


def test_vector_checks_before_any_kernel():
    """The Python layer refuses vectors that are too short or of the wrong type before a pointer
    reaches the library (a short buffer would be overrun on the device)."""
    import pytest
    import torch

    from meltpooldg_b200.operators import _ptr

    class FakeCuda:
        is_cuda = True

        def __init__(self, n, dtype, contiguous=True):
            self.n, self.dtype, self.contiguous = n, dtype, contiguous

        def is_contiguous(self):
            return self.contiguous

        def numel(self):
            return self.n

        def data_ptr(self):
            return 4096

    assert _ptr(None, 10, torch.float64) is None
    assert _ptr(FakeCuda(10, torch.float64), 10, torch.float64) == 4096
    assert _ptr(FakeCuda(12, torch.float32), 10, torch.float32) == 4096  # a longer buffer is fine
    with pytest.raises(ValueError):
        _ptr(FakeCuda(9, torch.float64), 10, torch.float64)
    with pytest.raises(TypeError):
        _ptr(FakeCuda(10, torch.float32), 10, torch.float64)
    with pytest.raises(ValueError):
        _ptr(FakeCuda(10, torch.float64, contiguous=False), 10, torch.float64)
    with pytest.raises(ValueError):
        _ptr(torch.zeros(10, dtype=torch.float64), 10, torch.float64)  # host memory
