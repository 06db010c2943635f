"""The FRSolver-shaped C++ class of include/zb_frsolver.hpp, compiled with the
host compiler and linked against libzefr_b200.so, driven the way the
reference's driver drives FRSolver (tests/native/frsolver_shim.cpp).

On the CPU: the header compiles, links and, with no GPU, turns the library's
error status into std::runtime_error with its message.  On the GPU: the
residual (whole and split), one RK44 step and the state access through the
reference's strides equal the Python binding's results bit for bit and the
reference's golden residual to 1e-12."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import golden_cases as gc
from zefr_b200 import meshgen
from zefr_b200.solver import FRSolver, params_from_reference

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CXX = shutil.which("g++") or shutil.which("c++")


def _build(tmp_path):
    exe = str(tmp_path / "frsolver_shim")
    lib = os.path.join(ROOT, "zefr_b200")
    subprocess.run([CXX, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include", os.path.join(HERE, "native", "frsolver_shim.cpp"), "-o", exe,
                    "-L", lib, "-lzefr_b200", "-Wl,-rpath," + lib], check=True, capture_output=True, timeout=300)
    return exe


def _inputs(tmp_path, name="quad_p3_euler_vortex"):
    g = gc.load(name)
    msh = str(tmp_path / "case.msh")
    meshgen.write_gmsh(g.mesh, msh)
    p = params_from_reference(g.params, g.order)
    pfile = str(tmp_path / "params.bin")
    with open(pfile, "wb") as f:
        f.write(ctypes.string_at(ctypes.addressof(p), ctypes.sizeof(p)))
    ufile = str(tmp_path / "U.bin")
    np.ascontiguousarray(g.U0).tofile(ufile)
    return g, p, msh, pfile, ufile


@pytest.mark.skipif(CXX is None, reason="no host C++ compiler")
def test_shim_compiles_and_reports_errors(tmp_path):
    exe = _build(tmp_path)
    g, p, msh, pfile, ufile = _inputs(tmp_path)
    r = subprocess.run([exe, msh, pfile, ufile, str(tmp_path / "out.bin")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok ") or (r.stdout.startswith("no device: ") and len(r.stdout.strip()) > 12)


@pytest.mark.gpu
def test_shim_matches_python_binding_and_reference(tmp_path):
    exe = _build(tmp_path)
    g, p, msh, pfile, ufile = _inputs(tmp_path)
    out = str(tmp_path / "out.bin")
    r = subprocess.run([exe, msh, pfile, ufile, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok "), r.stdout + r.stderr
    n = g.U0.size
    data = np.fromfile(out, dtype=np.float64)
    assert data.size == 3 * n
    R0, R1, U1 = (data[i * n:(i + 1) * n].reshape(g.U0.shape) for i in range(3))
    s = FRSolver(g.mesh, p, g.bounds)
    assert np.array_equal(R0, s.residual(g.U0, 0))
    assert np.array_equal(R1, R0)
    assert gc.rel_err(R0, g.R0) < 1e-12
    s.set_state(g.U0)
    s.step(1)
    assert np.array_equal(U1, s.get_state())
