"""The C++ side of the drop-in boundary: include/compat/linearSolverContext.h
(the reference's linearSolver::Context / Matrix / Vector surface) and a
reference-style assembler subclass calling the C-ABI (tests/compat_harness.cpp),
compiled with g++ -std=c++20 against the built library.

On the CPU: the block-CSR accessors (rowVals, rowCols, diag, dofDiag), the
C-ABI's argument errors surfacing as std::runtime_error. On the GPU: the
subclass assembles and solves a pressure correction through the Context, and
the result equals the same calls made through the Python binding."""
import os
import subprocess

import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_harness(tmp_path):
    exe = str(tmp_path / "compat_harness")
    libdir = os.path.dirname(rt.LIB_PATH)
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "compat_harness.cpp"), "-L", libdir, "-lopenaccel_b200",
           f"-Wl,-rpath,{libdir}", "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def test_compat_context_on_cpu(tmp_path):
    exe = build_harness(tmp_path)
    r = subprocess.run([exe, "cpu"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "compat cpu ok" in r.stdout


@pytest.mark.gpu
def test_compat_subclass_assembles_and_solves_on_gpu(tmp_path):
    exe = build_harness(tmp_path)
    m = meshgen.cavity(5, perturb=0.2, seed=8)
    np.array([m.nn, m.ne, m.nf, m.bnd_velocity.shape[0]], np.int32).tofile(tmp_path / "sizes.i32")
    m.coords.astype(np.float64).tofile(tmp_path / "coords.f64")
    m.conn.astype(np.int32).tofile(tmp_path / "conn.i32")
    np.stack([m.face_elem, m.face_ord, m.face_bnd], axis=1).astype(np.int32).tofile(tmp_path / "faces.i32")
    m.bnd_velocity.astype(np.float64).tofile(tmp_path / "bnd.f64")
    r = subprocess.run([exe, "gpu", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    A = np.fromfile(tmp_path / "A.f64")
    b = np.fromfile(tmp_path / "b.f64")
    x = np.fromfile(tmp_path / "x.f64")
    # the same sequence through the Python binding
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(mom_rtol=1e-6, pc_rtol=1e-8))
    gf.initialize()
    gf.simple_iterate(1)
    A_r, b_r = gf.assemble_pcorr()
    x_r, _, _ = gf.solve("pcorr", 1e-12, 5000)
    np.testing.assert_array_equal(A, A_r)
    np.testing.assert_array_equal(b, b_r)
    assert np.linalg.norm(x - x_r) <= 1e-10 * np.linalg.norm(x_r)
    it, r0, r1, s0 = open(tmp_path / "control.txt").read().split()
    assert float(s0) == pytest.approx(float(r0) / gf.scales()[1], rel=1e-12)
