"""The allocation-free pressure-correction solve, oa_pcorr_solve_static.

It is for callers that cannot allocate device memory when they solve (an
application that owns all device memory and hands out slices itself, a
solver plug-in whose host framework forbids allocation on its hot path): its
work vectors live in a fixed file-scope device array instead of cudaMalloc'd
buffers. These tests call it through the C-ABI on device buffers the test
owns and check it against the regular entry point (oa_solve on the same
assembled system), on two calls in a row with two different systems, so state
left in the shared array by the first call cannot leak into the second; once
at a small size and once at exactly the row limit, where the carve-up of the
static array is tightest, and at a row count that is not a multiple of 32.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def host_residual(rp, cols, A, b, x):
    """||b - A x|| / ||b|| in FP64 on the host, independent of either solver's
    report; its own rounding (||A|| ||x|| eps / ||b||) is of order 1e-12 here,
    so it is held to 1e-11 while the solvers report below 1e-12."""
    import scipy.sparse as sp

    M = sp.csr_matrix((A, cols, rp), shape=(b.size, b.size))
    return np.linalg.norm(b - M @ x) / np.linalg.norm(b)


# Both solves stop at a relative residual below 1e-12; the solutions then agree
# to about cond(A) times that. The pressure-correction operator of these
# meshes has a condition number of order 1e4, so 1e-8 leaves a margin while
# staying five decades below the gap between the two systems (> 1e-3).
X_TOL = 1e-8


def _system(gf, seed):
    """Assemble the pressure-correction system of a flow state: a seeded
    Gaussian initial velocity, one SIMPLE outer iteration, then the assembly
    the next iteration would solve."""
    m = gf.mesh.src
    gf.set_field("U", meshgen.initial_velocity(m, sigma=0.1, seed=seed))
    gf.set_field("p", np.zeros(m.nn))
    gf.initialize()
    gf.simple_iterate(1)
    A, b = gf.assemble_pcorr()
    x_ref, _, res_ref = gf.solve("pcorr", 1e-13, 5000)
    assert res_ref < 1e-12
    return A, b, x_ref


def _static_solve(dev, A, b):
    import torch

    L = rt.lib()
    x = torch.zeros(b.size, dtype=torch.float64, device="cuda")
    Ad = torch.from_numpy(A).to("cuda")
    bd = torch.from_numpy(b).to("cuda")
    it, res = C.c_int(), C.c_double()
    st = L.oa_pcorr_solve_static(dev["nn"], dev["rp"].data_ptr(), dev["cols"].data_ptr(), dev["diag"].data_ptr(),
                                 Ad.data_ptr(), bd.data_ptr(), x.data_ptr(), 1e-13, 5000, C.byref(it),
                                 C.byref(res), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, L.oa_last_error().decode()
    torch.cuda.synchronize()
    return x.cpu().numpy(), it.value, res.value


@pytest.mark.parametrize("n", [24, 49, (63, 63, 31)])
def test_static_solve_matches_regular_solve_twice(n):
    import torch

    m = meshgen.cavity(n, perturb=0.2, seed=21)
    assert m.nn <= rt.OA_STATIC_SOLVE_MAX_ROWS
    if not np.isscalar(n):
        assert m.nn == rt.OA_STATIC_SOLVE_MAX_ROWS
    gm = rt.Mesh(m)
    gf = rt.Flow(gm, rt.default_settings())
    rp, cols = gm.graph()
    diag = np.array([np.searchsorted(cols[rp[i]:rp[i + 1]], i) for i in range(m.nn)], dtype=np.int32)
    dev = {"nn": m.nn, "rp": torch.from_numpy(rp).to("cuda"), "cols": torch.from_numpy(cols).to("cuda"),
           "diag": torch.from_numpy(diag).to("cuda")}
    # first call
    A1, b1, x1_ref = _system(gf, seed=1)
    x1, it1, res1 = _static_solve(dev, A1, b1)
    assert res1 < 1e-12 and it1 > 0
    assert host_residual(rp, cols, A1, b1, x1) < 1e-11
    assert rel(x1, x1_ref) < X_TOL
    # second call, different system: the shared array must not carry state over
    A2, b2, x2_ref = _system(gf, seed=2)
    x2, it2, res2 = _static_solve(dev, A2, b2)
    assert res2 < 1e-12
    assert host_residual(rp, cols, A2, b2, x2) < 1e-11
    assert rel(x2, x2_ref) < X_TOL
    assert rel(x2, x1) > 1e-3  # genuinely a different system
    if m.nn <= 20000:
        # and against a direct solve on the host, independent of the library's solvers
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl

        xd = spl.spsolve(sp.csr_matrix((A2, cols, rp), shape=(m.nn, m.nn)).tocsc(), b2)
        assert rel(x2, xd) < 1e-9


def test_static_solve_rejects_oversized_system():
    L = rt.lib()
    n = rt.OA_STATIC_SOLVE_MAX_ROWS + 1
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    it, res = C.c_int(), C.c_double()
    st = L.oa_pcorr_solve_static(n, dummy, dummy, dummy, dummy, dummy, dummy, 1e-8, 10, C.byref(it), C.byref(res),
                                 None)
    assert st == 1
    assert b"exceed the static limit" in L.oa_last_error()
