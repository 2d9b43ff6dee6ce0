"""Failure paths of the C-ABI, driven by inputs made on the host (no device
fault is provoked): each bad input must come back as its status code with a
message, and the handle must stay usable where the reference's errorMsg
convention would let a caller continue.

- a non-finite value in the field state reaches the solvers as a non-finite
  right-hand side -> OA_ERR_SOLVER (Krylov status 2), in both precisions;
- a hex mesh with a face shared by three elements -> OA_ERR_MESH;
- a hex whose nodes are moved so that it turns inside out -> OA_ERR_GEOMETRY
  (non-positive sub-control volume, the Jacobian determinant check of
  hex_scv_det / hex_gradient_operator);
- an oversize or non-converging allocation-free solve -> its status codes.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu

OA_ERR_MESH, OA_ERR_GEOMETRY, OA_ERR_SOLVER = 2, 3, 5


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_nan_state_is_a_solver_error(prec):
    m = meshgen.cavity(5, perturb=0.2, seed=3)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(precision=prec))
    gf.initialize()
    gf.simple_iterate(1)
    p = gf.get_field("p")
    p[17] = np.nan  # enters the Rhie-Chow fluxes of the pressure-correction rhs
    gf.set_field("p", p)
    gf.assemble_pcorr()
    with pytest.raises(rt.OpenAccelError) as ei:
        gf.solve("pcorr", 1e-8, 100)
    assert ei.value.status == OA_ERR_SOLVER
    assert "non-finite" in str(ei.value)
    U = gf.get_field("U")
    U[3 * 40] = np.inf
    gf.set_field("U", U)
    with pytest.raises(rt.OpenAccelError) as ei:
        gf.simple_iterate(1)
    assert ei.value.status == OA_ERR_SOLVER


def test_face_shared_by_three_elements_is_a_mesh_error():
    m = meshgen.cavity(3)
    bad = dataclasses.replace(m, conn=np.ascontiguousarray(np.concatenate([m.conn, m.conn[4:5]])[::-1]))
    with pytest.raises(rt.OpenAccelError) as ei:
        rt.Mesh(bad)
    assert ei.value.status == OA_ERR_MESH and "invalid hex mesh" in str(ei.value)


def test_inverted_hex_is_a_geometry_error():
    m = meshgen.cavity(4)
    x = m.coords.copy()
    # push an interior node through the opposite faces of its elements
    i = 2 + 5 * (2 + 5 * 2)
    x[i] += np.array([0.9, 0.0, 0.0])
    bad = dataclasses.replace(m, coords=x)
    with pytest.raises(rt.OpenAccelError) as ei:
        rt.Mesh(bad)
    assert ei.value.status == OA_ERR_GEOMETRY
    # a valid mesh is still accepted afterwards (no sticky error state)
    rt.Mesh(m)


def test_static_solve_reports_non_convergence():
    import torch

    m = meshgen.cavity(6, perturb=0.2, seed=21)
    gm = rt.Mesh(m)
    gf = rt.Flow(gm, rt.default_settings())
    gf.initialize()
    gf.simple_iterate(1)
    A, b = gf.assemble_pcorr()
    rp, cols = gm.graph()
    diag = np.array([np.searchsorted(cols[rp[i]:rp[i + 1]], i) for i in range(m.nn)], dtype=np.int32)
    d = {k: torch.from_numpy(v).to("cuda") for k, v in (("rp", rp), ("cols", cols), ("diag", diag), ("A", A),
                                                          ("b", b))}
    x = torch.zeros(m.nn, dtype=torch.float64, device="cuda")
    L = rt.lib()
    it, res = C.c_int(), C.c_double()
    # two iterations cannot reach 1e-12: the call must say so
    st = L.oa_pcorr_solve_static(m.nn, d["rp"].data_ptr(), d["cols"].data_ptr(), d["diag"].data_ptr(),
                                 d["A"].data_ptr(), d["b"].data_ptr(), x.data_ptr(), 1e-12, 2, C.byref(it),
                                 C.byref(res), None)
    assert st == OA_ERR_SOLVER
    assert b"not converged" in L.oa_last_error()
    assert res.value > 1e-12
    # a non-finite right-hand side is reported as such
    d["b"][5] = float("nan")
    st = L.oa_pcorr_solve_static(m.nn, d["rp"].data_ptr(), d["cols"].data_ptr(), d["diag"].data_ptr(),
                                 d["A"].data_ptr(), d["b"].data_ptr(), x.data_ptr(), 1e-8, 50, C.byref(it),
                                 C.byref(res), None)
    assert st == OA_ERR_SOLVER


def test_gcr_stagnation_falls_back_to_bicgstab(monkeypatch):
    """GCR(2) truncated to two directions can stagnate when the symmetric part
    of A M^-1 is not definite. Two random pressure-correction systems (random
    DU, mass flows and pressure on a skewed 12^3 cavity) solved back to back,
    the second with the AMG hierarchy the first one built (the numeric phase is
    refreshed every eighth solve, and the drift test that would refresh it for
    so different a matrix is switched off), make it stagnate: the solve must
    switch to BiCGStab, say so in its ControlData, count the GCR iterations it
    spent, and still reach the direct solution."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    monkeypatch.setenv("OA_AMG_DRIFT", "1e300")

    m = meshgen.cavity(12, perturb=0.2, seed=21)
    gm = rt.Mesh(m)
    gf = rt.Flow(gm, rt.default_settings(precision=rt.OA_PREC_FP64))
    for seed in (1, 2):
        rng = np.random.default_rng(seed)
        gf.set_field("p", rng.normal(0, 1, m.nn))
        gf.set_field("gradP", rng.normal(0, 1, 3 * m.nn))
        gf.set_field("du", rng.uniform(0.1, 1.0, 3 * m.nn))
        gf.set_field("mDot", rng.normal(0, 0.01, 12 * m.ne))
        A, b = gf.assemble_pcorr()
        x, it, res = gf.solve("pcorr", 1e-13, 5000)
        cd = gf.last_control("pcorr")
        if seed == 1:
            assert cd["fallback"] == 0 and res < 1e-12
    assert cd["fallback"] == 1
    assert cd["n_iterations"] == it and it > 2
    assert res < 1e-12
    rp, cols = gm.graph()
    xd = spl.spsolve(sp.csr_matrix((A, cols, rp), shape=(m.nn, m.nn)).tocsc(), b)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9
