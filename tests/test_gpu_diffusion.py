"""GPU parity of the tet4 scalar-diffusion path against the oracle, through the
C-ABI: mesh set-up, assembly (FP64 to 1e-12, the FP32-stored form to FP32
rounding), solve and correction steps, the golden fixture, determinism."""
import os

import numpy as np
import pytest

from openaccel_b200 import meshgen

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def rt():
    from openaccel_b200 import runtime

    runtime.lib()
    return runtime


def _case(n=5, perturb=0.2, seed=31):
    m, g, s, _ = meshgen.conduction(n, sigma=1.0, seed=seed, perturb=perturb)
    phi = np.random.Generator(np.random.PCG64(seed + 1)).uniform(0.0, 1.0, m.nn)
    return m, g, s, phi


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_tet4_mesh_graph_and_volume(rt, oracle_mod):
    m, g, s, _ = _case()
    M = rt.Mesh(m)
    c = oracle_mod.DiffCase(m, g, s)
    rp, cols = M.graph()
    orp, ocols = c.graph()
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(cols, ocols)
    assert _rel(M.dual_volume(), c.field("vol")) <= 1e-13


@pytest.mark.parametrize("shifted", [1, 0])
def test_diffusion_assembly_fp64(rt, oracle_mod, shifted):
    m, g, s, phi = _case()
    M = rt.Mesh(m)
    d = rt.Diffusion(M, rt.default_diffusion_settings(shifted=shifted, urf=0.8))
    c = oracle_mod.DiffCase(m, g, s, oracle_mod.default_diff_settings(shifted=shifted, urf=0.8))
    for name, v in [("gamma", g), ("src", s), ("phi", phi)]:
        d.set_field(name, v)
    c.field("phi")[:] = phi
    A, b = d.assemble()
    Ao, bo = c.assemble()
    assert _rel(A, Ao) <= 1e-12
    assert _rel(b, bo) <= 1e-12


def test_diffusion_assembly_mixed(rt, oracle_mod):
    m, g, s, phi = _case()
    M = rt.Mesh(m)
    d = rt.Diffusion(M, rt.default_diffusion_settings(precision=rt.OA_PREC_MIXED))
    c = oracle_mod.DiffCase(m, g, s)
    for name, v in [("gamma", g), ("src", s), ("phi", phi)]:
        d.set_field(name, v)
    c.field("phi")[:] = phi
    A, b = d.assemble()
    Ao, bo = c.assemble()
    assert _rel(A, Ao) <= 1e-6  # FP32-stored matrix
    assert _rel(b, bo) <= 1e-12  # the rhs stays FP64


def test_diffusion_solve_matches_direct(rt, oracle_mod):
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla

    m, g, s, phi = _case(n=6)
    M = rt.Mesh(m)
    c = oracle_mod.DiffCase(m, g, s)
    c.field("phi")[:] = phi
    Ao, bo = c.assemble()
    rp, cols = c.graph()
    xd = sla.spsolve(sp.csr_matrix((Ao, cols, rp), shape=(m.nn, m.nn)).tocsc(), bo)
    for amg in (1, 0):
        d = rt.Diffusion(M, rt.default_diffusion_settings(amg=amg))
        for name, v in [("gamma", g), ("src", s), ("phi", phi)]:
            d.set_field(name, v)
        d.assemble(copy=False)
        x, it, res, _ = d.solve(rtol=1e-13, maxit=4000)
        assert res <= 1e-13
        assert _rel(x, xd) <= 1e-10


def test_diffusion_steps_fp64(rt, oracle_mod):
    m, g, s, _ = _case(n=5)
    M = rt.Mesh(m)
    d = rt.Diffusion(M, rt.default_diffusion_settings(rtol=1e-13))
    c = oracle_mod.DiffCase(m, g, s, oracle_mod.default_diff_settings(rtol=1e-13))
    d.set_field("gamma", g)
    d.set_field("src", s)
    for _ in range(4):
        st = d.step()
        c.step()
        assert st["res"] <= 1e-13
    assert _rel(d.get_field("phi"), c.field("phi")) <= 1e-10


def test_diffusion_steps_mixed_within_1e6(rt, oracle_mod):
    m, g, s, _ = _case(n=6)
    M = rt.Mesh(m)
    d = rt.Diffusion(M, rt.default_diffusion_settings(precision=rt.OA_PREC_MIXED, rtol=1e-10))
    c = oracle_mod.DiffCase(m, g, s, oracle_mod.default_diff_settings(rtol=1e-13))
    d.set_field("gamma", g)
    d.set_field("src", s)
    for _ in range(4):
        st = d.step()
        c.step()
        assert st["res"] <= 1e-10 and st["refinements"] >= 1
    assert _rel(d.get_field("phi"), c.field("phi")) <= 1e-6


def test_diffusion_golden_fixture(rt):
    ref = np.load(os.path.join(ROOT, "tests", "golden", "conduction4_perturbed.npz"))
    m, g, s, _ = meshgen.conduction(4, sigma=1.0, seed=4242, perturb=0.2)
    M = rt.Mesh(m)
    rp, cols = M.graph()
    np.testing.assert_array_equal(rp, ref["row_ptr"])
    np.testing.assert_array_equal(cols, ref["cols"])
    assert _rel(M.dual_volume(), ref["vol"]) <= 1e-13
    d = rt.Diffusion(M, rt.default_diffusion_settings(rtol=1e-13, maxit=5000))
    d.set_field("gamma", g)
    d.set_field("src", s)
    d.set_field("phi", ref["phi0"])
    A, b = d.assemble()
    assert _rel(A, ref["A"]) <= 1e-12
    assert _rel(b, ref["b"]) <= 1e-12
    d.set_field("phi", np.zeros(m.nn))
    for _ in range(3):
        d.step()
    assert _rel(d.get_field("phi"), ref["phi_it3"]) <= 1e-10


def test_diffusion_assembly_deterministic(rt):
    m, g, s, phi = _case(n=8)
    M = rt.Mesh(m)
    d = rt.Diffusion(M)
    for name, v in [("gamma", g), ("src", s), ("phi", phi)]:
        d.set_field(name, v)
    A1, b1 = d.assemble()
    A2, b2 = d.assemble()
    assert np.array_equal(A1, A2) and np.array_equal(b1, b2)


def test_topology_checks(rt):
    import ctypes as C

    hexm = rt.Mesh(meshgen.cavity(3))
    s = rt.default_diffusion_settings()
    h = C.c_void_p()
    assert rt.lib().oa_diffusion_create(hexm.h, C.byref(s), None, None, 0, C.byref(h)) == 2  # OA_ERR_MESH
    m, _, _, _ = _case(n=3)
    tetm = rt.Mesh(m)
    fs = rt.default_settings()
    bv = np.zeros(3)
    assert rt.lib().oa_flow_create(tetm.h, C.byref(fs), rt._dp(bv), 1, C.byref(h)) == 2
