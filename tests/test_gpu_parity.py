"""GPU parity of the CUDA path (through the C-ABI) against the CPU oracle.

Bars: assembled matrices and right-hand sides within 1e-12 relative
(norm-wise) in FP64; converged SIMPLE fields within 1e-10; the mixed form's
fields within 1e-6 of the FP64 oracle.
"""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu

TOL_ASM = 1e-12


def rel(a, b):
    d = np.linalg.norm(np.asarray(a) - np.asarray(b))
    n = np.linalg.norm(np.asarray(b))
    return d / n if n > 0 else d


def make_pair(oracle_mod, n=6, perturb=0.2, seed=11, sigma=0.1, prec=rt.OA_PREC_FP64, **kw):
    m = meshgen.cavity(n, perturb=perturb, seed=seed)
    U0 = meshgen.initial_velocity(m, sigma=sigma, seed=seed)
    s_o = oracle_mod.default_settings(**kw)
    s_g = rt.default_settings(precision=prec, **kw)
    oc = oracle_mod.FlowCase(m, s_o, U0=U0)
    gm = rt.Mesh(m)
    gf = rt.Flow(gm, s_g)
    gf.set_field("U", U0)
    return m, oc, gm, gf


def random_state(m, oc, gf, seed=5):
    """Same random p, gradP, du, mDot in both (assembly parity is state-agnostic)."""
    rng = np.random.default_rng(seed)
    fields = {
        "p": rng.normal(0, 1, m.nn),
        "gradP": rng.normal(0, 1, 3 * m.nn),
        "gradU": rng.normal(0, 1, 9 * m.nn),
        "du": rng.uniform(0.1, 1.0, 3 * m.nn),
        "mDot": rng.normal(0, 0.01, 12 * m.ne),
        "div": rng.normal(0, 1e-3, m.nn),
    }
    for k, v in fields.items():
        oc.field(k)[:] = v
        gf.set_field(k, v)


def test_graph_and_dual_volume(oracle_mod):
    m, oc, gm, gf = make_pair(oracle_mod)
    rp, cols = gm.graph()
    orp, ocols = oc.graph()
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(cols, ocols)
    assert rel(gm.dual_volume(), oc.field("vol")) < 1e-14


@pytest.mark.parametrize("shift", [(1, 1), (0, 1), (1, 0), (0, 0)])
def test_pcorr_assembly_parity(oracle_mod, shift):
    us, gs = shift
    m, oc, gm, gf = make_pair(oracle_mod, n=7, u_shifted=us, p_grad_shifted=gs)
    random_state(m, oc, gf)
    A_o, b_o = oc.assemble_pcorr()
    A_g, b_g = gf.assemble_pcorr()
    assert rel(A_g, A_o) < TOL_ASM
    assert rel(b_g, b_o) < TOL_ASM


@pytest.mark.parametrize("shift", [(1, 1), (0, 1), (1, 0), (0, 0)])
def test_momentum_assembly_parity(oracle_mod, shift):
    us, gs = shift
    m, oc, gm, gf = make_pair(oracle_mod, n=7, u_shifted=us, u_grad_shifted=gs)
    random_state(m, oc, gf)
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    assert rel(A_g, A_o) < TOL_ASM
    assert rel(b_g, b_o) < TOL_ASM
    assert rel(gf.get_field("du"), oc.field("du")) < TOL_ASM


def _variable_properties(m, oc, gf, seed=9):
    """Per-node density and viscosity, and mass flows of which one in ten is
    exactly zero (the upwind choices at a zero flux must match the oracle's)."""
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.5, 2.0, m.nn)
    mu = rng.uniform(0.5e-2, 2e-2, m.nn)
    mdot = rng.normal(0, 0.01, 12 * m.ne)
    mdot[rng.uniform(size=mdot.size) < 0.1] = 0.0
    for k, v in (("rho", rho), ("mu", mu), ("mDot", mdot)):
        oc.field(k)[:] = v
        gf.set_field(k, v)


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_pcorr_assembly_parity_variable_density(oracle_mod, prec):
    # the staged path: per-ip fluxes and corner coefficients from the mass-flow
    # kernel, gathered by the row kernel (FP32 matrix in the mixed form, whose
    # rhs stays FP64)
    m, oc, gm, gf = make_pair(oracle_mod, n=7, prec=prec)
    random_state(m, oc, gf)
    _variable_properties(m, oc, gf)
    A_o, b_o = oc.assemble_pcorr()
    A_g, b_g = gf.assemble_pcorr()
    assert rel(A_g, A_o) < (TOL_ASM if prec == rt.OA_PREC_FP64 else 1e-6)
    assert rel(b_g, b_o) < TOL_ASM


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_momentum_assembly_parity_variable_properties(oracle_mod, prec):
    # the mixed form's fluxes are FP32 arithmetic (Jacobians on FP32 corner
    # offsets, U and mu from an FP32 copy): matrix, rhs and DU (from the FP32
    # diagonal) within 1e-5 of the FP64 oracle, norm-wise
    m, oc, gm, gf = make_pair(oracle_mod, n=7, prec=prec)
    random_state(m, oc, gf)
    _variable_properties(m, oc, gf)
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    tol = TOL_ASM if prec == rt.OA_PREC_FP64 else 1e-5
    assert rel(A_g, A_o) < tol
    assert rel(b_g, b_o) < tol
    assert rel(gf.get_field("du"), oc.field("du")) < tol


def test_mdot_div_gradient_parity(oracle_mod):
    m, oc, gm, gf = make_pair(oracle_mod, n=7)
    random_state(m, oc, gf)
    oc.update_mdot()
    gf.update_mdot()
    assert rel(gf.get_field("mDot"), oc.field("mDot")) < TOL_ASM
    oc.update_div()
    gf.update_div()
    assert rel(gf.get_field("div"), oc.field("div")) < TOL_ASM
    oc.update_grad_p()
    gf.update_gradient("p")
    assert rel(gf.get_field("gradP"), oc.field("gradP")) < TOL_ASM
    oc.update_grad_u()
    gf.update_gradient("U")
    assert rel(gf.get_field("gradU"), oc.field("gradU")) < TOL_ASM


def test_initialize_parity(oracle_mod):
    m, oc, gm, gf = make_pair(oracle_mod, n=6)
    oc.initialize()
    gf.initialize()
    for k in ["mDot", "div", "gradU", "gradP"]:
        assert rel(gf.get_field(k), oc.field(k)) < TOL_ASM, k


def test_simple_iterations_parity_fp64(oracle_mod):
    """Ten SIMPLE outer iterations on a skewed 8^3 cavity; both sides solve
    each linear system tightly, so the trajectories agree to round-off."""
    kw = dict(mom_rtol=1e-13, pc_rtol=1e-13, mom_maxit=500, pc_maxit=5000)
    m, oc, gm, gf = make_pair(oracle_mod, n=8, **kw)
    oc.initialize()
    gf.initialize()
    for it in range(10):
        so = oc.simple_iteration()
        sg = gf.simple_iterate(1)[0]
        assert abs(sg["continuity_rms"] - so["continuity_rms"]) <= 1e-9 * abs(so["continuity_rms"]) + 1e-18
    for k in ["U", "p", "mDot"]:
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k


def test_golden_fixture_gpu(oracle_mod):
    """GPU FP64 path against the committed oracle fixture."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "cavity4_perturbed.npz"))
    m = meshgen.cavity(4, perturb=0.2, seed=12345)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=12345)
    gm = rt.Mesh(m)
    gf = rt.Flow(gm, rt.default_settings(mom_rtol=1e-13, pc_rtol=1e-13))
    gf.set_field("U", U0)
    gf.initialize()
    rp, cols = gm.graph()
    np.testing.assert_array_equal(rp, g["row_ptr"])
    A, b = gf.assemble_momentum()
    assert rel(A, g["A_mom"]) < TOL_ASM and rel(b, g["b_mom"]) < TOL_ASM
    A, b = gf.assemble_pcorr()
    assert rel(A, g["A_pc"]) < TOL_ASM and rel(b, g["b_pc"]) < TOL_ASM
    gf2 = rt.Flow(gm, rt.default_settings(mom_rtol=1e-13, pc_rtol=1e-13))
    gf2.set_field("U", U0)
    gf2.initialize()
    gf2.simple_iterate(5)
    for k in ["U", "p", "mDot"]:
        assert rel(gf2.get_field(k), g[k + "_it5"]) < 1e-10, k


def test_mixed_precision_fields_close(oracle_mod):
    """Mixed FP32/FP64 form after 10 iterations stays within 1e-6 of the FP64
    oracle (north-star field tolerance)."""
    kw = dict(mom_rtol=1e-7, pc_rtol=1e-10, mom_maxit=500, pc_maxit=5000)
    m, oc, gm, gf = make_pair(oracle_mod, n=8, prec=rt.OA_PREC_MIXED, **kw)
    oc.initialize()
    gf.initialize()
    for _ in range(10):
        oc.simple_iteration()
    gf.simple_iterate(10)
    U_o = oc.field("U")
    assert np.abs(gf.get_field("U") - U_o).max() < 1e-6 * max(1.0, np.abs(U_o).max())


def test_deterministic_bitwise(oracle_mod):
    m, oc, gm, gf = make_pair(oracle_mod, n=6)
    random_state(m, oc, gf)
    A1, b1 = gf.assemble_momentum()
    A2, b2 = gf.assemble_momentum()
    np.testing.assert_array_equal(A1, A2)
    np.testing.assert_array_equal(b1, b2)


def test_solver_parity(oracle_mod):
    m, oc, gm, gf = make_pair(oracle_mod, n=7)
    random_state(m, oc, gf)
    A, b = oc.assemble_pcorr()
    gf.assemble_pcorr()
    x_o, _, _ = oc.bicgstab(1, A, b, rtol=1e-13, maxit=5000)
    x_g, it, res = gf.solve("pcorr", 1e-13, 5000)
    assert res < 1e-12
    assert rel(x_g, x_o) < 1e-10


def test_scaled_continuity_and_control_data(oracle_mod):
    """The continuity residual (RMS of the nodal mass imbalance / rho U_lid h^2)
    matches the oracle's over three SIMPLE iterations, and the ControlData
    records of the solves carry the reference's fields: the initial residual is
    the RMS of the rhs (x0 = 0), the scaled one is that over the flux scale,
    the final one is the solver's exit residual."""
    m, oc, gm, gf = make_pair(oracle_mod, n=6, mom_rtol=1e-13, pc_rtol=1e-13)
    oc.initialize()
    gf.initialize()
    u_ref, mass_scale, mom_scale = gf.scales()
    assert u_ref == 1.0
    assert mass_scale == pytest.approx(oc.mass_scale(), rel=1e-15)
    assert mom_scale == pytest.approx(oc.mass_scale(), rel=1e-15)  # U_lid = 1
    for _ in range(3):
        so = oc.simple_iteration()
        sg = gf.simple_iterate(1)[0]
        assert sg["continuity_rms"] == pytest.approx(so["continuity_rms"], rel=1e-6)
        assert sg["continuity_rms_raw"] == pytest.approx(so["continuity_raw"], rel=1e-6)
    pc, mom = sg["pc"], sg["mom"]
    assert pc["solver_initial_res"][0] == pytest.approx(sg["continuity_rms_raw"], rel=1e-14)
    assert pc["scaled_initial_res"][0] == pytest.approx(sg["continuity_rms"], rel=1e-14)
    assert pc["solver_final_res"][0] <= 1e-12 * pc["solver_initial_res"][0]
    assert pc["n_iterations"] == sg["pc_iters"] and pc["fallback"] in (0, 1)
    assert mom["n_iterations"] == sg["mom_iters"]
    assert gf.last_control("pcorr") == pc
    # momentum: initial residual per component = RMS of that component of b
    A, b = gf.assemble_momentum()
    gf.solve("momentum", 1e-10, 500)
    cd = gf.last_control("momentum")
    rms = np.sqrt(np.mean(b.reshape(-1, 3) ** 2, axis=0))
    np.testing.assert_allclose(cd["solver_initial_res"], rms, rtol=1e-13)
    np.testing.assert_allclose(cd["scaled_initial_res"], rms / mom_scale, rtol=1e-13)
    assert np.linalg.norm(cd["solver_final_res"]) <= 1e-10 * np.linalg.norm(rms) * 1.0001


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 1, 1), (3, 2, 1)])
def test_smallest_meshes(oracle_mod, shape):
    # every node a boundary node, rows with 1 to 4 elements: assembly and two
    # SIMPLE iterations against the oracle
    kw = dict(mom_rtol=1e-13, pc_rtol=1e-13, mom_maxit=500, pc_maxit=5000)
    m = meshgen.cavity(shape, perturb=0.0)
    U0 = np.zeros((m.nn, 3))
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(**kw))
    gf.set_field("U", U0)
    oc.initialize()
    gf.initialize()
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    assert rel(A_g, A_o) < TOL_ASM and rel(b_g, b_o) < TOL_ASM
    for _ in range(2):
        oc.simple_iteration()
    gf.simple_iterate(2)
    for k in ["U", "p"]:
        assert np.abs(gf.get_field(k) - oc.field(k)).max() <= 1e-10 * max(1.0, np.abs(oc.field(k)).max()), k
