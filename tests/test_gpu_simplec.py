"""Pressure-velocity coupling variants on the GPU against the oracle:
SIMPLEC (consistent_: D~ = V / (a_ii + sum of the row's off-diagonal
coefficients) on the pressure-correction lhs and in the velocity correction,
D on the Rhie-Chow rhs) and the fractional-step coefficient D = dt / rho
(navierStokesAssembler::computeDUCoefficients,
navierStokesAssembler.cpp:84-232; pressureCorrectionAssemblerElemTerms.cpp:126-134;
segregatedFlowEquations.cpp:134-278).

Bars: coefficients and assembled systems within 1e-12 (FP64), fields within
1e-10 after five tight-solved SIMPLE iterations."""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


def rel(a, b):
    d = np.linalg.norm(np.asarray(a) - np.asarray(b))
    n = np.linalg.norm(np.asarray(b))
    return d / n if n > 0 else d


def pair(oracle_mod, n=6, **kw):
    m = meshgen.cavity(n, perturb=0.2, seed=17)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=17)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(**kw))
    gf.set_field("U", U0)
    return m, oc, gf


def test_simplec_coefficients_and_pressure_correction(oracle_mod):
    m, oc, gf = pair(oracle_mod, du_mode=1, urf_p=0.5)
    oc.initialize()
    gf.initialize()
    oc.assemble_momentum()
    gf.assemble_momentum()
    assert rel(gf.get_field("du"), oc.field("du")) < 1e-12
    dT = oc.field("duTilde")
    assert rel(gf.get_field("duTilde"), dT) < 1e-12
    assert rel(dT, oc.field("du")) > 1e-3  # the off-diagonal sum changes it
    A_o, b_o = oc.assemble_pcorr()
    A_g, b_g = gf.assemble_pcorr()
    assert rel(A_g, A_o) < 1e-12
    assert rel(b_g, b_o) < 1e-12


@pytest.mark.parametrize("mode", [1, 2])
def test_simple_iterations_simplec_and_fractional_step(oracle_mod, mode):
    m, oc, gf = pair(oracle_mod, du_mode=mode, urf_p=0.5, mom_rtol=1e-13, pc_rtol=1e-13)
    oc.initialize()
    gf.initialize()
    for _ in range(5):
        oc.simple_iteration()
    gf.simple_iterate(5)
    for k in ("U", "p", "mDot", "du"):
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k
    if mode == 2:
        np.testing.assert_allclose(gf.get_field("du"), 1.0, rtol=1e-15)  # dt / rho


def test_simplec_mixed_form_close_to_fp64(oracle_mod):
    """The mixed form with SIMPLEC within 1e-6 of the FP64 oracle (largest
    difference over the largest value, the north star's field bar), with the
    solver tolerances of the mixed-form parity test."""
    kw = dict(du_mode=1, urf_p=0.5, mom_rtol=1e-7, pc_rtol=1e-10, mom_maxit=500, pc_maxit=5000)
    m = meshgen.cavity(6, perturb=0.2, seed=17)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=17)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(precision=rt.OA_PREC_MIXED, **kw))
    gf.set_field("U", U0)
    oc.initialize()
    gf.initialize()
    for _ in range(5):
        oc.simple_iteration()
    gf.simple_iterate(5)
    for k in ("U", "p"):
        ref = oc.field(k)
        assert np.abs(gf.get_field(k) - ref).max() < 1e-6 * np.abs(ref).max(), k
