"""High-resolution advection on the GPU against the oracle: the velocity
extrema and blending factor (nodeField::updateMinMaxFields /
updateBlendingFactorField), the momentum assembly with the blended deferred
correction (navierStokesAssemblerElemTerms.cpp:287-330), and SIMPLE
iterations with the scheme switched on.

Bars: extrema exact, blending factor within 1e-12 (the limiter divides by a
projected increment, so the summation order of x_ip shows at that level),
assembled systems within 1e-12 in FP64 and 1e-5 in the mixed form's FP32 flux
arithmetic, fields within 1e-10 after five tight-solved SIMPLE iterations."""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


def rel(a, b):
    d = np.linalg.norm(np.asarray(a) - np.asarray(b))
    n = np.linalg.norm(np.asarray(b))
    return d / n if n > 0 else d


def pair(oracle_mod, n=7, prec=rt.OA_PREC_FP64, seed=11, **kw):
    m = meshgen.cavity(n, perturb=0.2, seed=seed)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=seed)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(hr=1, **kw), U0=U0)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(hr=1, precision=prec, **kw))
    gf.set_field("U", U0)
    return m, oc, gf


@pytest.mark.parametrize("ushift", [1, 0])
def test_blending_factor_parity(oracle_mod, ushift):
    m, oc, gf = pair(oracle_mod, u_shifted=ushift, u_grad_shifted=ushift)
    oc.initialize()
    gf.initialize()
    np.testing.assert_array_equal(gf.get_field("minU"), oc.field("minU"))
    np.testing.assert_array_equal(gf.get_field("maxU"), oc.field("maxU"))
    assert rel(gf.get_field("gradU"), oc.field("gradU")) < 1e-13
    b_g, b_o = gf.get_field("betaU"), oc.field("betaU")
    assert np.abs(b_g - b_o).max() < 1e-12
    assert b_o.max() > 0.05  # the limiter is active, not trivially beta_max or 0


@pytest.mark.parametrize("prec,tol", [(rt.OA_PREC_FP64, 1e-12), (rt.OA_PREC_MIXED, 1e-5)])
@pytest.mark.parametrize("shift", [(1, 1), (0, 0)])
def test_momentum_assembly_with_deferred_correction(oracle_mod, prec, tol, shift):
    us, gs = shift
    m, oc, gf = pair(oracle_mod, prec=prec, u_shifted=us, u_grad_shifted=gs)
    rng = np.random.default_rng(5)
    fields = {"gradU": rng.normal(0, 1, 9 * m.nn), "gradP": rng.normal(0, 1, 3 * m.nn),
              "mDot": rng.normal(0, 0.01, 12 * m.ne), "div": rng.normal(0, 1e-3, m.nn),
              "betaU": rng.uniform(0, 1, 3 * m.nn)}
    for k, v in fields.items():
        oc.field(k)[:] = v
        gf.set_field(k, v)
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    assert rel(A_g, A_o) < tol
    assert rel(b_g, b_o) < tol
    # the correction changes the rhs: switching beta off moves b well beyond tol
    gf.set_field("betaU", np.zeros(3 * m.nn))
    _, b0 = gf.assemble_momentum()
    assert rel(b0, b_o) > 100 * tol


def test_simple_iterations_high_resolution(oracle_mod):
    m, oc, gf = pair(oracle_mod, n=6, mom_rtol=1e-13, pc_rtol=1e-13)
    oc.initialize()
    gf.initialize()
    for _ in range(5):
        oc.simple_iteration()
    gf.simple_iterate(5)
    for k in ("U", "p", "mDot", "betaU"):
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k
