"""CPU known-answer checks of the SST node-level oracle."""
import numpy as np


def _base(nn=4):
    z = np.zeros(nn)
    return dict(k=np.full(nn, 1e-2), omega=np.full(nn, 1e2), k_prev=np.full(nn, 1e-2), rho=np.ones(nn),
                mu=np.full(nn, 1e-5), ymin=np.full(nn, 0.1), gradU=np.zeros(9 * nn), gradK=np.zeros(3 * nn),
                gradW=np.zeros(3 * nn), div=z.copy(), vol=np.full(nn, 2.0), mut_old=z.copy(), pk_wall=None,
                wall_node=np.zeros(nn, np.int32))


def test_quiescent_flow(oracle_mod):
    """No shear: mu_t = rho k / omega (a1 omega dominates), P_k = 0, the k and
    omega rhs are pure destruction."""
    c = oracle_mod.sst_constants()
    f = _base()
    o = oracle_mod.sst_nodes(f, dt=0.5)
    np.testing.assert_allclose(o["mut"], 1e-2 / 1e2, rtol=1e-12)
    assert np.all(o["Pk"] == 0.0)
    np.testing.assert_allclose(o["k_rhs"], -c.beta_star * 1e2 * 1e-2 * 2.0, rtol=1e-14)
    np.testing.assert_allclose(o["k_diag"], 2.0 / 0.5 + c.beta_star * 1e2 * 2.0, rtol=1e-14)
    beta = o["F1"] * c.beta1 + (1 - o["F1"]) * c.beta2
    np.testing.assert_allclose(o["w_rhs"], -beta * 1e4 * 2.0, rtol=1e-14)


def test_f1_near_and_far_from_walls(oracle_mod):
    f = _base(2)
    f["ymin"] = np.array([1e-5, 10.0])
    o = oracle_mod.sst_nodes(f)
    assert o["F1"][0] > 0.999999 and o["F1"][1] < 1e-6


def test_production_limiter_and_wall_nodes(oracle_mod):
    c = oracle_mod.sst_constants()
    f = _base(3)
    g = np.zeros((3, 9))
    g[:, 1] = 1e3  # du/dy: strong shear
    f["gradU"] = g.ravel()
    f["wall_node"] = np.array([0, 1, 1], np.int32)
    f["pk_wall"] = np.array([0.0, 0.25, 0.5])
    o = oracle_mod.sst_nodes(f)
    # interior: P_k = mu_t * S^2 with S^2 = (du/dy)^2; the k source is limited to 10 D_k
    np.testing.assert_allclose(o["Pk"][0], o["mut"][0] * 1e6, rtol=1e-12)
    Dk = c.beta_star * 1e2 * 1e-2
    np.testing.assert_allclose(o["k_rhs"][0], (c.prod_limit * Dk - Dk) * 2.0, rtol=1e-12)
    np.testing.assert_array_equal(o["Pk"][1:], [0.25, 0.5])


def test_negative_divergence_goes_to_the_diagonal(oracle_mod):
    f = _base(2)
    f["div"] = np.array([-0.5, 0.5])
    o = oracle_mod.sst_nodes(f)
    f0 = _base(2)
    o0 = oracle_mod.sst_nodes(f0)
    np.testing.assert_allclose(o["k_diag"] - o0["k_diag"], [0.5, 0.0], atol=1e-15)
    np.testing.assert_allclose(o["k_rhs"] - o0["k_rhs"], [-0.5 * 1e-2, 0.5 * 1e-2], rtol=1e-12)


def test_sst_diffusivities_known_answers(oracle_mod):
    # F1 = 1 takes the inner constants, F1 = 0 the outer ones, mu_eff = mu + mu_t
    c = oracle_mod.sst_constants()
    mu = np.array([1e-3, 1e-3, 2e-3])
    mut = np.array([0.5, 0.5, 0.0])
    F1 = np.array([1.0, 0.0, 0.3])
    mu_eff, gk, gw = oracle_mod.sst_diffusivities(mu, mut, F1, c)
    np.testing.assert_allclose(mu_eff, mu + mut, rtol=0, atol=0)
    np.testing.assert_allclose(gk[:2], [1e-3 + 0.5 * c.sigma_k1, 1e-3 + 0.5 * c.sigma_k2], rtol=1e-15)
    np.testing.assert_allclose(gw[:2], [1e-3 + 0.5 * c.sigma_w1, 1e-3 + 0.5 * c.sigma_w2], rtol=1e-15)
    assert gk[2] == mu[2] and gw[2] == mu[2]
