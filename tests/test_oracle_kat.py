"""CPU checks of the oracle: analytic known answers, agreement with the
reference's own compiled geometry templates (oracle/_ref), structural
properties of the assembled systems, and the committed golden fixtures."""
import ctypes as C
import os

import numpy as np
import pytest

from openaccel_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
UNIT = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)


def test_unit_cube_scs_areas(oracle_mod):
    a = oracle_mod.hex8_scs_areav(UNIT)
    # every SCS of a unit cube is a quarter of a unit face, pointing L -> R
    lr = [(0, 1), (1, 2), (2, 3), (0, 3), (4, 5), (5, 6), (6, 7), (4, 7), (0, 4), (1, 5), (2, 6), (3, 7)]
    for ip, (l, r) in enumerate(lr):
        d = UNIT[r] - UNIT[l]
        np.testing.assert_allclose(a[ip], 0.25 * d, atol=1e-15)


def test_scv_volumes_sum_to_element_volume(oracle_mod):
    rng = np.random.default_rng(1)
    for _ in range(20):
        A = np.eye(3) + rng.uniform(-0.2, 0.2, (3, 3))
        x = UNIT @ A.T + rng.uniform(-1, 1, 3)
        v = oracle_mod.hex8_scv_volumes(x)
        assert np.all(v > 0)
        np.testing.assert_allclose(v.sum(), abs(np.linalg.det(A)), rtol=1e-13)


def test_gradient_operator_exact_for_linear_fields(oracle_mod):
    rng = np.random.default_rng(2)
    x = UNIT + rng.uniform(-0.15, 0.15, UNIT.shape)
    c = np.array([0.3, -1.2, 2.5])
    f = x @ c
    for shifted in (True, False):
        g, err = oracle_mod.hex8_grad_op(x, shifted)
        assert err == 0
        np.testing.assert_allclose(np.einsum("ink,n->ik", g, f), np.tile(c, (12, 1)), rtol=1e-12, atol=1e-12)
        # partition of unity: gradients sum to zero
        np.testing.assert_allclose(g.sum(axis=1), 0.0, atol=1e-12)


def test_closed_element_surface(oracle_mod):
    # sum of outward SCS area vectors around each SCV plus its exposed faces is zero,
    # equivalently: SCS areas are antisymmetric per element; here check that the
    # 12 SCS areas of an affine element scale with the affine map
    rng = np.random.default_rng(3)
    A = np.eye(3) + rng.uniform(-0.3, 0.3, (3, 3))
    a0 = oracle_mod.hex8_scs_areav(UNIT)
    a1 = oracle_mod.hex8_scs_areav(UNIT @ A.T)
    cof = np.linalg.det(A) * np.linalg.inv(A).T
    np.testing.assert_allclose(a1, a0 @ cof.T, rtol=1e-12, atol=1e-14)


REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnalu_hex8_ref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference geometry library not built (needs the reference tree)")
def test_oracle_matches_reference_geometry_templates(oracle_mod):
    """Pin the restated master element against the reference's own
    subdivide_hex_8 / quad_area_by_triangulation / hex_volume_grandy."""
    L = C.CDLL(REF_LIB)
    rng = np.random.default_rng(4)
    for _ in range(200):
        x = UNIT + rng.uniform(-0.24, 0.24, UNIT.shape)
        a = np.zeros((12, 3))
        v = np.zeros(8)
        L.ref_hex8_scs_areav(x.ctypes.data_as(C.c_void_p), a.ctypes.data_as(C.c_void_p))
        L.ref_hex8_scv_volumes(x.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p))
        np.testing.assert_allclose(oracle_mod.hex8_scs_areav(x), a, rtol=0, atol=4e-16)
        np.testing.assert_allclose(oracle_mod.hex8_scv_volumes(x), v, rtol=0, atol=4e-16)


def test_dual_volume_and_graph(oracle_mod):
    m = meshgen.cavity(5, perturb=0.2, seed=7)
    c = oracle_mod.FlowCase(m)
    np.testing.assert_allclose(c.field("vol").sum(), 1.0, rtol=1e-13)
    rp, cols = c.graph()
    deg = np.diff(rp)
    # interior nodes: self + 6 edge neighbours; corners: self + 3
    assert deg.max() == 7 and deg.min() == 4
    for i in range(m.nn):
        row = cols[rp[i]:rp[i + 1]]
        assert np.all(np.diff(row) > 0) and i in row


@pytest.mark.parametrize("blocks", [3, 5])
def test_star_prism_volume_graph_and_row_sums(oracle_mod, blocks):
    """A hex mesh that is not one block (3 or 5 elements around the centre
    line's edges): dual volumes add up to the prism (polygon area x height),
    the centre-line nodes have blocks + 2 stencil neighbours (+ self), and
    the pressure-correction rows still sum to zero."""
    m = meshgen.star_prism(blocks, 4, 3, radius=1.0, height=0.5)
    c = oracle_mod.FlowCase(m, U0=np.random.default_rng(1).normal(0, 0.1, (m.nn, 3)))
    k = 2 * blocks
    area = 0.5 * k * np.sin(2 * np.pi / k)
    np.testing.assert_allclose(c.field("vol").sum(), 0.5 * area, rtol=1e-13)
    rp, cols = c.graph()
    centre = np.where(np.linalg.norm(m.coords[:, :2], axis=1) < 1e-12)[0]
    interior_centre = centre[(m.coords[centre, 2] > 0) & (m.coords[centre, 2] < 0.5)]
    assert np.all(np.diff(rp)[interior_centre] == blocks + 3)
    c.initialize()
    c.field("du")[:] = np.random.default_rng(2).uniform(0.5, 1.5, 3 * m.nn)
    A, b = c.assemble_pcorr()
    rows = np.add.reduceat(A, rp[:-1])
    rows[0] = 0.0
    assert np.abs(rows).max() < 1e-13 * np.abs(A).max()


def test_pcorr_row_sums_vanish(oracle_mod):
    """Rhie-Chow Laplacian: sum_n dN_n/dx = 0, so every row of the
    pressure-correction matrix sums to zero (lumping keeps row sums)."""
    m = meshgen.cavity(4, perturb=0.2, seed=3)
    rng = np.random.default_rng(5)
    c = oracle_mod.FlowCase(m, U0=rng.normal(0, 0.1, (m.nn, 3)))
    c.initialize()
    c.field("du")[:] = rng.uniform(0.5, 1.5, 3 * m.nn)
    A, b = c.assemble_pcorr()
    rp, _ = c.graph()
    rows = np.add.reduceat(A, rp[:-1])
    scale = np.abs(A).max()
    rows[0] = 0.0  # reference-pressure row keeps only its diagonal
    assert np.abs(rows).max() < 1e-13 * scale


def test_uniform_velocity_zero_divergence(oracle_mod):
    m = meshgen.cavity(4, perturb=0.2, seed=9)
    U = np.tile([0.3, -0.1, 0.2], (m.nn, 1))
    c = oracle_mod.FlowCase(m, U0=U)
    c.initialize()
    div = c.field("div").reshape(-1)
    # interior nodes: closed control surface, constant flux field -> zero net mass flow
    idx = np.arange(m.nn)
    i, j, k = idx % 5, (idx // 5) % 5, idx // 25
    inner = (i > 0) & (i < 4) & (j > 0) & (j < 4) & (k > 0) & (k < 4)
    assert np.abs(div[inner]).max() < 1e-15


def test_gradient_converges_to_exact_on_linear_field(oracle_mod):
    m = meshgen.cavity(4, perturb=0.0)
    coef = np.array([0.7, -0.4, 1.3])
    c = oracle_mod.FlowCase(m)
    c.field("p")[:] = m.coords @ coef
    for _ in range(60):
        c.update_grad_p()
    g = c.field("gradP").reshape(-1, 3)
    idx = np.arange(m.nn)
    i, j, k = idx % 5, (idx // 5) % 5, idx // 25
    inner = (i > 0) & (i < 4) & (j > 0) & (j < 4) & (k > 0) & (k < 4)
    np.testing.assert_allclose(g[inner], np.tile(coef, (inner.sum(), 1)), rtol=1e-12)


GOLDEN = os.path.join(ROOT, "tests", "golden", "cavity4_perturbed.npz")


def test_golden_fixture_regenerates(oracle_mod):
    """The committed fixture (tests/golden/make_golden.py) is reproduced by
    the current oracle bit for bit."""
    from tests.golden.make_golden import generate

    g = np.load(GOLDEN)
    cur = generate(oracle_mod)
    for k in g.files:
        np.testing.assert_array_equal(cur[k], g[k], err_msg=k)


def test_continuity_scale_is_rho_ulid_h2(oracle_mod):
    """The continuity residual is the RMS of the nodal mass imbalance divided by
    rho U_lid h^2 (h = mean element edge length): exactly (1/n)^2 on the unit
    cavity with a unit lid, and the numpy mean edge length on a skewed one."""
    from openaccel_b200 import meshgen

    m = meshgen.cavity(4)
    c = oracle_mod.FlowCase(m, oracle_mod.default_settings(rho=1.0))
    assert c.mass_scale() == pytest.approx(1.0 / 16.0, rel=1e-15)
    m = meshgen.cavity(5, perturb=0.2, seed=9, lid_velocity=(0.0, 2.0, 0.0))
    c = oracle_mod.FlowCase(m, oracle_mod.default_settings(rho=1.5))
    lr = [(0, 1), (1, 2), (2, 3), (0, 3), (4, 5), (5, 6), (6, 7), (4, 7), (0, 4), (1, 5), (2, 6), (3, 7)]
    x = m.coords[m.conn]
    h = np.mean([np.linalg.norm(x[:, a] - x[:, b], axis=1) for a, b in lr])
    assert c.mass_scale() == pytest.approx(1.5 * 2.0 * h * h, rel=1e-12)
    c.initialize()
    st = c.simple_iteration()
    assert st["continuity_rms"] == pytest.approx(st["continuity_raw"] / c.mass_scale(), rel=1e-15)


REF_ASM_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_assembler.so")


@pytest.mark.skipif(not os.path.exists(REF_ASM_LIB),
                    reason="reference assembler library not built (needs the reference tree)")
@pytest.mark.parametrize("bs", [1, 3])
def test_oracle_scatter_matches_reference_apply_coeff(oracle_mod, bs):
    """Pin the oracle's scatter against the reference's own
    assembler<N>::applyCoeff_ (src/assemble/assembler.h:311-453, compiled from
    the reference tree): random element matrices of hex8 elements, in random
    node orders, added into the reduced-stencil block-CSR system, where the
    face- and body-diagonal columns the stencil lacks are lumped into the
    diagonal block. Bitwise equal."""
    L = C.CDLL(REF_ASM_LIB)
    m = meshgen.cavity(4, perturb=0.2, seed=3)
    c = oracle_mod.FlowCase(m, oracle_mod.default_settings())
    rp, cols = c.graph()
    diag = np.array([np.searchsorted(cols[rp[i]:rp[i + 1]], i) for i in range(m.nn)], dtype=np.int32)
    rng = np.random.default_rng(11 + bs)
    A_o = np.zeros(bs * bs * cols.size)
    b_o = np.zeros(bs * m.nn)
    A_r, b_r = A_o.copy(), b_o.copy()
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    for e in rng.permutation(m.ne):
        nodes = np.ascontiguousarray(rng.permutation(m.conn[e]), np.int32)
        n = nodes.size
        lhs = rng.normal(size=(n * bs) ** 2)
        rhs = rng.normal(size=n * bs)
        c.apply_coeff(bs, A_o, b_o, nodes, rhs, lhs)
        L.ref_apply_coeff(bs, m.nn, ptr(rp), ptr(cols), ptr(diag), ptr(A_r), ptr(b_r), ptr(nodes), n, ptr(rhs),
                          ptr(lhs), 1)
    np.testing.assert_array_equal(A_o, A_r)
    np.testing.assert_array_equal(b_o, b_r)
    assert np.abs(A_o).sum() > 0


def test_blending_factor_known_answers(oracle_mod):
    """High-resolution limiter (nodeField::updateBlendingFactorField) on a
    uniform 4^3 mesh with U = (x, 0, 0): along x the projected increment to an
    SCS ip is h/2 against an extremum h away, ratio 2, which the smooth map
    sends to 1 = beta_max; components with zero gradient are not limited; on
    the x = 0 and x = 1 faces one extremum is the node's own value, so
    beta_x = 0. After the first update the relaxation 0.75 * 0 + 0.25 * beta
    leaves 0.25 inside and 0 on those faces; a constant field stays at
    0.25 * beta_max."""
    m = meshgen.cavity(4)
    c = oracle_mod.FlowCase(m, oracle_mod.default_settings(hr=1, beta_max=1.0))
    x = m.coords
    U = np.zeros((m.nn, 3))
    U[:, 0] = x[:, 0]
    c.field("U")[:] = U.ravel()
    for _ in range(60):  # the gradient under-relaxation (0.5625) converges to the exact gradient
        c.update_grad_u()
    c.update_blending_u()
    beta = c.field("betaU").reshape(-1, 3)
    xb = (np.isclose(x[:, 0], 0.0)) | (np.isclose(x[:, 0], 1.0))
    np.testing.assert_allclose(beta[~xb, 0], 0.25, atol=1e-12)
    np.testing.assert_allclose(beta[xb, 0], 0.0, atol=1e-12)
    np.testing.assert_allclose(beta[:, 1:], 0.25, atol=1e-12)
    c2 = oracle_mod.FlowCase(m, oracle_mod.default_settings(hr=1, beta_max=0.8))
    c2.field("U")[:] = 1.0
    c2.update_grad_u()
    c2.update_blending_u()
    np.testing.assert_allclose(c2.field("betaU"), 0.2, atol=1e-15)


def test_transport_assembly_known_answers(oracle_mod):
    """k / omega transport restatement: a constant field gives a zero rhs and
    zero row sums before the node terms; the node terms then sit on the
    diagonal and the rhs; relaxation divides the diagonal only."""
    m = meshgen.cavity(4, perturb=0.2, seed=6)
    c = oracle_mod.FlowCase(m, U0=meshgen.initial_velocity(m, sigma=0.1, seed=6))
    c.initialize()
    rng = np.random.default_rng(3)
    gam = rng.uniform(0.01, 0.02, m.nn)
    zero = np.zeros(m.nn)
    A, b = c.assemble_transport(np.full(m.nn, 2.5), gam, zero, zero, 1.0)
    rp, cols = c.graph()
    scale = np.abs(A).max()
    # advection of a constant: the rhs is -phi * (net outflow) = -phi * div
    np.testing.assert_allclose(b, -2.5 * c.field("div"), atol=1e-14 * scale)
    diag = np.array([A[rp[i] + np.searchsorted(cols[rp[i]:rp[i + 1]], i)] for i in range(m.nn)])
    sd, sr = rng.uniform(0, 1e-3, m.nn), rng.normal(0, 1e-3, m.nn)
    A2, b2 = c.assemble_transport(np.full(m.nn, 2.5), gam, sd, sr, 0.5)
    diag2 = np.array([A2[rp[i] + np.searchsorted(cols[rp[i]:rp[i + 1]], i)] for i in range(m.nn)])
    np.testing.assert_allclose(diag2, (diag + sd) / 0.5, rtol=1e-13)
    np.testing.assert_allclose(b2, b + sr, atol=1e-14 * scale)


def _linear_state(oc, m, G):
    oc.field("U")[:] = (m.coords @ G.T).ravel()
    for k in ("p", "gradP", "mDot", "div"):
        oc.field(k)[:] = 0.0


def test_symmetry_planes_close_every_control_volume(oracle_mod):
    # a linear velocity field with uniform mu, no pressure and no mass flow: the
    # interior viscous fluxes of a control volume cancel except where its surface
    # meets the boundary; the symmetry term (the full stress at the face ip)
    # closes it, so with every face a symmetry plane the momentum residual
    # vanishes at every node, while a no-slip wall leaves its zero-normal-stress
    # projection behind
    m = meshgen.symmetry_box(4, perturb=0.25, seed=3)
    G = np.random.default_rng(1).normal(size=(3, 3))
    res = {}
    for name, types in (("sym", [1, 1, 1, 1]), ("mixed", [0, 0, 1, 1]), ("wall", [0, 0, 0, 0])):
        oc = oracle_mod.FlowCase(m, oracle_mod.default_settings())
        oc.set_boundary_types(types)
        _linear_state(oc, m, G)
        _, b = oc.assemble_momentum()
        res[name] = np.abs(b).max()
    assert res["sym"] < 1e-15
    assert res["mixed"] > 1e-4 and res["wall"] > 1e-4


def test_symmetry_area_and_side_velocity(oracle_mod):
    m = meshgen.symmetry_box((4, 3, 5), perturb=0.2, seed=4, lid_velocity=(1.0, 0.0, 0.0))
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings())
    oc.set_boundary_types([0, 0, 1, 1])
    area = oc.field("symArea").reshape(-1, 3)
    y = m.coords[:, 1]
    on0, on1 = np.isclose(y, 0.0), np.isclose(y, 1.0)
    # the planes are flat: every assembled area is along -y (y = 0) or +y (y = 1),
    # and each plane's areas add up to the plane's area (1)
    assert np.abs(area[:, [0, 2]]).max() < 1e-15
    assert abs(area[on0, 1].sum() + 1.0) < 1e-14 and abs(area[on1, 1].sum() - 1.0) < 1e-14
    assert np.all(area[~(on0 | on1)] == 0.0)
    # the lid's velocity reaches the lid nodes on the symmetry planes (the
    # symmetry boundaries no longer overwrite them), the walls win at their edges
    side = oc.field("sideU").reshape(-1, 3)
    x, z = m.coords[:, 0], m.coords[:, 2]
    lid_sym = np.isclose(z, 1.0) & (on0 | on1) & ~np.isclose(x, 0.0) & ~np.isclose(x, 1.0)
    assert lid_sym.any() and np.all(side[lid_sym, 0] == 1.0)
    with pytest.raises(ValueError):
        oc.set_boundary_types([0, 0, 2, 1])
    with pytest.raises(ValueError):
        oc.set_boundary_types([0, 1])


def test_symmetry_gradient_correction(oracle_mod):
    # with correctGradients_ the pressure gradient at a symmetry node has no
    # normal (y) part and the velocity gradient keeps only its in-plane
    # components and the normal-normal one
    m = meshgen.symmetry_box(4, perturb=0.2, seed=6)
    rng = np.random.default_rng(6)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings())
    oc.set_boundary_types([0, 0, 1, 1], correct_gradients=True)
    oc.field("p")[:] = rng.normal(size=m.nn)
    oc.field("U")[:] = rng.normal(size=3 * m.nn)
    oc.update_grad_p()
    oc.update_grad_u()
    y = m.coords[:, 1]
    sym = np.isclose(y, 0.0) | np.isclose(y, 1.0)
    gp = oc.field("gradP").reshape(-1, 3)
    gu = oc.field("gradU").reshape(-1, 3, 3)
    assert np.abs(gp[sym, 1]).max() < 1e-13 and np.abs(gp[~sym, 1]).max() > 1e-3
    # G_iy = 0 for i != y and G_yj = 0 for j != y
    assert np.abs(gu[sym][:, [0, 2], 1]).max() < 1e-13 and np.abs(gu[sym][:, 1, [0, 2]]).max() < 1e-13
    assert np.abs(gu[sym][:, 1, 1]).max() > 1e-3
