"""CPU checks of the tet4 oracle (master element and the scalar-diffusion
path): analytic known answers, structural properties of the assembled system,
the committed golden fixture, and why the solve is BiCGStab rather than CG."""
import os

import numpy as np
import pytest

from openaccel_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_TET = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
LR = [(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]
SIDE = [(0, 1, 3), (1, 2, 3), (0, 3, 2), (0, 2, 1)]


def _random_tet(rng):
    A = np.eye(3) + rng.uniform(-0.3, 0.3, (3, 3))
    if np.linalg.det(A) < 0:
        A[:, 0] *= -1
    return REF_TET @ A.T + rng.uniform(-1, 1, 3), A


def test_scv_volumes_sum_to_tet_volume(oracle_mod):
    rng = np.random.default_rng(11)
    for _ in range(20):
        x, A = _random_tet(rng)
        v = oracle_mod.tet4_scv_volumes(x)
        assert np.all(v > 0)
        np.testing.assert_allclose(v.sum(), np.linalg.det(A) / 6.0, rtol=1e-13)
    # regular reference tet: the four SCVs are equal
    v = oracle_mod.tet4_scv_volumes(np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], float))
    np.testing.assert_allclose(v, v.mean(), rtol=1e-13)


def test_gradient_exact_for_linear_fields(oracle_mod):
    rng = np.random.default_rng(12)
    for _ in range(10):
        x, _ = _random_tet(rng)
        c = rng.normal(size=3)
        g, err = oracle_mod.tet4_grad_op(x)
        assert err == 0
        np.testing.assert_allclose(g.T @ (x @ c), c, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(g.sum(axis=0), 0.0, atol=1e-12)
    # an inverted tet trips the determinant check
    _, err = oracle_mod.tet4_grad_op(REF_TET[[0, 2, 1, 3]])
    assert err == 1


def test_control_volumes_are_closed(oracle_mod):
    """Around every node, the outward SCS areas plus the node's share of the
    element's boundary faces sum to zero."""
    rng = np.random.default_rng(13)
    for _ in range(10):
        x, _ = _random_tet(rng)
        a = oracle_mod.tet4_scs_areav(x)
        closure = np.zeros((4, 3))
        for ip, (l, r) in enumerate(LR):
            closure[l] += a[ip]
            closure[r] -= a[ip]
        for f in range(4):
            fa = oracle_mod.tri3_face_areav(x[list(SIDE[f])])
            for k, n in enumerate(SIDE[f]):
                closure[n] += fa[k]
        np.testing.assert_allclose(closure, 0.0, atol=1e-14)


def test_face_ordinals_point_outward():
    m, _, _, _ = meshgen.conduction(3)
    x = m.coords[m.conn]
    for f, o in zip(m.face_elem, m.face_ord):
        p = x[f][list(meshgen.TET_SIDE_NODES[o])]
        nrm = np.cross(p[1] - p[0], p[2] - p[0])
        opp = x[f][[n for n in range(4) if n not in meshgen.TET_SIDE_NODES[o]][0]]
        assert np.dot(nrm, p[0] - opp) > 0


def test_kuhn_mesh_sizes():
    m, g, s, ge = meshgen.conduction(5)
    assert m.nn == 6 ** 3 and m.ne == 6 * 5 ** 3 and m.nf == 6 * 2 * 5 ** 2
    x = m.coords[m.conn]
    vol = np.einsum("ij,ij->i", x[:, 1] - x[:, 0], np.cross(x[:, 2] - x[:, 0], x[:, 3] - x[:, 0])) / 6
    assert np.all(vol > 0)
    np.testing.assert_allclose(vol.sum(), 1.0, rtol=1e-13)
    assert g.shape == (m.nn,) and np.all(g > 0) and np.all((s >= 0) & (s < 1))


def test_graph_and_dual_volume(oracle_mod):
    m, g, s, _ = meshgen.conduction(4, perturb=0.2)
    c = oracle_mod.DiffCase(m, g, s)
    rp, cols = c.graph()
    # interior rows of the Kuhn split: self + 14 edge neighbours
    n = 4
    i = np.arange(m.nn)
    ii, jj, kk = i % (n + 1), (i // (n + 1)) % (n + 1), i // (n + 1) ** 2
    interior = (ii > 0) & (ii < n) & (jj > 0) & (jj < n) & (kk > 0) & (kk < n)
    assert np.all(np.diff(rp)[interior] == 15)
    np.testing.assert_allclose(c.field("vol").sum(), 1.0, rtol=1e-13)


def test_linear_field_is_a_discrete_solution(oracle_mod):
    """With constant Gamma and no source, T = x satisfies the discrete system
    (fixed values 0 / 1 on x = 0 / 1, zero flux elsewhere): the defect rhs vanishes."""
    m, _, _, _ = meshgen.conduction(5, perturb=0.25, seed=7)
    c = oracle_mod.DiffCase(m, np.full(m.nn, 2.5), np.zeros(m.nn))
    c.field("phi")[:] = m.coords[:, 0]
    A, b = c.assemble()
    assert np.abs(b).max() < 1e-13 * np.abs(A).max()


def test_interior_rows_conserve(oracle_mod):
    """Interior rows of the diffusion operator sum to zero (a constant field
    carries no flux); fixed-value rows do not (they carry the boundary flux)."""
    m, g, s, _ = meshgen.conduction(4, perturb=0.2)
    c = oracle_mod.DiffCase(m, g, s)
    A, _ = c.assemble()
    rp, _ = c.graph()
    rows = np.add.reduceat(A, rp[:-1])
    wall = c.field("wallNode") > 0
    assert np.abs(rows[~wall]).max() < 1e-13 * np.abs(A).max()
    assert np.abs(rows[wall]).max() > 1e-3 * np.abs(A).max()


def test_bicgstab_converges_where_cg_does_not(oracle_mod):
    """The assembled operator is not symmetric (Gamma differs between the SCS
    ips of an element; fixed-value rows carry only the boundary flux), so CG
    is not applicable: it fails to converge, BiCGStab reaches 1e-10."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla

    m, g, s, _ = meshgen.conduction(6, perturb=0.2)
    c = oracle_mod.DiffCase(m, g, s)
    A, b = c.assemble()
    rp, cols = c.graph()
    M = sp.csr_matrix((A, cols, rp), shape=(m.nn, m.nn))
    assert abs(M - M.T).max() > 1e-3 * abs(M).max()
    xd = sla.spsolve(M.tocsc(), b)
    _, it_cg, res_cg = c.cg(A, b, rtol=1e-10, maxit=2000)
    assert res_cg > 1e-6
    x, it, res = c.bicgstab(A, b, rtol=1e-12, maxit=2000)
    assert res <= 1e-12
    np.testing.assert_allclose(x, xd, rtol=0, atol=1e-10 * np.abs(xd).max())


def test_steps_converge_to_steady_state(oracle_mod):
    """Repeated steps drive the defect to zero (the wall rhs relaxation leaves
    a quarter of the wall defect per step). The fixed value enters only
    through the boundary flux, so wall nodes next to T = 0 settle slightly
    below 0; with the reference's lower clip at 0 those nodes stay at 0."""
    m, g, s, _ = meshgen.conduction(4, perturb=0.2)
    c = oracle_mod.DiffCase(m, g, s, oracle_mod.default_diff_settings(rtol=1e-13, lower_clip=-1e300))
    for _ in range(60):
        c.step()
    A, b = c.assemble()
    assert np.abs(b).max() < 1e-12 * np.abs(A).max()
    phi = c.field("phi")
    assert phi.min() < 0.0 and phi.max() > 1.0  # the source heats the interior above T = 1
    c2 = oracle_mod.DiffCase(m, g, s, oracle_mod.default_diff_settings(rtol=1e-13))
    for _ in range(10):
        c2.step()
    assert c2.field("phi").min() >= 0.0


def test_conduction_golden_fixture_regenerates(oracle_mod):
    from tests.golden import make_golden

    ref = np.load(os.path.join(ROOT, "tests", "golden", "conduction4_perturbed.npz"))
    new = make_golden.generate_conduction(oracle_mod)
    for k in ref.files:
        np.testing.assert_allclose(new[k], ref[k], rtol=1e-13, atol=1e-15, err_msg=k)
