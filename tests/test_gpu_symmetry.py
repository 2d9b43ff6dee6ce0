"""Symmetry planes (oa_flow_set_boundary_types) on the GPU against the oracle.

A symmetry face adds the full viscous stress of the element's velocities to
the momentum row of its nearest node
(navierStokesAssemblerElemBoundaryConditions.cpp:2082-2375), carries no mass
flow and no gradient contribution (nodeField.hpp:4764); after the assembly a
symmetry node's rhs loses its normal component (applySymmetryConditions_,
navierStokesAssembler.cpp:387-471) and its diagonal block gains 0.25 D n n^T
(assembleNormalRelaxation, :473-699). Bars: assembly within 1e-12 in FP64 and
1e-5 in the mixed form, fields within 1e-10 after SIMPLE iterations, the
whole-iteration graph bit-identical to the eager path."""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu

TYPES = [rt.OA_BTYPE_WALL, rt.OA_BTYPE_WALL, rt.OA_BTYPE_SYMMETRY, rt.OA_BTYPE_SYMMETRY]
TIGHT = dict(mom_rtol=1e-13, pc_rtol=1e-13, mom_maxit=500, pc_maxit=5000)


def rel(a, b):
    d = np.linalg.norm(np.asarray(a) - np.asarray(b))
    n = np.linalg.norm(np.asarray(b))
    return d / n if n > 0 else d


def pair(oracle_mod, m, types, prec=rt.OA_PREC_FP64, correct=False, seed=3, **kw):
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=seed)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    oc.set_boundary_types(types, correct_gradients=correct)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(precision=prec, **kw))
    gf.set_boundary_types(types, correct_gradients=correct)
    gf.set_field("U", U0)
    return oc, gf


def random_state(m, oc, gf, seed=5):
    rng = np.random.default_rng(seed)
    fields = {"p": rng.normal(0, 1, m.nn), "gradP": rng.normal(0, 1, 3 * m.nn),
              "gradU": rng.normal(0, 1, 9 * m.nn), "du": rng.uniform(0.1, 1.0, 3 * m.nn),
              "mDot": rng.normal(0, 0.01, 12 * m.ne), "div": rng.normal(0, 1e-3, m.nn)}
    for k, v in fields.items():
        oc.field(k)[:] = v
        gf.set_field(k, v)


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_symmetry_assembly_parity(oracle_mod, prec):
    m = meshgen.symmetry_box(6, perturb=0.2, seed=3)
    oc, gf = pair(oracle_mod, m, TYPES, prec)
    random_state(m, oc, gf)
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    tol = 1e-12 if prec == rt.OA_PREC_FP64 else 1e-5
    assert rel(A_g, A_o) < tol and rel(b_g, b_o) < tol
    assert rel(gf.get_field("du"), oc.field("du")) < tol
    # the symmetry rows: no rhs along the plane normal (y)
    y = m.coords[:, 1]
    sym = np.isclose(y, 0.0) | np.isclose(y, 1.0)
    assert np.abs(b_g.reshape(-1, 3)[sym, 1]).max() < 1e-12 * np.abs(b_g).max()
    # the plain wall assembly differs
    w = rt.Flow(rt.Mesh(m), rt.default_settings(precision=prec))
    for k in ("U", "p", "gradP", "gradU", "du", "mDot", "div"):
        w.set_field(k, gf.get_field(k))
    _, b_w = w.assemble_momentum()
    assert rel(b_w, b_o) > 1e-3


def test_symmetry_linear_field_known_answer():
    # every face a symmetry plane, a linear velocity field, uniform mu, no
    # pressure and no mass flow: every control volume is closed by the
    # symmetry stress, so the momentum residual vanishes at every node
    m = meshgen.symmetry_box(5, perturb=0.25, seed=7)
    G = np.random.default_rng(2).normal(size=(3, 3))
    gf = rt.Flow(rt.Mesh(m), rt.default_settings())
    gf.set_boundary_types([rt.OA_BTYPE_SYMMETRY] * 4)
    gf.set_field("U", (m.coords @ G.T).ravel())
    for k, n in (("p", m.nn), ("gradP", 3 * m.nn), ("mDot", 12 * m.ne), ("div", m.nn)):
        gf.set_field(k, np.zeros(n))
    _, b = gf.assemble_momentum()
    assert np.abs(b).max() < 1e-14


@pytest.mark.parametrize("correct", [False, True])
def test_symmetry_gradients(oracle_mod, correct):
    m = meshgen.symmetry_box(6, perturb=0.2, seed=4)
    kw = dict(u_shifted=0, u_grad_shifted=0, p_shifted=0, p_grad_shifted=0)
    oc, gf = pair(oracle_mod, m, TYPES, correct=correct, **kw)
    random_state(m, oc, gf)
    oc.update_grad_p()
    gf.update_gradient("p")
    oc.update_grad_u()
    gf.update_gradient("U")
    assert rel(gf.get_field("gradP"), oc.field("gradP")) < 1e-12
    assert rel(gf.get_field("gradU"), oc.field("gradU")) < 1e-12


@pytest.mark.parametrize("correct", [False, True])
def test_symmetry_simple_iterations(oracle_mod, correct):
    m = meshgen.symmetry_box(6, perturb=0.2, seed=9)
    oc, gf = pair(oracle_mod, m, TYPES, correct=correct, seed=9, **TIGHT)
    oc.initialize()
    gf.initialize()
    for _ in range(5):
        so = oc.simple_iteration()
        sg = gf.simple_iterate(1)[0]
        assert abs(sg["continuity_rms"] - so["continuity_rms"]) <= 1e-9 * abs(so["continuity_rms"]) + 1e-18
    for k in ("U", "p", "mDot", "gradP", "gradU"):
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k


def test_symmetry_on_a_general_hex_mesh(oracle_mod):
    # five-block star prism (16 lanes per row): the lid as a symmetry plane
    m = meshgen.star_prism(5, 5, 4, perturb=0.2, seed=5)
    oc, gf = pair(oracle_mod, m, [rt.OA_BTYPE_SYMMETRY, rt.OA_BTYPE_WALL], seed=5, **TIGHT)
    random_state(m, oc, gf)
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    assert rel(A_g, A_o) < 1e-12 and rel(b_g, b_o) < 1e-12


def test_symmetry_mixed_high_resolution_and_transient(oracle_mod):
    # the mixed form within 1e-6 of the FP64 oracle over SIMPLE iterations
    m = meshgen.symmetry_box(6, perturb=0.2, seed=11)
    kw = dict(mom_rtol=1e-7, pc_rtol=1e-10, mom_maxit=500, pc_maxit=5000)
    oc, gf = pair(oracle_mod, m, TYPES, rt.OA_PREC_MIXED, seed=11, **kw)
    oc.initialize()
    gf.initialize()
    for _ in range(4):
        oc.simple_iteration()
    gf.simple_iterate(4)
    U_o = oc.field("U")
    assert np.abs(gf.get_field("U") - U_o).max() < 1e-6 * max(1.0, np.abs(U_o).max())
    # high resolution in FP64
    oc, gf = pair(oracle_mod, m, TYPES, seed=11, hr=1, **TIGHT)
    oc.initialize()
    gf.initialize()
    for _ in range(3):
        oc.simple_iteration()
    gf.simple_iterate(3)
    for k in ("U", "p", "betaU"):
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k
    # transient BDF2: only wall-face nodes get the boundary rhs relaxation
    oc, gf = pair(oracle_mod, m, TYPES, seed=11, urf_u=1.0, urf_p=0.5, mom_rtol=1e-13, pc_rtol=1e-13)
    oc.initialize()
    gf.initialize()
    for dt in (0.1, 0.05):
        oc.advance_time(2, dt)
        gf.advance_time(rt.OA_TIME_BDF2, dt)
        A_o, b_o = oc.assemble_momentum()
        A_g, b_g = gf.assemble_momentum()
        assert rel(A_g, A_o) < 1e-12 and rel(b_g, b_o) < 1e-12
        for _ in range(2):
            oc.simple_iteration()
        gf.simple_iterate(2)
    for k in ("U", "p"):
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k


@pytest.mark.parametrize("precision", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_symmetry_iteration_graph_matches_eager(precision):
    m = meshgen.symmetry_box(10, perturb=0.2, seed=12)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=12)
    runs = []
    for graphs in (1, 2):
        f = rt.Flow(rt.Mesh(m), rt.default_settings(use_graphs=graphs, precision=precision))
        f.set_boundary_types(TYPES, correct_gradients=True)
        f.set_field("U", U0)
        f.initialize()
        st = f.simple_iterate(5)
        runs.append((f, st))
    (fe, se), (fg, sg) = runs
    for k in ("U", "p", "mDot", "gradU", "gradP"):
        np.testing.assert_array_equal(fg.get_field(k), fe.get_field(k), err_msg=k)
    for a, b in zip(se, sg):
        assert a["pc_iters"] == b["pc_iters"] and a["continuity_rms"] == b["continuity_rms"]


def test_boundary_type_errors():
    m = meshgen.symmetry_box(3)
    f = rt.Flow(rt.Mesh(m), rt.default_settings())
    for bad in ([0, 0, 1], [0, 0, 1, 2], [0, 0, -1, 1]):
        with pytest.raises(rt.OpenAccelError) as ei:
            f.set_boundary_types(bad)
        assert ei.value.status == 1
    # back to all walls: the plain wall assembly again
    f.set_field("U", meshgen.initial_velocity(m, sigma=0.1, seed=1))
    _, b0 = f.assemble_momentum()
    f.set_boundary_types(TYPES)
    _, b1 = f.assemble_momentum()
    f.set_boundary_types([0, 0, 0, 0])
    _, b2 = f.assemble_momentum()
    assert rel(b1, b0) > 1e-6
    np.testing.assert_array_equal(b2, b0)
