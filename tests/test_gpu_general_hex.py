"""Hex meshes that are not one consistently oriented block.

meshgen.star_prism splits a polygon into 3 or 5 quadrilateral blocks that
meet at its centre and extrudes them: along the centre line 3 or 5 elements
share every edge, so no labelling gives each node one element per local
corner. The row kernels then take a node's incident (element, corner) pairs
in element order, 8 lanes per row when no node has more than 8 incident
elements (3 blocks) and 16 otherwise (5 blocks: 10 elements at the centre
line), with the CSR slot maps built for those lanes. The 4-block prism is
orientable and takes the relabelling path instead. Parity against the CPU
oracle (element loops, any hex mesh) at the bars of the block meshes.
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


def make_pair(oracle_mod, blocks, n=5, nz=4, prec=rt.OA_PREC_FP64, **kw):
    m = meshgen.star_prism(blocks, n, nz, perturb=0.2, seed=blocks)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=blocks)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    gm = rt.Mesh(m)
    gf = rt.Flow(gm, rt.default_settings(precision=prec, **kw))
    gf.set_field("U", U0)
    return m, oc, gm, gf


def random_state(m, oc, gf, seed=5):
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


@pytest.mark.parametrize("blocks", [3, 4, 5])
def test_star_mesh_graph_volume_and_assembly(oracle_mod, blocks):
    m, oc, gm, gf = make_pair(oracle_mod, blocks)
    incident = np.bincount(m.conn.ravel(), minlength=m.nn).max()
    assert incident == (2 * blocks if blocks == 5 else 8)
    rp, cols = gm.graph()
    orp, ocols = oc.graph()
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(cols, ocols)
    assert rel(gm.dual_volume(), oc.field("vol")) < 1e-14
    random_state(m, oc, gf)
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    assert rel(A_g, A_o) < TOL_ASM and rel(b_g, b_o) < TOL_ASM
    assert rel(gf.get_field("du"), oc.field("du")) < TOL_ASM
    A_o, b_o = oc.assemble_pcorr()
    A_g, b_g = gf.assemble_pcorr()
    assert rel(A_g, A_o) < TOL_ASM and rel(b_g, b_o) < TOL_ASM


@pytest.mark.parametrize("blocks", [3, 5])
def test_star_mesh_field_updates(oracle_mod, blocks):
    m, oc, gm, gf = make_pair(oracle_mod, blocks)
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


@pytest.mark.parametrize("blocks", [3, 5])
def test_star_mesh_simple_iterations(oracle_mod, blocks):
    kw = dict(mom_rtol=1e-13, pc_rtol=1e-13, mom_maxit=500, pc_maxit=5000)
    m, oc, gm, gf = make_pair(oracle_mod, blocks, **kw)
    oc.initialize()
    gf.initialize()
    for _ in range(5):
        so = oc.simple_iteration()
        sg = gf.simple_iterate(1)[0]
        assert abs(sg["continuity_rms"] - so["continuity_rms"]) <= 1e-9 * abs(so["continuity_rms"]) + 1e-18
    for k in ["U", "p", "mDot"]:
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k


def test_star_mesh_mixed_and_high_resolution(oracle_mod):
    # five blocks (16 lanes per row): the mixed form within 1e-6 of the FP64
    # oracle, and the high-resolution blending factor and assembly in FP64
    kw = dict(mom_rtol=1e-7, pc_rtol=1e-10, mom_maxit=500, pc_maxit=5000)
    m, oc, gm, gf = make_pair(oracle_mod, 5, prec=rt.OA_PREC_MIXED, **kw)
    oc.initialize()
    gf.initialize()
    for _ in range(5):
        oc.simple_iteration()
    gf.simple_iterate(5)
    U_o = oc.field("U")
    assert np.abs(gf.get_field("U") - U_o).max() < 1e-6 * max(1.0, np.abs(U_o).max())
    kw = dict(mom_rtol=1e-13, pc_rtol=1e-13, mom_maxit=500, pc_maxit=5000, hr=1)
    m, oc, gm, gf = make_pair(oracle_mod, 5, **kw)
    oc.initialize()
    gf.initialize()
    for _ in range(3):
        oc.simple_iteration()
    gf.simple_iterate(3)
    for k in ["U", "p", "betaU"]:
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k
