"""Batched independent cavities (uneven sizes and viscosities) assembled and
solved as one disjoint-union system: GPU against the oracle on the same batch,
and the batch against the cavities run one by one."""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


KW = dict(mom_rtol=1e-13, pc_rtol=1e-13, mom_maxit=500, pc_maxit=5000)


def _gpu_flow(mesh, mu, refs, **kw):
    gm = rt.Mesh(mesh)
    gf = rt.Flow(gm, rt.default_settings(ref_node=-1, **kw))
    gf.set_field("mu", mu)
    gf.set_reference_nodes(refs)
    gf.initialize()
    return gm, gf


def test_batch_matches_oracle(oracle_mod):
    b = meshgen.batch_cavities(sizes=[4, 6, 5], seed=7)
    gm, gf = _gpu_flow(b.mesh, b.mu, b.ref_nodes, **KW)
    oc = oracle_mod.FlowCase(b.mesh, oracle_mod.default_settings(ref_node=-1, **KW))
    oc.field("mu")[:] = b.mu
    oc.set_ref_nodes(b.ref_nodes)
    oc.initialize()
    A_o, b_o = oc.assemble_pcorr()
    A_g, b_g = gf.assemble_pcorr()
    assert rel(A_g, A_o) < 1e-12 and rel(b_g, b_o) < 1e-12
    for _ in range(4):
        oc.simple_iteration()
    gf.simple_iterate(4)
    for k in ["U", "p", "mDot"]:
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k


def test_batch_equals_separate_runs():
    sizes = [4, 6, 5]
    b = meshgen.batch_cavities(sizes=sizes, seed=7)
    gm, gf = _gpu_flow(b.mesh, b.mu, b.ref_nodes, **KW)
    gf.simple_iterate(4)
    U = gf.get_field("U").reshape(-1, 3)
    p = gf.get_field("p")
    for m, n in enumerate(sizes):
        c = meshgen.cavity(n)
        gm1 = rt.Mesh(c)
        f1 = rt.Flow(gm1, rt.default_settings(mu=float(b.viscosities[m]), **KW))
        f1.initialize()
        f1.simple_iterate(4)
        lo, hi = b.node_offsets[m], b.node_offsets[m + 1]
        assert rel(U[lo:hi].ravel(), f1.get_field("U")) < 1e-9
        assert rel(p[lo:hi], f1.get_field("p")) < 1e-9


def _segment_residuals(gm, A, b, x, offsets):
    import scipy.sparse as sp

    rp, cols = gm.graph()
    M = sp.csr_matrix((A, cols, rp), shape=(b.size, b.size))
    r = b - M @ x
    return np.array([np.linalg.norm(r[a:e]) / np.linalg.norm(b[a:e]) for a, e in zip(offsets[:-1], offsets[1:])])


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_batch_converges_per_cavity(prec):
    # a small, stiff cavity beside two large ones: the whole batch's residual
    # norm is dominated by the large ones, yet the solve stops only when every
    # cavity's own ||r|| <= rtol ||b|| (the segments are the stencil graph's
    # connected components), and the reported residual is the worst cavity's
    b = meshgen.batch_cavities(sizes=[14, 3, 12], seed=11, mu_min=1e-3, mu_max=1e-1)
    gm, gf = _gpu_flow(b.mesh, b.mu, b.ref_nodes, precision=prec, pc_rtol=1e-8)
    gf.simple_iterate(3)
    A, bb = gf.assemble_pcorr()
    x, it, res = gf.solve("pcorr", 1e-8, 5000)
    seg = _segment_residuals(gm, A, bb, x, b.node_offsets)
    assert seg.max() <= 1.02e-8, seg
    assert res == pytest.approx(seg.max(), rel=1e-3 if prec == rt.OA_PREC_FP64 else 1e-2, abs=1e-12)


def test_batch_graph_iterations_match_eager():
    # the captured outer iteration applies the same per-cavity tests
    b = meshgen.batch_cavities(sizes=[6, 4, 5], seed=3)
    runs = []
    for graphs in (1, 2):
        gm, gf = _gpu_flow(b.mesh, b.mu, b.ref_nodes, precision=rt.OA_PREC_MIXED, use_graphs=graphs)
        st = gf.simple_iterate(4)
        runs.append((st, gf.get_field("U"), gf.get_field("p")))
    (s1, u1, p1), (s2, u2, p2) = runs
    np.testing.assert_array_equal(u1, u2)
    np.testing.assert_array_equal(p1, p2)
    assert [s["pc_iters"] for s in s1] == [s["pc_iters"] for s in s2]
