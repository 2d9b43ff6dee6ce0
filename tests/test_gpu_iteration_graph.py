"""The whole SIMPLE outer iteration as one CUDA graph (settings.use_graphs = 2).

After a first eager iteration (which sets up the solvers and the AMG
hierarchy), oa_simple_iterate launches one graph per outer iteration: the
momentum and pressure-correction solves run their convergence loops as
device-side conditional WHILE nodes, the AMG refresh and the BiCGStab fallback
as IF nodes, and every scalar the host reports comes back in one pinned copy.
The decisions are the eager path's own, taken on the device, so the fields,
the iteration counts and the ControlData must match the eager path exactly.
"""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu

FIELDS = ("U", "p", "mDot", "gradU", "gradP", "du", "div")
STAT_KEYS = ("mom_iters", "pc_iters", "pc_refinements", "continuity_rms")


def flow(m, U0, **kw):
    f = rt.Flow(rt.Mesh(m), rt.default_settings(**kw))
    f.set_field("U", U0)
    f.initialize()
    return f


def run_both(m, U0, iters, **kw):
    eager = flow(m, U0, use_graphs=1, **kw)
    graph = flow(m, U0, use_graphs=2, **kw)
    se = eager.simple_iterate(iters)
    sg = graph.simple_iterate(iters)
    return eager, graph, se, sg


def assert_same(eager, graph, se, sg):
    for k in FIELDS:
        np.testing.assert_array_equal(graph.get_field(k), eager.get_field(k), err_msg=k)
    for a, b in zip(se, sg):
        for k in STAT_KEYS:
            assert a[k] == b[k], (k, a[k], b[k])
        assert a["pc_res"] == b["pc_res"] and a["mom_res"] == b["mom_res"]
    for sys in (0, 1):
        ce, cg = eager.last_control(sys), graph.last_control(sys)
        assert ce == cg


@pytest.mark.parametrize("precision", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_graph_iterations_match_eager(precision):
    m = meshgen.cavity(16, perturb=0.2, seed=3)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=3)
    eager, graph, se, sg = run_both(m, U0, 6, precision=precision)
    assert_same(eager, graph, se, sg)
    # the phases are timed by event nodes inside the graph
    assert all(s["ms_pcorr_solve"] > 0 and s["ms_momentum_assembly"] > 0 for s in sg[1:])


def test_graph_amg_refresh_schedule_follows_eager():
    # refresh 4 over 9 iterations: numeric phases inside the graph at solves 4 and 8
    m = meshgen.cavity(14, perturb=0.2, seed=5)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=5)
    eager = flow(m, U0, use_graphs=1, precision=rt.OA_PREC_MIXED)
    graph = flow(m, U0, use_graphs=2, precision=rt.OA_PREC_MIXED)
    for f in (eager, graph):
        f.set_tuning(block_rows=128, block_elements=128, block_assembly=128, gcr_chunk=2, amg_refresh=4)
    se = eager.simple_iterate(9)
    sg = graph.simple_iterate(9)
    assert_same(eager, graph, se, sg)


def test_graph_recaptured_after_tuning_and_time_step():
    m = meshgen.cavity(12, perturb=0.2, seed=8)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=8)
    eager = flow(m, U0, use_graphs=1)
    graph = flow(m, U0, use_graphs=2)
    se, sg = [], []
    for f, s in ((eager, se), (graph, sg)):
        s += f.simple_iterate(3)
        f.set_tuning(block_rows=64, block_elements=32, block_assembly=64, gcr_chunk=4, amg_refresh=8)
        s += f.simple_iterate(2)
        f.advance_time(rt.OA_TIME_BDF1, 0.1)
        s += f.simple_iterate(2)
        f.advance_time(rt.OA_TIME_BDF2, 0.05)
        s += f.simple_iterate(2)
    assert_same(eager, graph, se, sg)


def test_graph_high_resolution_and_simplec():
    m = meshgen.cavity(12, perturb=0.2, seed=9)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=9)
    eager, graph, se, sg = run_both(m, U0, 4, hr=1, du_mode=1, precision=rt.OA_PREC_MIXED)
    assert_same(eager, graph, se, sg)


def test_graph_counts_its_launches():
    m = meshgen.cavity(12, perturb=0.2, seed=2)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=2)
    f = flow(m, U0, use_graphs=2, precision=rt.OA_PREC_MIXED)
    f.simple_iterate(1)  # eager
    f.simple_iterate(1)  # captures and launches
    l0 = rt.launch_count()
    st = f.simple_iterate(1)[0]
    n = rt.launch_count() - l0
    # at least the assembly and correction kernels plus one V-cycle per
    # pressure iteration, and far fewer than a launch per row
    assert n > 20 + st["pc_iters"] * 5
    assert n < 20000


@pytest.mark.parametrize("precision", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_graph_with_bicgstab_pressure_solves(monkeypatch, precision):
    # the pressure solve's BiCGStab loops (the fallback branch of the graph)
    # taken from the start: graph and eager still agree bit for bit
    monkeypatch.setenv("OA_KRYLOV", "bicgstab")
    m = meshgen.cavity(12, perturb=0.2, seed=13)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=13)
    eager, graph, se, sg = run_both(m, U0, 4, precision=precision)
    assert_same(eager, graph, se, sg)
