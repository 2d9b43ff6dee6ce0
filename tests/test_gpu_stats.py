"""Per-iteration statistics of oa_simple_iterate: Krylov counts, residuals
and the device time of each phase (CUDA events on the flow's stream)."""
import math

import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_iteration_stats_and_phase_times(prec):
    m = meshgen.cavity(8, perturb=0.2, seed=5)
    gm = rt.Mesh(m)
    f = rt.Flow(gm, rt.default_settings(precision=prec))
    f.set_field("U", meshgen.initial_velocity(m, sigma=0.1, seed=5))
    f.initialize()
    st = f.simple_iterate(3)
    assert len(st) == 3
    for s in st:
        assert s["pc_iters"] > 0 and s["mom_iters"] > 0
        assert s["pc_res"] <= rt.default_settings().pc_rtol * 1.0001
        assert math.isfinite(s["continuity_rms"]) and s["continuity_rms"] > 0
        for k in rt.PHASES:
            assert math.isfinite(s[k]) and s[k] > 0.0, k
    if prec == rt.OA_PREC_MIXED:
        assert all(s["pc_refinements"] >= 1 for s in st)


def test_residual_history_of_a_run(tmp_path):
    # the CSV log of an eager run and of a whole-iteration-graph run hold one
    # row per outer iteration with the reported residuals
    import csv

    m = meshgen.cavity(8, perturb=0.2, seed=6)
    for graphs in (1, 2):
        f = rt.Flow(rt.Mesh(m), rt.default_settings(use_graphs=graphs, precision=rt.OA_PREC_MIXED))
        f.set_field("U", meshgen.initial_velocity(m, sigma=0.1, seed=6))
        f.initialize()
        path = tmp_path / f"history{graphs}.csv"
        h = rt.ResidualHistory(str(path))
        st = f.simple_iterate(2, history=h) + f.simple_iterate(3, history=h)
        with open(path) as fh:
            rows = list(csv.DictReader(fh))
        assert len(rows) == 5 and [int(r["iteration"]) for r in rows] == [1, 2, 3, 4, 5]
        for r, s in zip(rows, st):
            assert float(r["continuity_rms"]) == s["continuity_rms"]
            assert int(r["pc_iters"]) == s["pc_iters"] and float(r["pc_initial"]) == s["pc"]["solver_initial_res"][0]
            assert float(r["mom_final_w"]) == s["mom"]["solver_final_res"][2]
        assert h.column("continuity_rms")[-1] < h.column("continuity_rms")[0]
