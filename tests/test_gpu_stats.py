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
