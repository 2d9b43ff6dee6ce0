"""The autotuner (oa_flow_autotune): it returns a tuning from its candidate
sets, leaves the flow's state as it found it, and block sizes do not change
results (the row and element kernels' arithmetic is per thread group, so any
block size gives bit-identical output)."""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


def flow(m, U0, **kw):
    f = rt.Flow(rt.Mesh(m), rt.default_settings(**kw))
    f.set_field("U", U0)
    f.initialize()
    return f


def test_autotune_choices_and_state_restored():
    m = meshgen.cavity(20, perturb=0.2, seed=4)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=4)
    f = flow(m, U0, precision=rt.OA_PREC_MIXED, use_graphs=1)
    f.simple_iterate(2)
    before = {k: f.get_field(k) for k in ("U", "p", "mDot", "gradU", "gradP", "du", "div")}
    t = f.autotune(iters=2)
    assert t["block_rows"] in (32, 64, 128) and t["block_elements"] in (32, 64, 128)
    assert t["block_assembly"] in (32, 64, 128) and t["gcr_chunk"] in (2, 4) and t["amg_refresh"] in (4, 8, 16)
    assert t["amg_cheb_degree"] in (3, 4) and t["amg_prolong_damping"] in (0.74, 0.85)
    assert 0 < t["ms_per_iteration_after"] <= t["ms_per_iteration_before"] * 1.0000001
    for k, v in before.items():
        np.testing.assert_array_equal(f.get_field(k), v)
    st = f.simple_iterate(2)
    assert st[-1]["pc_res"] < 1e-8


def test_block_sizes_do_not_change_results():
    m = meshgen.cavity(12, perturb=0.2, seed=6)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=6)
    a = flow(m, U0)
    b = flow(m, U0)
    b.set_tuning(block_rows=32, block_elements=64, block_assembly=32, gcr_chunk=2, amg_refresh=8)
    a.simple_iterate(3)
    b.simple_iterate(3)
    for k in ("U", "p", "mDot"):
        np.testing.assert_array_equal(a.get_field(k), b.get_field(k))


def test_amg_smoothing_tuning_changes_schedule_not_answers():
    # a different Chebyshev degree / prolongation damping changes the V-cycle,
    # hence the iterates within the solve tolerance, but not the converged
    # answer; bad values are rejected
    m = meshgen.cavity(12, perturb=0.2, seed=7)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=7)
    kw = dict(mom_rtol=1e-12, pc_rtol=1e-12)
    a = flow(m, U0, **kw)
    b = flow(m, U0, **kw)
    b.set_tuning(block_rows=128, block_elements=128, block_assembly=128, gcr_chunk=2, amg_refresh=8,
                 amg_cheb_degree=4, amg_prolong_damping=0.85)
    a.simple_iterate(3)
    b.simple_iterate(3)
    for k in ("U", "p"):
        va, vb = a.get_field(k), b.get_field(k)
        assert np.linalg.norm(va - vb) <= 1e-9 * np.linalg.norm(va)
    with pytest.raises(rt.OpenAccelError):
        b.set_tuning(block_rows=128, block_elements=128, block_assembly=128, gcr_chunk=2, amg_refresh=8,
                     amg_cheb_degree=9)
