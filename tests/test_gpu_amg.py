"""The AMG preconditioner's smoothers on the device: the Chebyshev smoother of
the small levels against damped Jacobi everywhere (OA_AMG_CHEB_DEGREE=0), on
the same pressure-correction systems of a skewed cavity."""
import numpy as np
import pytest

from openaccel_b200 import meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu


def _run(prec, n_iter=4):
    m = meshgen.cavity(24, perturb=0.2, seed=9)
    f = rt.Flow(rt.Mesh(m), rt.default_settings(precision=prec, pc_rtol=1e-10))
    f.set_field("U", meshgen.initial_velocity(m, sigma=0.1, seed=9))
    f.initialize()
    st = f.simple_iterate(n_iter)
    return st, f.get_field("U"), f.get_field("p")


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_chebyshev_levels_converge_faster_to_the_same_fields(monkeypatch, prec):
    monkeypatch.setenv("OA_AMG_CHEB_DEGREE", "0")
    st_j, U_j, p_j = _run(prec)
    monkeypatch.delenv("OA_AMG_CHEB_DEGREE")
    st_c, U_c, p_c = _run(prec)
    it_j = sum(s["pc_iters"] for s in st_j)
    it_c = sum(s["pc_iters"] for s in st_c)
    assert all(s["pc_res"] <= 1e-10 * 1.0001 for s in st_c)
    assert it_c < it_j, (it_c, it_j)
    # both solve each correction to 1e-10, so in FP64 the fields agree to
    # about that; in the mixed form the FP32 momentum solve stops at its own
    # rtol (1e-6) from a slightly different pressure, which bounds the gap
    tol = 1e-7 if prec == rt.OA_PREC_FP64 else 1e-5
    assert np.abs(U_c - U_j).max() <= tol * np.abs(U_j).max()
    assert np.abs(p_c - p_j).max() <= tol * np.abs(p_j).max()


def test_chebyshev_degree_out_of_range_is_rejected(monkeypatch):
    monkeypatch.setenv("OA_AMG_CHEB_DEGREE", "9")
    with pytest.raises(rt.OpenAccelError):
        _run(rt.OA_PREC_FP64, n_iter=1)


@pytest.mark.parametrize("prec", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_gcr_and_bicgstab_reach_the_same_fields(monkeypatch, prec):
    # the pressure correction's default Krylov method (GCR(2), one V-cycle per
    # iteration) against BiCGStab (two per iteration) on the same systems
    monkeypatch.setenv("OA_KRYLOV", "bicgstab")
    st_b, U_b, p_b = _run(prec)
    monkeypatch.delenv("OA_KRYLOV")
    st_g, U_g, p_g = _run(prec)
    assert all(s["pc_res"] <= 1e-10 * 1.0001 for s in st_g)
    vcycles_b = 2 * sum(s["pc_iters"] for s in st_b)
    vcycles_g = sum(s["pc_iters"] for s in st_g)
    assert vcycles_g <= vcycles_b, (vcycles_g, vcycles_b)
    tol = 1e-7 if prec == rt.OA_PREC_FP64 else 1e-5
    assert np.abs(U_g - U_b).max() <= tol * np.abs(U_b).max()
    assert np.abs(p_g - p_b).max() <= tol * np.abs(p_b).max()


@pytest.mark.parametrize("precision", [rt.OA_PREC_FP64, rt.OA_PREC_MIXED])
def test_hierarchy_refreshed_when_the_matrix_drifts(precision):
    # a high-Reynolds channel (mu = 1e-5) changes its pressure-correction
    # matrix a lot between the first outer iterations; with the default refresh
    # interval the drift test refreshes the AMG numerics early, so every solve
    # converges in a V-cycle count like the first one's (with a stale
    # hierarchy the second solve ran to maxit), in eager and graph form alike
    from openaccel_b200 import meshgen

    m = meshgen.channel(32, 12, 12, ratio=1.05)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=7)
    runs = []
    for graphs in (1, 2):
        f = rt.Flow(rt.Mesh(m), rt.default_settings(precision=precision, mu=1e-5, pc_rtol=1e-8, pc_maxit=3000,
                                                    use_graphs=graphs))
        f.set_field("U", U0)
        f.initialize()
        st = f.simple_iterate(4)
        for s in st:
            assert s["pc_iters"] < 100 and s["pc_res"] <= 1e-8 * 1.0001 and s["pc"]["fallback"] == 0, s["pc_iters"]
        runs.append((f, st))
    (fe, se), (fg, sg) = runs
    np.testing.assert_array_equal(fg.get_field("p"), fe.get_field("p"))
    assert [s["pc_iters"] for s in se] == [s["pc_iters"] for s in sg]
