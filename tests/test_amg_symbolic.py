"""CPU check of the smoothed-aggregation symbolic phase: the prolongation,
T = A P and the Galerkin operator P^T A P rebuilt from the host term lists
(the same sums the device evaluates) agree with scipy sparse products, on a
pressure-correction matrix and on the tet4 diffusion matrix."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from openaccel_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NAMES = "agg prp pcols pdiag pgptr pglist ptrp ptrows ptsrc trp tcols ttptr tta ttp crp ccols cdg ctptr ctp ctt".split()


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("sa") / "sa_harness.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread", "-o", out,
                    os.path.join(ROOT, "tests", "amg_symbolic_harness.cpp")], check=True)
    return C.CDLL(out)


def _lists(L, A):
    ip = C.POINTER(C.c_int)
    nc = L.sa_build(A.shape[0], A.indptr.astype(np.int32).ctypes.data_as(ip),
                    A.indices.astype(np.int32).ctypes.data_as(ip))
    h = {}
    for nm in NAMES:
        f = getattr(L, "sa_len_" + nm)
        f.restype = C.c_long
        a = np.zeros(f(), np.int32)
        getattr(L, "sa_get_" + nm)(a.ctypes.data_as(ip))
        h[nm] = a
    return nc, h


def _check(L, A, wp=0.74):
    import scipy.sparse as sp

    A = A.tocsr()
    A.sort_indices()
    N = A.shape[0]
    nc, h = _lists(L, A)
    assert 0 < nc < N
    d = A.diagonal()
    s = np.add.reduceat(A.data[h["pglist"]], h["pgptr"][:-1])
    rows = np.repeat(np.arange(N), np.diff(h["prp"]))
    delta = np.zeros(h["pcols"].size)
    delta[h["prp"][:-1] + h["pdiag"]] = 1.0
    pv = delta - wp / d[rows] * s
    P = sp.csr_matrix((pv, h["pcols"], h["prp"]), shape=(N, nc))
    Pt = sp.csr_matrix((np.ones(N), (np.arange(N), h["agg"])), shape=(N, nc))
    Pref = (Pt - wp * (sp.diags(1 / d) @ (A @ Pt))).tocsr()
    scale = abs(Pref).max()
    assert abs(P - Pref).max() <= 1e-14 * scale
    PT = sp.csr_matrix((pv[h["ptsrc"]], h["ptrows"], h["ptrp"]), shape=(nc, N))
    assert abs(PT - Pref.T).max() <= 1e-14 * scale
    tv = np.add.reduceat(A.data[h["tta"]] * pv[h["ttp"]], h["ttptr"][:-1])
    T = sp.csr_matrix((tv, h["tcols"], h["trp"]), shape=(N, nc))
    AP = A @ Pref
    assert abs(T - AP).max() <= 1e-13 * abs(AP).max()
    cv = np.add.reduceat(pv[h["ctp"]] * tv[h["ctt"]], h["ctptr"][:-1])
    Ac = sp.csr_matrix((cv, h["ccols"], h["crp"]), shape=(nc, nc))
    Acr = (Pref.T @ A @ Pref).tocsr()
    assert abs(Ac - Acr).max() <= 1e-13 * abs(Acr).max()
    # coarse structure: sorted columns with the diagonal where cdg says
    assert np.all(h["ccols"][h["crp"][:-1] + h["cdg"]] == np.arange(nc))
    for c in range(0, nc, max(1, nc // 50)):
        row = h["ccols"][h["crp"][c]:h["crp"][c + 1]]
        assert np.all(np.diff(row) > 0)


def test_pressure_correction_matrix(harness, oracle_mod):
    import scipy.sparse as sp

    m = meshgen.cavity(10, perturb=0.2, seed=3)
    U0 = meshgen.initial_velocity(m, sigma=0.1, seed=3)
    c = oracle_mod.FlowCase(m, oracle_mod.default_settings(), U0=U0)
    c.initialize()
    c.assemble_momentum()
    A, _ = c.assemble_pcorr()
    rp, cols = c.graph()
    _check(harness, sp.csr_matrix((A, cols, rp), shape=(m.nn, m.nn)))


def test_tet4_diffusion_matrix(harness, oracle_mod):
    import scipy.sparse as sp

    m, g, s, _ = meshgen.conduction(6, perturb=0.2)
    c = oracle_mod.DiffCase(m, g, s)
    A, _ = c.assemble()
    rp, cols = c.graph()
    _check(harness, sp.csr_matrix((A, cols, rp), shape=(m.nn, m.nn)))
