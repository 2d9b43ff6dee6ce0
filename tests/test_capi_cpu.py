"""CPU checks of the drop-in boundary: the CUDA library loads without a GPU
and exports every entry point include/openaccel_b200.h declares; argument
validation that needs no device fails loudly with a status and message."""
import ctypes as C
import os
import re

import pytest

from openaccel_b200 import runtime

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "openaccel_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(oa_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_runtime_exports():
    assert declared_symbols() == sorted(runtime.EXPORTS)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(runtime.LIB_PATH):
        pytest.fail(f"CUDA library missing: {runtime.LIB_PATH}")
    L = C.CDLL(runtime.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_version_and_argument_errors_without_gpu():
    L = runtime.lib()
    assert b"sm_100a" in L.oa_version()
    # null output handle: rejected before any device work
    st = L.oa_mesh_create(None, 0, None, 0, 8, None, None, None, 0, None)
    assert st == 1
    assert b"bad arguments" in L.oa_last_error()
    assert L.oa_flow_sync(None) == 1
    # the boundary-type, SST driver and diffusivity entry points check their
    # arguments before touching a device
    assert L.oa_flow_set_boundary_types(None, None, 0, 0) == 1
    c = runtime.SstConstants()
    assert L.oa_flow_sst_iterate(None, 1, C.byref(c), None, None, None, 1.0, 1e-8, 10, None) == 1
    assert L.oa_sst_diffusivities(-1, C.byref(c), None, None, None, None, None, None, None) == 1
    assert L.oa_update_gradient(None, 2) == 1


def test_meshgen_conventions():
    from openaccel_b200 import meshgen

    m = meshgen.cavity(3)
    assert m.nn == 64 and m.ne == 27 and m.nf == 54
    # lid faces first (boundary 0), z+ ordinal 5
    assert (m.face_ord[m.face_bnd == 0] == 5).all()
    # right-handed elements
    x = m.coords[m.conn[0]]
    assert (x[1] - x[0])[0] > 0 and (x[3] - x[0])[1] > 0 and (x[4] - x[0])[2] > 0


def test_residual_history_csv(tmp_path):
    import csv

    from openaccel_b200 import runtime as rt

    def stats(i):
        cd = lambda r: dict(n_iterations=3, fallback=0, solver_initial_res=[r, 2 * r, 3 * r],
                            solver_final_res=[r / 10, r / 20, r / 30], scaled_initial_res=[r, r, r])
        d = dict(mom_iters=3 + i, pc_iters=20 + i, pc_refinements=2, mom_res=1e-3, pc_res=1e-5,
                 continuity_rms=10.0 ** -i, continuity_rms_raw=2.0 * 10.0 ** -i, mom=cd(0.5), pc=cd(0.25))
        d.update({k: 0.1 * (j + 1) for j, k in enumerate(rt.PHASES)})
        return d

    path = tmp_path / "history.csv"
    h = rt.ResidualHistory(str(path))
    h.add([stats(1), stats(2)])
    h.add([stats(3)])
    with open(path) as fh:
        rows = list(csv.DictReader(fh))
    assert [int(r["iteration"]) for r in rows] == [1, 2, 3]
    assert [float(r["continuity_rms"]) for r in rows] == [0.1, 0.01, 0.001]
    assert float(rows[0]["mom_initial_v"]) == 1.0 and float(rows[2]["mom_final_w"]) == 0.5 / 30
    assert float(rows[1]["pc_initial"]) == 0.25 and int(rows[2]["pc_iters"]) == 23
    assert float(rows[0]["ms_pcorr_solve"]) == 0.4
    assert h.column("mom_iters") == [4, 5, 6] and len(rt.ResidualHistory.COLUMNS) == len(rows[0])
