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


def test_meshgen_conventions():
    from openaccel_b200 import meshgen

    m = meshgen.cavity(3)
    assert m.nn == 64 and m.ne == 27 and m.nf == 54
    # lid faces first (boundary 0), z+ ordinal 5
    assert (m.face_ord[m.face_bnd == 0] == 5).all()
    # right-handed elements
    x = m.coords[m.conn[0]]
    assert (x[1] - x[0])[0] > 0 and (x[3] - x[0])[1] > 0 and (x[4] - x[0])[2] > 0
