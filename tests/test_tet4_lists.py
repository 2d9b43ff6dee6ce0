"""CPU check of the tet4 assembly's contribution lists (the element-to-CSR
slot map in the entry-owner direction, oa_tet4_lists.h): every element
corner's coefficient of every element node, and every fixed-value face's
boundary-ip coefficient, lands in exactly one CSR entry, the one of its (row,
column) pair, listed in ascending staged order; and summing synthetic staged
values through the lists reproduces a scatter-add of the same values."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from openaccel_b200 import meshgen
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SIDE = np.array([[0, 1, 3], [1, 2, 3], [0, 3, 2], [0, 2, 1]])  # Tet4CVFEM.C sideNodeOrdinals_
OPP = np.array([2, 0, 1, 3])  # the element node on no side of the face


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("tl") / "tl_harness.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread", "-o", out,
                    os.path.join(ROOT, "tests", "tet4_lists_harness.cpp")], check=True)
    return C.CDLL(out)


def _case(n, seed):
    m, g, s, _ = meshgen.conduction(n, seed=seed, perturb=0.1)
    rp, cols = po.DiffCase(m, g, s).graph()
    diag = np.array([np.searchsorted(cols[rp[i]:rp[i + 1]], i) for i in range(m.nn)], np.int32)
    conn = np.ascontiguousarray(m.conn, np.int32)
    fe, fo = m.face_elem.astype(np.int64), m.face_ord.astype(np.int64)
    side = np.ascontiguousarray(conn[fe[:, None], SIDE[fo]], np.int32)
    opp = np.ascontiguousarray(conn[fe, OPP[fo]], np.int32)
    fixed = (m.bnd_kind[m.face_bnd] == meshgen.BND_FIXED_VALUE).astype(np.uint8)
    return m, rp, cols, diag, conn, side, opp, fixed


def _build(L, m, rp, cols, diag, conn, side, opp, fixed):
    ip = C.POINTER(C.c_int)
    up = C.POINTER(C.c_ubyte)
    assert L.tl_build(m.nn, m.ne, m.nf, rp.ctypes.data_as(ip), cols.ctypes.data_as(ip), diag.ctypes.data_as(ip),
                      conn.ctypes.data_as(ip), side.ctypes.data_as(ip), opp.ctypes.data_as(ip),
                      fixed.ctypes.data_as(up)) == 0
    L.tl_len_eidx.restype = C.c_long
    eptr = np.zeros(rp[-1] + 1, np.int32)
    eidx = np.zeros(L.tl_len_eidx(), np.int32)
    ediag = np.zeros(rp[-1], np.uint8)
    L.tl_get(eptr.ctypes.data_as(ip), eidx.ctypes.data_as(ip), ediag.ctypes.data_as(up))
    return eptr, eidx, ediag


@pytest.mark.parametrize("n,seed", [(3, 1), (5, 7)])
def test_lists_cover_every_contribution_once_in_its_entry(harness, n, seed):
    m, rp, cols, diag, conn, side, opp, fixed = _case(n, seed)
    eptr, eidx, ediag = _build(harness, m, rp, cols, diag, conn, side, opp, fixed)
    ne, nnz = m.ne, rp[-1]
    # every element contribution once, fixed-value face contributions once, nothing else
    face_ids = 16 * ne + 3 * np.repeat(np.nonzero(fixed)[0], 3) + np.tile(np.arange(3), int(fixed.sum()))
    expect = np.concatenate([np.arange(16 * ne), face_ids])
    assert np.array_equal(np.sort(eidx), np.sort(expect))
    # ascending within every list
    for s in range(nnz):
        seg = eidx[eptr[s]:eptr[s + 1]]
        assert np.all(np.diff(seg) > 0)
    # (row, column) of each contribution matches its entry
    entry_row = np.repeat(np.arange(m.nn), np.diff(rp))
    owner = np.repeat(np.arange(nnz), np.diff(eptr))
    el = eidx < 16 * ne
    e, a, k = eidx[el] // 16, (eidx[el] // 4) % 4, eidx[el] % 4
    assert np.array_equal(entry_row[owner[el]], conn[e, a])
    assert np.array_equal(cols[owner[el]], conn[e, k])
    fidx = eidx[~el] - 16 * ne
    f, q = fidx // 3, fidx % 3
    assert np.array_equal(entry_row[owner[~el]], side[f, q])
    assert np.array_equal(cols[owner[~el]], opp[f])
    # diagonal marks
    assert np.array_equal(np.nonzero(ediag)[0], rp[:-1] + diag)


def test_gather_equals_scatter_add(harness):
    m, rp, cols, diag, conn, side, opp, fixed = _case(4, 3)
    eptr, eidx, _ = _build(harness, m, rp, cols, diag, conn, side, opp, fixed)
    ne, nnz = m.ne, rp[-1]
    vals = np.random.default_rng(0).normal(size=16 * ne + 3 * m.nf)
    gathered = np.add.reduceat(vals[eidx], eptr[:-1]) * (np.diff(eptr) > 0)
    # scatter-add reference through a dense (row, col) -> entry map
    slot = {(r, c): s for r in range(m.nn) for s, c in zip(range(rp[r], rp[r + 1]), cols[rp[r]:rp[r + 1]])}
    ref = np.zeros(nnz)
    for e in range(ne):
        for a_ in range(4):
            for k_ in range(4):
                ref[slot[(conn[e, a_], conn[e, k_])]] += vals[16 * e + 4 * a_ + k_]
    for f in np.nonzero(fixed)[0]:
        for q_ in range(3):
            ref[slot[(side[f, q_], opp[f])]] += vals[16 * ne + 3 * f + q_]
    assert np.allclose(gathered, ref, rtol=1e-12, atol=1e-12)
