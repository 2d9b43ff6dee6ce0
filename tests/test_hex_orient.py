"""CPU checks of the hex8 relabelling (openaccel_b200/csrc/oa_hex_orient.h)
that lets the row kernels take hex meshes whose elements start their corner
numbering at different corners or axes, such as the reference's own cavity
example mesh: the 24 rotations are proper (positive Jacobian kept); after
orientation no node is the same local corner of two elements; every element
keeps its node set; the ip and face maps are consistent with the
permutation; a mesh that is not a block is told apart (the row kernels then
run on incident-element lists) from one that is not a valid hex mesh."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from openaccel_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SIGN = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]])
LR = [(0, 1), (1, 2), (2, 3), (0, 3), (4, 5), (5, 6), (6, 7), (4, 7), (0, 4), (1, 5), (2, 6), (3, 7)]
FACE = [(0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (0, 4, 7, 3), (0, 3, 2, 1), (4, 5, 6, 7)]


@pytest.fixture(scope="module")
def H(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("ho") / "ho_harness.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", out,
                    os.path.join(ROOT, "tests", "hex_orient_harness.cpp")], check=True)
    return C.CDLL(out)


def rotation(H, r):
    p = (C.c_int * 8)()
    assert H.ho_rotation(int(r), p) == 0
    return np.array(list(p))


def orient(H, m_nn, conn):
    conn = np.ascontiguousarray(conn, np.int32)
    out = np.zeros_like(conn)
    rot = np.zeros(conn.shape[0], np.uint8)
    st = H.ho_orient(m_nn, conn.shape[0], conn.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                     rot.ctypes.data_as(C.c_void_p))
    return st, out, rot


def corner_conflicts(nn, conn):
    seen = np.zeros((nn, 8), bool)
    bad = 0
    for a in range(8):
        nodes = conn[:, a]
        bad += len(nodes) - len(np.unique(nodes))
    return bad


def test_rotations_are_the_24_proper_ones(H):
    assert H.ho_count() == 24
    perms = {tuple(rotation(H, r)) for r in range(24)}
    assert len(perms) == 24 and tuple(range(8)) == tuple(rotation(H, 0))
    for r in range(24):
        P = rotation(H, r)
        # the map new corner k -> old corner P[k] is a linear map of the corner
        # signs with determinant +1
        M = np.linalg.lstsq(SIGN.astype(float), SIGN[P].astype(float), rcond=None)[0]
        assert np.allclose(SIGN @ M, SIGN[P]) and np.isclose(np.linalg.det(M), 1.0)


def test_ip_and_face_maps(H):
    for r in range(24):
        P = rotation(H, r)
        for q, (a, b) in enumerate(LR):
            o, s = C.c_int(), C.c_int()
            H.ho_ip_map(r, q, C.byref(o), C.byref(s))
            la, lb = LR[o.value]
            assert (s.value == 1 and (la, lb) == (P[a], P[b])) or (s.value == -1 and (la, lb) == (P[b], P[a]))
        inv = np.argsort(P)
        for f in range(6):
            g = H.ho_face_map(r, f)
            assert sorted(inv[list(FACE[f])]) == sorted(FACE[g])


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_randomly_rotated_block_is_reoriented(H, seed):
    m = meshgen.cavity(5, perturb=0.2, seed=seed)
    rng = np.random.default_rng(seed)
    rots = rng.integers(0, 24, m.ne)
    conn = np.stack([m.conn[e][rotation(H, rots[e])] for e in range(m.ne)])
    assert corner_conflicts(m.nn, conn) > 0
    st, out, rot = orient(H, m.nn, conn)
    assert st == 0
    assert corner_conflicts(m.nn, out) == 0
    assert all(set(out[e]) == set(conn[e]) for e in range(m.ne))
    for e in range(m.ne):
        np.testing.assert_array_equal(out[e], conn[e][rotation(H, rot[e])])
    # positive Jacobian kept (corner-1, corner-3, corner-4 edges)
    x = m.coords[out]
    J = np.stack([x[:, 1] - x[:, 0], x[:, 3] - x[:, 0], x[:, 4] - x[:, 0]], axis=1)
    assert (np.linalg.det(J) > 0).all()


def test_reference_cavity_example_mesh(H):
    path = os.path.join(os.environ.get("OA_REFERENCE_ROOT", os.path.join(os.path.dirname(ROOT), "reference")),
                        "examples", "cavity", "mesh.e")
    if not os.path.exists(path):
        pytest.skip("reference checkout not present")
    from openaccel_b200 import exodus

    m = exodus.read_mesh(path)
    assert corner_conflicts(m.nn, m.conn) == 40
    st, out, rot = orient(H, m.nn, m.conn)
    assert st == 0 and corner_conflicts(m.nn, out) == 0


def test_non_block_mesh_is_rejected(H):
    """Three hexes closing a fan around an interior vertical edge (valence 3):
    walking around the edge returns with a rotated frame, so no consistent
    block orientation exists."""
    ang = np.deg2rad(np.arange(6) * 60.0)
    ring = [[np.cos(a), np.sin(a)] for a in ang]
    x = [[0.0, 0.0]] + ring
    coords = np.array([p + [z] for z in (0.0, 1.0) for p in x], float)
    top = len(x)
    quads = [(0, 1, 2, 3), (0, 3, 4, 5), (0, 5, 6, 1)]
    conn = np.array([[a, b, c, d, a + top, b + top, c + top, d + top] for a, b, c, d in quads])
    st, out, rot = orient(H, coords.shape[0], conn)
    assert st == 1


@pytest.mark.parametrize("blocks,expect", [(3, 1), (4, 0), (5, 1)])
def test_star_prisms(H, blocks, expect):
    """Polygon split into 3, 4 or 5 blocks around its centre: only 4 (four
    elements around every edge) is a consistently orientable block."""
    m = meshgen.star_prism(blocks, 3, 2)
    st, out, rot = orient(H, m.nn, m.conn)
    assert st == expect
    if st == 0:
        assert corner_conflicts(m.nn, out) == 0
        assert corner_conflicts(m.nn, m.conn) > 0  # it did need the relabelling


def test_face_shared_by_three_elements_is_invalid(H):
    m = meshgen.cavity(2)
    conn = np.concatenate([m.conn, m.conn[:1]])  # a duplicated element
    st, out, rot = orient(H, m.nn, np.ascontiguousarray(conn[::-1]))
    assert st == 2
