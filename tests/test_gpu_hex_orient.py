"""Hex meshes whose elements number their corners from different starting
corners or axes (as meshes from other tools do, the reference's cavity
example among them): the library relabels them into a consistently oriented
block and the result must not depend on the labelling. Parity with the
oracle, which runs element by element in the caller's labelling: assembled
systems within 1e-12, fields (mass flows in the caller's ip order) within
1e-10 after five tight-solved SIMPLE iterations; and the same through an
Exodus II file written and read back by openaccel_b200.exodus."""
import numpy as np
import pytest

from openaccel_b200 import exodus, meshgen
from openaccel_b200 import runtime as rt

pytestmark = pytest.mark.gpu

SIGN = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]])
FACE = [(0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (0, 4, 7, 3), (0, 3, 2, 1), (4, 5, 6, 7)]


def rel(a, b):
    d = np.linalg.norm(np.asarray(a) - np.asarray(b))
    n = np.linalg.norm(np.asarray(b))
    return d / n if n > 0 else d


def proper_rotations():
    out = []
    for perm in ([0, 1, 2], [0, 2, 1], [1, 0, 2], [1, 2, 0], [2, 0, 1], [2, 1, 0]):
        for s in np.array(np.meshgrid([1, -1], [1, -1], [1, -1])).T.reshape(-1, 3):
            M = np.zeros((3, 3), int)
            M[range(3), perm] = s
            if round(np.linalg.det(M)) != 1:
                continue
            P = []
            for k in range(8):
                o = np.zeros(3, int)
                o[perm] = s * SIGN[k]
                P.append(int(np.where((SIGN == o).all(axis=1))[0][0]))
            out.append(P)
    return out


def rotated_mesh(m, seed):
    """The same mesh with every element's corners relabelled by a random
    proper rotation; face ordinals re-expressed in the new labelling."""
    R = proper_rotations()
    rng = np.random.default_rng(seed)
    conn = np.array([m.conn[e][R[r]] for e, r in enumerate(rng.integers(0, len(R), m.ne))], np.int32)
    ford = m.face_ord.copy()
    for f, e in enumerate(m.face_elem):
        nodes = set(m.conn[e][list(FACE[m.face_ord[f]])])
        ford[f] = next(g for g in range(6) if set(conn[e][list(FACE[g])]) == nodes)
    import dataclasses

    return dataclasses.replace(m, conn=conn, face_ord=ford.astype(np.int32))


def test_rotated_connectivity_matches_oracle(oracle_mod):
    base = meshgen.cavity(6, perturb=0.2, seed=31)
    m = rotated_mesh(base, 5)
    U0 = meshgen.initial_velocity(base, sigma=0.1, seed=31)
    kw = dict(mom_rtol=1e-13, pc_rtol=1e-13)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(**kw))
    gf.set_field("U", U0)
    oc.initialize()
    gf.initialize()
    np.testing.assert_allclose(gf.get_field("mDot"), oc.field("mDot"), rtol=0, atol=1e-15)
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    assert rel(A_g, A_o) < 1e-12 and rel(b_g, b_o) < 1e-12
    A_o, b_o = oc.assemble_pcorr()
    A_g, b_g = gf.assemble_pcorr()
    assert rel(A_g, A_o) < 1e-12 and rel(b_g, b_o) < 1e-12
    for _ in range(5):
        oc.simple_iteration()
    gf.simple_iterate(5)
    for k in ("U", "p", "mDot"):
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k
    # and the unrotated mesh gives the same node fields
    g0 = rt.Flow(rt.Mesh(base), rt.default_settings(**kw))
    g0.set_field("U", U0)
    g0.initialize()
    g0.simple_iterate(5)
    for k in ("U", "p"):
        assert rel(gf.get_field(k), g0.get_field(k)) < 1e-10, k


def test_exodus_round_trip_runs_the_engine(tmp_path):
    base = meshgen.cavity(5, perturb=0.2, seed=3)
    m = rotated_mesh(base, 9)
    path = tmp_path / "cavity.e"
    exodus.write_mesh(path, m.coords, m.conn, m.face_elem, m.face_ord, m.face_bnd, ["lid", "walls"])
    r = exodus.read_mesh(path)
    assert r.side_set_names == ["lid", "walls"]
    np.testing.assert_array_equal(r.conn, m.conn)
    import dataclasses

    mr = dataclasses.replace(m, coords=r.coords, conn=r.conn, face_elem=r.face_elem, face_ord=r.face_ord,
                             face_bnd=r.face_bnd)
    gf = rt.Flow(rt.Mesh(mr), rt.default_settings(mom_rtol=1e-13, pc_rtol=1e-13))
    g0 = rt.Flow(rt.Mesh(base), rt.default_settings(mom_rtol=1e-13, pc_rtol=1e-13))
    for f in (gf, g0):
        f.initialize()
        f.simple_iterate(3)
    for k in ("U", "p"):
        assert rel(gf.get_field(k), g0.get_field(k)) < 1e-10, k


def test_rotated_connectivity_with_symmetry_planes(oracle_mod):
    # the symmetry face masks follow the relabelled face ordinals: a rotated
    # symmetry box against the oracle on the caller's labelling
    base = meshgen.symmetry_box(6, perturb=0.2, seed=33)
    m = rotated_mesh(base, 9)
    types = [rt.OA_BTYPE_WALL, rt.OA_BTYPE_WALL, rt.OA_BTYPE_SYMMETRY, rt.OA_BTYPE_SYMMETRY]
    U0 = meshgen.initial_velocity(base, sigma=0.1, seed=33)
    kw = dict(mom_rtol=1e-13, pc_rtol=1e-13)
    oc = oracle_mod.FlowCase(m, oracle_mod.default_settings(**kw), U0=U0)
    oc.set_boundary_types(types, correct_gradients=True)
    gf = rt.Flow(rt.Mesh(m), rt.default_settings(**kw))
    gf.set_boundary_types(types, correct_gradients=True)
    gf.set_field("U", U0)
    oc.initialize()
    gf.initialize()
    A_o, b_o = oc.assemble_momentum()
    A_g, b_g = gf.assemble_momentum()
    assert rel(A_g, A_o) < 1e-12 and rel(b_g, b_o) < 1e-12
    for _ in range(3):
        oc.simple_iteration()
    gf.simple_iterate(3)
    for k in ("U", "p", "gradU", "gradP"):
        assert rel(gf.get_field(k), oc.field(k)) < 1e-10, k
