"""CPU checks of the Exodus II reader / writer (openaccel_b200.exodus): a
written mesh with nodal result fields reads back bit for bit; the netCDF
container agrees with scipy's independent netCDF reader; the reference's own
cavity example mesh (when the reference checkout is present) reads into the
engine's arrays and runs through the oracle."""
import os

import numpy as np
import pytest

from openaccel_b200 import exodus, meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("OA_REFERENCE_ROOT", os.path.join(os.path.dirname(ROOT), "reference"))


def test_round_trip_with_fields(tmp_path):
    m = meshgen.cavity(4, perturb=0.2, seed=1)
    rng = np.random.default_rng(0)
    fields = {"velocity_x": rng.normal(size=(3, m.nn)), "pressure": rng.normal(size=(3, m.nn))}
    p = tmp_path / "m.e"
    exodus.write_mesh(p, m.coords, m.conn, m.face_elem, m.face_ord, m.face_bnd, ["lid", "walls"],
                      nodal_fields=fields, times=[0.1, 0.2, 0.3])
    r = exodus.read_mesh(p)
    np.testing.assert_array_equal(r.coords, m.coords)
    np.testing.assert_array_equal(r.conn, m.conn)
    np.testing.assert_array_equal(r.face_elem, m.face_elem)
    np.testing.assert_array_equal(r.face_ord, m.face_ord)
    np.testing.assert_array_equal(r.face_bnd, m.face_bnd)
    assert r.elem_type == "HEX8" and r.side_set_names == ["lid", "walls"]
    t, f = exodus.read_nodal_fields(p)
    np.testing.assert_array_equal(t, [0.1, 0.2, 0.3])
    for k, v in fields.items():
        np.testing.assert_array_equal(f[k], v)
    # an independent netCDF reader sees the same container
    scipy_io = pytest.importorskip("scipy.io")
    g = scipy_io.netcdf_file(str(p), "r", mmap=False)
    np.testing.assert_array_equal(g.variables["connect1"].data - 1, m.conn)
    np.testing.assert_array_equal(g.variables["vals_nod_var2"].data, fields["pressure"])
    g.close()


def test_tet_mesh_round_trip(tmp_path):
    tm, _, _, _ = meshgen.conduction(2)
    p = tmp_path / "t.e"
    exodus.write_mesh(p, tm.coords, tm.conn, tm.face_elem, tm.face_ord, tm.face_bnd)
    r = exodus.read_mesh(p)
    assert r.elem_type == "TETRA4"
    np.testing.assert_array_equal(r.conn, tm.conn)
    np.testing.assert_array_equal(r.face_ord, tm.face_ord)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "examples", "cavity", "mesh.e")),
                    reason="reference checkout not present")
def test_reference_cavity_mesh_through_the_oracle(oracle_mod):
    """examples/cavity/mesh.e: 400 hex8 one element thick, side sets top /
    sides / frontandback (Ioss lower-cases part names). Read, agree with
    scipy's reader, and run two SIMPLE iterations of the oracle with the top
    moving at (1, 0, 0). The example's front and back are symmetry planes,
    which this engine does not build; here they are no-slip walls and the lid
    is applied last so its nodes keep the lid velocity."""
    path = os.path.join(REF, "examples", "cavity", "mesh.e")
    r = exodus.read_mesh(path)
    assert (r.nn, r.ne, r.elem_type) == (882, 400, "HEX8")
    assert [n.lower() for n in r.side_set_names] == ["top", "sides", "frontandback"]
    scipy_io = pytest.importorskip("scipy.io")
    g = scipy_io.netcdf_file(path, "r", mmap=False)
    np.testing.assert_array_equal(g.variables["connect1"].data - 1, r.conn)
    np.testing.assert_array_equal(g.variables["coordz"].data, r.coords[:, 2])
    g.close()
    top = r.boundary_index("TOP")
    bnd = np.where(r.face_bnd == top, 1, 0).astype(np.int32)
    m = meshgen.HexMesh(0, 0, 0, r.coords, r.conn, r.face_elem, r.face_ord, bnd,
                        np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]]))
    c = oracle_mod.FlowCase(m, oracle_mod.default_settings(ref_node=0))
    c.initialize()
    for _ in range(2):
        st = c.simple_iteration()
    assert np.isfinite(st["continuity_rms"]) and np.abs(c.field("U")).max() > 0
