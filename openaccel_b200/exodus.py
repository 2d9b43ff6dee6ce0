"""Exodus II mesh and result files (the reference's mesh input and results
output: ``mesh.file_path`` / ``output_control.file_path``, read and written
through SEACAS Ioss in src/mesh/meshIO.cpp).

Exodus II files are netCDF "classic" or "64-bit offset" files. This module
reads and writes that container directly (big-endian header of dimensions,
attributes and variables, then fixed-size variables at their offsets and the
record variables interleaved per record), from the published netCDF file
format, and maps the Exodus conventions onto the engine's mesh arrays:

- coordinates ``coordx/coordy/coordz`` (or ``coord`` [num_dim][num_nodes]);
- element blocks ``connect<k>`` ([elements][nodes per element], 1-based node
  ids, attribute ``elem_type``); HEX8 and TETRA4 node orders are the Nalu
  master elements' own;
- side sets ``elem_ss<k>`` / ``side_ss<k>`` (1-based element ids, Exodus side
  numbers), named by ``ss_names``. Exodus HEX8 side s is Nalu hex8 face
  ordinal s - 1 (sides 1-4 around the element, 5 the bottom, 6 the top);
  TETRA4 side s is Nalu tet4 face ordinal s - 1.

Nodal result fields are written as Exodus nodal variables (``name_nod_var``,
``vals_nod_var<k>`` per time step), which the reference's results.e carries.
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np

NC_BYTE, NC_CHAR, NC_SHORT, NC_INT, NC_FLOAT, NC_DOUBLE = 1, 2, 3, 4, 5, 6
_NC_DIMENSION, _NC_VARIABLE, _NC_ATTRIBUTE = 10, 11, 12
_DTYPE = {NC_BYTE: ">i1", NC_CHAR: "S1", NC_SHORT: ">i2", NC_INT: ">i4", NC_FLOAT: ">f4", NC_DOUBLE: ">f8"}
_SIZE = {NC_BYTE: 1, NC_CHAR: 1, NC_SHORT: 2, NC_INT: 4, NC_FLOAT: 4, NC_DOUBLE: 8}


def _pad4(n):
    return (4 - n % 4) % 4


@dataclasses.dataclass
class NcVar:
    name: str
    dims: tuple
    nctype: int
    attrs: dict
    data: np.ndarray | None = None
    begin: int = 0
    vsize: int = 0


@dataclasses.dataclass
class NcFile:
    """Contents of a netCDF classic / 64-bit offset file."""

    dims: dict  # name -> length (0: the unlimited record dimension)
    attrs: dict
    variables: dict  # name -> NcVar
    numrecs: int = 0

    def record_dim(self):
        for k, v in self.dims.items():
            if v == 0:
                return k
        return None


class _Reader:
    def __init__(self, buf):
        self.b = buf
        self.p = 0

    def int(self):
        v = struct.unpack_from(">i", self.b, self.p)[0]
        self.p += 4
        return v

    def uint(self):
        v = struct.unpack_from(">I", self.b, self.p)[0]
        self.p += 4
        return v

    def int64(self):
        v = struct.unpack_from(">q", self.b, self.p)[0]
        self.p += 8
        return v

    def name(self):
        n = self.int()
        s = self.b[self.p:self.p + n].decode("utf-8")
        self.p += n + _pad4(n)
        return s

    def values(self, nctype, n):
        size = _SIZE[nctype] * n
        raw = self.b[self.p:self.p + size]
        self.p += size + _pad4(size)
        if nctype == NC_CHAR:
            return raw.decode("latin-1").rstrip("\x00")
        return np.frombuffer(raw, dtype=_DTYPE[nctype]).astype(_DTYPE[nctype][1:])

    def attrs(self):
        tag, n = self.int(), self.int()
        out = {}
        if tag == 0 and n == 0:
            return out
        if tag != _NC_ATTRIBUTE:
            raise ValueError("netCDF: attribute list expected")
        for _ in range(n):
            name = self.name()
            t = self.int()
            out[name] = (t, self.values(t, self.int()))
        return out


def read_netcdf(path) -> NcFile:
    """Parse a netCDF classic (CDF1) or 64-bit offset (CDF2) file."""
    with open(path, "rb") as fh:
        buf = fh.read()
    if buf[:3] != b"CDF" or buf[3] not in (1, 2):
        raise ValueError(f"{path}: not a netCDF classic or 64-bit offset file")
    version = buf[3]
    r = _Reader(buf)
    r.p = 4
    numrecs = r.uint()
    if numrecs == 0xFFFFFFFF:
        raise ValueError(f"{path}: streaming record count not supported")
    dims = {}
    tag, n = r.int(), r.int()
    if not (tag == 0 and n == 0):
        if tag != _NC_DIMENSION:
            raise ValueError("netCDF: dimension list expected")
        for _ in range(n):
            name = r.name()
            dims[name] = r.int()
    dim_names = list(dims)
    gattrs = r.attrs()
    variables = {}
    tag, n = r.int(), r.int()
    if not (tag == 0 and n == 0):
        if tag != _NC_VARIABLE:
            raise ValueError("netCDF: variable list expected")
        for _ in range(n):
            name = r.name()
            nd = r.int()
            ids = [r.int() for _ in range(nd)]
            vattrs = r.attrs()
            t = r.int()
            vsize = r.int()
            begin = r.int() if version == 1 else r.int64()
            variables[name] = NcVar(name, tuple(dim_names[i] for i in ids), t, vattrs, None, begin, vsize)
    f = NcFile(dims, gattrs, variables, numrecs)
    rec = f.record_dim()
    rec_vars = [v for v in variables.values() if v.dims and v.dims[0] == rec and rec is not None]
    recsize = sum(v.vsize for v in rec_vars)
    if len(rec_vars) == 1:  # a single record variable is not padded
        v = rec_vars[0]
        recsize = _SIZE[v.nctype] * int(np.prod([dims[d] for d in v.dims[1:]], dtype=np.int64))
    for v in variables.values():
        shape = [dims[d] for d in v.dims]
        dt = np.dtype(_DTYPE[v.nctype])
        if rec is not None and v.dims and v.dims[0] == rec:
            inner = shape[1:]
            n_in = int(np.prod(inner, dtype=np.int64))
            out = np.empty([numrecs] + inner, dtype=dt)
            for k in range(numrecs):
                off = v.begin + k * recsize
                out[k] = np.frombuffer(buf, dtype=dt, count=n_in, offset=off).reshape(inner)
            v.data = out
        else:
            n_el = int(np.prod(shape, dtype=np.int64))
            v.data = np.frombuffer(buf, dtype=dt, count=n_el, offset=v.begin).reshape(shape).copy()
    return f


def write_netcdf(path, f: NcFile):
    """Write a netCDF 64-bit offset (CDF2) file: fixed-size variables first,
    then the record variables interleaved per record."""
    dim_names = list(f.dims)
    rec = f.record_dim()

    def name_bytes(s):
        b = s.encode("utf-8")
        return struct.pack(">i", len(b)) + b + b"\0" * _pad4(len(b))

    def attr_bytes(attrs):
        if not attrs:
            return struct.pack(">ii", 0, 0)
        out = struct.pack(">ii", _NC_ATTRIBUTE, len(attrs))
        for k, (t, val) in attrs.items():
            if t == NC_CHAR:
                raw = val.encode("latin-1") if isinstance(val, str) else bytes(val)
                n = len(raw)
            else:
                arr = np.asarray(val, dtype=_DTYPE[t]).ravel()
                raw, n = arr.tobytes(), arr.size
            out += name_bytes(k) + struct.pack(">ii", t, n) + raw + b"\0" * _pad4(len(raw))
        return out

    vars_ = list(f.variables.values())
    fixed = [v for v in vars_ if not (rec is not None and v.dims and v.dims[0] == rec)]
    recs = [v for v in vars_ if rec is not None and v.dims and v.dims[0] == rec]
    for v in vars_:
        inner = [f.dims[d] for d in (v.dims[1:] if v in recs else v.dims)]
        size = _SIZE[v.nctype] * int(np.prod(inner, dtype=np.int64))
        v.vsize = size + _pad4(size)

    def header(offsets):
        h = b"CDF\x02" + struct.pack(">I", f.numrecs)
        if f.dims:
            h += struct.pack(">ii", _NC_DIMENSION, len(f.dims))
            for k in dim_names:
                h += name_bytes(k) + struct.pack(">i", f.dims[k])
        else:
            h += struct.pack(">ii", 0, 0)
        h += attr_bytes(f.attrs)
        if vars_:
            h += struct.pack(">ii", _NC_VARIABLE, len(vars_))
            for v in vars_:
                h += name_bytes(v.name) + struct.pack(">i", len(v.dims))
                h += b"".join(struct.pack(">i", dim_names.index(d)) for d in v.dims)
                h += attr_bytes(v.attrs) + struct.pack(">ii", v.nctype, v.vsize) + struct.pack(">q", offsets[v.name])
        else:
            h += struct.pack(">ii", 0, 0)
        return h

    hlen = len(header({v.name: 0 for v in vars_}))
    offsets, pos = {}, hlen
    for v in fixed:
        offsets[v.name] = pos
        pos += v.vsize
    rpos = pos
    for v in recs:
        offsets[v.name] = rpos
        rpos += v.vsize if len(recs) > 1 else 0
    with open(path, "wb") as fh:
        fh.write(header(offsets))
        for v in fixed:
            raw = np.ascontiguousarray(v.data, dtype=_DTYPE[v.nctype]).tobytes()
            fh.write(raw + b"\0" * (v.vsize - len(raw)))
        for k in range(f.numrecs):
            for v in recs:
                raw = np.ascontiguousarray(v.data[k], dtype=_DTYPE[v.nctype]).tobytes()
                pad = (v.vsize - len(raw)) if len(recs) > 1 else 0
                fh.write(raw + b"\0" * pad)


# Exodus side numbers -> Nalu face ordinals (hex8 and tet4 alike: side s is
# face s - 1; the node lists agree, Hex8CVFEM.C / Tet4CVFEM.C side ordinals)
@dataclasses.dataclass
class ExodusMesh:
    """Mesh read from an Exodus file, in the engine's arrays (0-based)."""

    coords: np.ndarray      # (nn, 3)
    conn: np.ndarray        # (ne, 8) hex8 or (ne, 4) tet4
    elem_type: str          # "HEX8" or "TETRA4"
    block_names: list
    face_elem: np.ndarray   # (nf,) element of each boundary face
    face_ord: np.ndarray    # (nf,) Nalu face ordinal
    face_bnd: np.ndarray    # (nf,) side-set index
    side_set_names: list
    elem_map: np.ndarray | None = None

    @property
    def nn(self):
        return self.coords.shape[0]

    @property
    def ne(self):
        return self.conn.shape[0]

    @property
    def nf(self):
        return self.face_elem.shape[0]

    def boundary_index(self, name):
        return self.side_set_names.index(name)


def _names(f: NcFile, var):
    v = f.variables.get(var)
    if v is None:
        return []
    out = []
    for row in np.atleast_2d(v.data):
        out.append(b"".join(bytes(c) for c in row).split(b"\0")[0].decode("latin-1").strip())
    return out


def read_mesh(path) -> ExodusMesh:
    """Coordinates, the element blocks (all of one type, hex8 or tet4,
    concatenated in block order) and the side sets of an Exodus II file."""
    f = read_netcdf(path)
    V = f.variables
    if "coordx" in V:
        coords = np.stack([V[c].data.astype(np.float64) for c in ("coordx", "coordy", "coordz")], axis=1)
    else:
        coords = np.ascontiguousarray(V["coord"].data.astype(np.float64).T)
    nblk = f.dims.get("num_el_blk", 0)
    conns, types = [], []
    for k in range(1, nblk + 1):
        v = V[f"connect{k}"]
        conns.append(v.data.astype(np.int64) - 1)
        t = v.attrs.get("elem_type", (NC_CHAR, ""))[1]
        types.append(str(t).upper())
    kinds = {("HEX8" if t.startswith("HEX") else "TETRA4" if t.startswith("TET") else t) for t in types}
    if len(kinds) != 1 or not kinds <= {"HEX8", "TETRA4"}:
        raise ValueError(f"{path}: element blocks of type {sorted(set(types))}; one of HEX8 or TETRA4 is supported")
    conn = np.concatenate(conns, axis=0).astype(np.int32)
    nss = f.dims.get("num_side_sets", 0)
    fe, fo, fb = [], [], []
    for k in range(1, nss + 1):
        e = V[f"elem_ss{k}"].data.astype(np.int64) - 1
        sd = V[f"side_ss{k}"].data.astype(np.int64) - 1
        fe.append(e)
        fo.append(sd)
        fb.append(np.full(e.shape, k - 1))
    cat = (lambda xs: np.concatenate(xs).astype(np.int32)) if nss else (lambda xs: np.zeros(0, np.int32))
    emap = V["elem_map"].data.astype(np.int64) if "elem_map" in V else None
    return ExodusMesh(coords, conn, kinds.pop(), _names(f, "eb_names"), cat(fe), cat(fo), cat(fb),
                      _names(f, "ss_names"), emap)


def _char_table(names, width=33):
    arr = np.zeros((len(names), width), dtype="S1")
    for i, n in enumerate(names):
        b = n.encode("latin-1")[:width - 1]
        arr[i, :len(b)] = np.frombuffer(b, dtype="S1")
    return arr


def write_mesh(path, coords, conn, face_elem, face_ord, face_bnd, side_set_names=None, block_name="block_1",
               nodal_fields=None, times=None, title="openaccel_b200"):
    """An Exodus II file with one element block, the side sets and,
    optionally, nodal result fields: nodal_fields maps a name to an array of
    shape (num_steps, nn) (one scalar per name; vector fields go in as
    components, e.g. velocity_x), times the step times."""
    coords = np.asarray(coords, np.float64)
    conn = np.asarray(conn)
    nn, ne, npe = coords.shape[0], conn.shape[0], conn.shape[1]
    etype = "HEX8" if npe == 8 else "TETRA4"
    face_bnd = np.asarray(face_bnd)
    nss = int(face_bnd.max()) + 1 if face_bnd.size else 0
    names = list(side_set_names) if side_set_names else [f"surface_{k + 1}" for k in range(nss)]
    dims = {"len_string": 33, "len_line": 81, "four": 4, "len_name": 33, "time_step": 0, "num_dim": 3,
            "num_nodes": nn, "num_elem": ne, "num_el_blk": 1, "num_el_in_blk1": ne, "num_nod_per_el1": npe}
    if nss:
        dims["num_side_sets"] = nss
    V = {}

    def var(name, dims_, t, data, attrs=None):
        V[name] = NcVar(name, tuple(dims_), t, attrs or {}, data)

    fields = nodal_fields or {}
    nsteps = 0
    if fields:
        nsteps = len(next(iter(fields.values())))
        dims["num_nod_var"] = len(fields)
    var("time_whole", ["time_step"], NC_DOUBLE, np.asarray(times if times is not None else np.arange(nsteps), float))
    var("eb_status", ["num_el_blk"], NC_INT, np.array([1]))
    var("eb_prop1", ["num_el_blk"], NC_INT, np.array([1]), {"name": (NC_CHAR, "ID")})
    for c, name in enumerate(("coordx", "coordy", "coordz")):
        var(name, ["num_nodes"], NC_DOUBLE, coords[:, c])
    var("eb_names", ["num_el_blk", "len_name"], NC_CHAR, _char_table([block_name]))
    var("coor_names", ["num_dim", "len_name"], NC_CHAR, _char_table(["x", "y", "z"]))
    var("elem_map", ["num_elem"], NC_INT, np.arange(1, ne + 1))
    var("connect1", ["num_el_in_blk1", "num_nod_per_el1"], NC_INT, conn.astype(np.int64) + 1,
        {"elem_type": (NC_CHAR, etype)})
    if nss:
        var("ss_status", ["num_side_sets"], NC_INT, np.ones(nss, int))
        var("ss_prop1", ["num_side_sets"], NC_INT, np.arange(1, nss + 1), {"name": (NC_CHAR, "ID")})
        var("ss_names", ["num_side_sets", "len_name"], NC_CHAR, _char_table(names))
        for k in range(nss):
            sel = face_bnd == k
            dims[f"num_side_ss{k + 1}"] = int(sel.sum())
            var(f"elem_ss{k + 1}", [f"num_side_ss{k + 1}"], NC_INT, np.asarray(face_elem)[sel].astype(np.int64) + 1)
            var(f"side_ss{k + 1}", [f"num_side_ss{k + 1}"], NC_INT, np.asarray(face_ord)[sel].astype(np.int64) + 1)
    if fields:
        var("name_nod_var", ["num_nod_var", "len_name"], NC_CHAR, _char_table(list(fields)))
        for k, (name, vals) in enumerate(fields.items()):
            var(f"vals_nod_var{k + 1}", ["time_step", "num_nodes"], NC_DOUBLE, np.asarray(vals, float).reshape(nsteps, nn))
    attrs = {"api_version": (NC_FLOAT, [8.0]), "version": (NC_FLOAT, [8.0]), "floating_point_word_size": (NC_INT, [8]),
             "file_size": (NC_INT, [1]), "title": (NC_CHAR, title)}
    write_netcdf(path, NcFile(dims, attrs, V, nsteps))


def read_nodal_fields(path):
    """Nodal result fields of an Exodus file: (times, {name: (num_steps, nn)})."""
    f = read_netcdf(path)
    names = _names(f, "name_nod_var")
    out = {n: f.variables[f"vals_nod_var{k + 1}"].data for k, n in enumerate(names)}
    t = f.variables["time_whole"].data if "time_whole" in f.variables else np.zeros(0)
    return t, out
