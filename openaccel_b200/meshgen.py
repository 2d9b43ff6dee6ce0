"""Seeded synthetic meshes and initial fields for the CVFEM flow workloads.

The reference reads Exodus meshes through STK; the workloads here are
generated in memory with the same element/face conventions:

* hex8 node ordering and face ordinals follow the Nalu hex8 master element
  (``external/nalu/src/master_element/Hex8CVFEM.C:415-422``): element
  ``(i, j, k)`` has nodes ``(i,j,k), (i+1,j,k), (i+1,j+1,k), (i,j+1,k)`` and the
  same four at ``k+1``; faces 0..5 are y-, x+, y+, x-, z-, z+.
* nodes are numbered lexicographically, ``id = i + (nx+1)*(j + (ny+1)*k)``,
  so CSR columns sorted by node id run -z, -y, -x, self, +x, +y, +z.
* boundary faces carry a boundary index; node-side Dirichlet values are
  applied boundary by boundary in index order, so nodes shared by two
  boundaries keep the value of the later one (the reference sets node-side
  fields part by part, ``nodeField.hpp:1224-1300``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# hex8 face ordinal -> element-local nodes (outward orientation)
HEX_FACE_NODES = np.array(
    [[0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [0, 4, 7, 3], [0, 3, 2, 1], [4, 5, 6, 7]],
    dtype=np.int32,
)


@dataclass
class HexMesh:
    """Unstructured view of a logically structured hex8 block."""

    nx: int
    ny: int
    nz: int
    coords: np.ndarray  # (nn, 3) float64
    conn: np.ndarray  # (ne, 8) int32
    face_elem: np.ndarray  # (nf,) int32
    face_ord: np.ndarray  # (nf,) int32
    face_bnd: np.ndarray  # (nf,) int32
    bnd_velocity: np.ndarray  # (nbnd, 3) float64 (no-slip wall velocity)
    meta: dict = field(default_factory=dict)

    @property
    def nn(self) -> int:
        return self.coords.shape[0]

    @property
    def ne(self) -> int:
        return self.conn.shape[0]

    @property
    def nf(self) -> int:
        return self.face_elem.shape[0]


def _node_id(i, j, k, nx, ny):
    return i + (nx + 1) * (j + (ny + 1) * k)


def hex_block(nx, ny, nz, x1d=None, y1d=None, z1d=None):
    """Nodes and connectivity of an nx*ny*nz hex8 block (lexicographic ids)."""
    x1d = np.linspace(0.0, 1.0, nx + 1) if x1d is None else np.asarray(x1d, np.float64)
    y1d = np.linspace(0.0, 1.0, ny + 1) if y1d is None else np.asarray(y1d, np.float64)
    z1d = np.linspace(0.0, 1.0, nz + 1) if z1d is None else np.asarray(z1d, np.float64)
    Z, Y, X = np.meshgrid(z1d, y1d, x1d, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).astype(np.float64)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    n0 = _node_id(i, j, k, nx, ny)
    sx, sy = 1, nx + 1
    sz = (nx + 1) * (ny + 1)
    conn = np.stack(
        [n0, n0 + sx, n0 + sx + sy, n0 + sy, n0 + sz, n0 + sz + sx, n0 + sz + sx + sy, n0 + sz + sy],
        axis=1,
    ).astype(np.int32)
    return coords, conn


def _elem_id(i, j, k, nx, ny):
    return i + nx * (j + ny * k)


def block_faces(nx, ny, nz):
    """All boundary faces of the block as (elem, ordinal, side) with side in
    {'x-','x+','y-','y+','z-','z+'}, in a fixed order (side, then element id)."""
    out = {}
    a, b = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")  # j,k for x faces
    out["x-"] = (_elem_id(0, a, b, nx, ny).ravel(), 3)
    out["x+"] = (_elem_id(nx - 1, a, b, nx, ny).ravel(), 1)
    a, b = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    out["y-"] = (_elem_id(a, 0, b, nx, ny).ravel(), 0)
    out["y+"] = (_elem_id(a, ny - 1, b, nx, ny).ravel(), 2)
    a, b = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    out["z-"] = (_elem_id(a, b, 0, nx, ny).ravel(), 4)
    out["z+"] = (_elem_id(a, b, nz - 1, nx, ny).ravel(), 5)
    return {s: (np.sort(e).astype(np.int32), o) for s, (e, o) in out.items()}


def cavity(n, perturb=0.0, seed=12345, lid_velocity=(1.0, 0.0, 0.0)):
    """Lid-driven cavity on the unit cube with n^3 hex8 elements (or nx*ny*nz
    when n is a triple).

    Boundary 0 is the lid (z = 1) moving with ``lid_velocity``; boundary 1 is
    the other five no-slip faces. Boundary 1 is applied last, so the lid's edge
    nodes carry zero wall velocity (the cavity example lists the lid first).
    ``perturb`` displaces interior nodes by U(-perturb*h, perturb*h) per
    coordinate (numpy PCG64 stream ``seed``; h = 1/n, the x spacing of a box).
    """
    nx, ny, nz = (n, n, n) if np.isscalar(n) else (int(v) for v in n)
    coords, conn = hex_block(nx, ny, nz)
    if perturb > 0.0:
        h = 1.0 / nx
        rng = np.random.Generator(np.random.PCG64(seed))
        noise = rng.uniform(-perturb * h, perturb * h, size=coords.shape)
        idx = np.arange(coords.shape[0])
        i = idx % (nx + 1)
        j = (idx // (nx + 1)) % (ny + 1)
        k = idx // ((nx + 1) * (ny + 1))
        interior = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
        coords[interior] += noise[interior]
    faces = block_faces(nx, ny, nz)
    fe, fo, fb = [], [], []
    for side in ["z+"]:
        e, o = faces[side]
        fe.append(e), fo.append(np.full_like(e, o)), fb.append(np.zeros_like(e))
    for side in ["x-", "x+", "y-", "y+", "z-"]:
        e, o = faces[side]
        fe.append(e), fo.append(np.full_like(e, o)), fb.append(np.ones_like(e))
    bnd_velocity = np.array([list(lid_velocity), [0.0, 0.0, 0.0]], dtype=np.float64)
    return HexMesh(
        nx, ny, nz, coords, conn,
        np.concatenate(fe).astype(np.int32), np.concatenate(fo).astype(np.int32),
        np.concatenate(fb).astype(np.int32), bnd_velocity,
        meta={"kind": "cavity", "n": n, "perturb": perturb, "seed": seed},
    )


def symmetry_box(n, perturb=0.0, seed=12345, lid_velocity=(1.0, 0.0, 0.0)):
    """The cavity box with its two y faces as separate boundaries, for
    symmetry planes: boundary 0 the lid (z = 1), 1 the x faces and the floor
    (no-slip), 2 the face y = 0, 3 the face y = 1. Node layout and
    ``perturb`` as in :func:`cavity` (interior nodes only, so the y faces stay
    planes)."""
    c = cavity(n, perturb=perturb, seed=seed, lid_velocity=lid_velocity)
    faces = block_faces(c.nx, c.ny, c.nz)
    fe, fo, fb = [], [], []
    for side, bnd in (("z+", 0), ("x-", 1), ("x+", 1), ("z-", 1), ("y-", 2), ("y+", 3)):
        e, o = faces[side]
        fe.append(e), fo.append(np.full_like(e, o)), fb.append(np.full_like(e, bnd))
    bnd_velocity = np.array([list(lid_velocity), [0.0] * 3, [0.0] * 3, [0.0] * 3], dtype=np.float64)
    meta = dict(c.meta, kind="symmetry_box")
    return HexMesh(c.nx, c.ny, c.nz, c.coords, c.conn, np.concatenate(fe).astype(np.int32),
                   np.concatenate(fo).astype(np.int32), np.concatenate(fb).astype(np.int32), bnd_velocity, meta=meta)


def initial_velocity(mesh: HexMesh, sigma=0.0, seed=12345):
    """Zero, or seeded Gaussian N(0, sigma^2) on interior nodes (walls keep 0)."""
    U = np.zeros((mesh.nn, 3), dtype=np.float64)
    if sigma > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed + 1))
        g = rng.normal(0.0, sigma, size=U.shape)
        if mesh.meta.get("kind") == "star":
            interior = np.ones(mesh.nn, dtype=bool)
            fn = mesh.conn[mesh.face_elem[:, None], HEX_FACE_NODES[mesh.face_ord]]
            interior[fn.ravel()] = False
        else:
            nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
            idx = np.arange(mesh.nn)
            i = idx % (nx + 1)
            j = (idx // (nx + 1)) % (ny + 1)
            k = idx // ((nx + 1) * (ny + 1))
            interior = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
        U[interior] = g[interior]
    return U


def stretched_1d(n, ratio, length=1.0):
    """n cells on [0, length], geometric growth `ratio` from both ends to the
    middle (symmetric wall-normal stretching)."""
    half = n // 2
    w = ratio ** np.arange(half)
    w = np.concatenate([w, w[::-1]]) if n % 2 == 0 else np.concatenate([w, [ratio ** half], w[::-1]])
    x = np.concatenate([[0.0], np.cumsum(w)])
    return length * x / x[-1]


def channel(nx=256, ny=96, nz=96, ratio=1.05, length=(4.0, 1.0, 1.0), perturb=0.0, seed=3):
    """Channel-shaped hex block: nx x ny x nz elements, x streamwise, y
    wall-normal with geometric stretching `ratio` from both walls, z spanwise.
    Boundary 0 is the y walls, 1 the x faces (the inlet and outlet planes,
    no-slip walls here: inlet and outlet conditions are not modelled) and 2
    the z faces (the spanwise planes, meant as symmetry planes)."""
    coords, conn = hex_block(nx, ny, nz, np.linspace(0.0, length[0], nx + 1), stretched_1d(ny, ratio, length[1]),
                             np.linspace(0.0, length[2], nz + 1))
    faces = block_faces(nx, ny, nz)
    fe, fo, fb = [], [], []
    for side, bnd in (("y-", 0), ("y+", 0), ("x-", 1), ("x+", 1), ("z-", 2), ("z+", 2)):
        e, o = faces[side]
        fe.append(e), fo.append(np.full_like(e, o)), fb.append(np.full_like(e, bnd))
    bnd_velocity = np.zeros((3, 3), dtype=np.float64)
    return HexMesh(nx, ny, nz, coords, conn, np.concatenate(fe).astype(np.int32),
                   np.concatenate(fo).astype(np.int32), np.concatenate(fb).astype(np.int32), bnd_velocity,
                   meta={"kind": "channel", "ratio": ratio})


def star_prism(blocks=3, n=6, nz=6, radius=1.0, height=1.0, perturb=0.0, seed=7, lid_velocity=(1.0, 0.0, 0.0)):
    """A hex mesh that is not one block: a regular polygon with 2*blocks
    corners split into ``blocks`` quadrilaterals that meet at its centre, each
    meshed n x n (bilinear), extruded into nz layers. Along the centre line
    ``blocks`` elements meet around every edge (3 or 5 instead of 4), so no
    consistent corner labelling exists; nodes there have 2*blocks incident
    elements (10 for 5 blocks). Lid (z = height) is boundary 0 moving with
    ``lid_velocity``, the side and bottom walls boundary 1 (applied last).
    ``perturb`` displaces nodes off every boundary by U(-perturb h, perturb h)
    per coordinate, h = radius / n."""
    nb = int(blocks)
    th = np.pi * np.arange(2 * nb) / nb
    V = radius * np.stack([np.cos(th), np.sin(th)], axis=1)
    C = np.zeros(2)
    s1 = np.linspace(0.0, 1.0, n + 1)
    # 2D nodes of every block, merged along the shared edges
    keys, pts, ids = {}, [], []
    for b in range(nb):
        q10, q11, q01 = V[(2 * b) % (2 * nb)], V[(2 * b + 1) % (2 * nb)], V[(2 * b + 2) % (2 * nb)]
        bid = np.empty((n + 1, n + 1), dtype=np.int64)
        for j, t in enumerate(s1):
            for i, sv in enumerate(s1):
                X = (1 - sv) * (1 - t) * C + sv * (1 - t) * q10 + sv * t * q11 + (1 - sv) * t * q01
                key = (round(X[0] * 1e9), round(X[1] * 1e9))
                if key not in keys:
                    keys[key] = len(pts)
                    pts.append(X)
                bid[i, j] = keys[key]
        ids.append(bid)
    P = np.array(pts)
    n2 = P.shape[0]
    z = np.linspace(0.0, height, nz + 1)
    coords = np.concatenate([np.column_stack([P, np.full(n2, zk)]) for zk in z]).astype(np.float64)
    conn, fe, fo, fb = [], [], [], []
    for b in range(nb):
        bid = ids[b]
        for k in range(nz):
            for j in range(n):
                for i in range(n):
                    q = [bid[i, j], bid[i + 1, j], bid[i + 1, j + 1], bid[i, j + 1]]
                    e = len(conn)
                    conn.append([v + k * n2 for v in q] + [v + (k + 1) * n2 for v in q])
                    if k == nz - 1:
                        fe.append(e), fo.append(5), fb.append(0)
                    if k == 0:
                        fe.append(e), fo.append(4), fb.append(1)
                    if i == n - 1:
                        fe.append(e), fo.append(1), fb.append(1)
                    if j == n - 1:
                        fe.append(e), fo.append(2), fb.append(1)
    conn = np.array(conn, dtype=np.int32)
    fe, fo, fb = (np.array(v, dtype=np.int32) for v in (fe, fo, fb))
    # lid faces first, then the walls (node-side values: the later boundary wins)
    order = np.argsort(fb, kind="stable")
    fe, fo, fb = fe[order], fo[order], fb[order]
    if perturb > 0.0:
        on_bnd = np.zeros(coords.shape[0], dtype=bool)
        on_bnd[conn[fe[:, None], HEX_FACE_NODES[fo]].ravel()] = True
        rng = np.random.Generator(np.random.PCG64(seed))
        noise = rng.uniform(-perturb * radius / n, perturb * radius / n, size=coords.shape)
        coords[~on_bnd] += noise[~on_bnd]
    bnd_velocity = np.array([list(lid_velocity), [0.0, 0.0, 0.0]], dtype=np.float64)
    return HexMesh(n, n, nz, coords, conn, fe, fo, fb, bnd_velocity,
                   meta={"kind": "star", "blocks": nb, "n": n, "nz": nz, "perturb": perturb, "seed": seed})


@dataclass
class CavityBatch:
    """Disjoint union of independent cavities (one mesh, one launch per kernel)."""

    mesh: HexMesh
    mu: np.ndarray  # (nn,) per-node viscosity (constant within each cavity)
    ref_nodes: np.ndarray  # one pressure-level node per cavity
    node_offsets: np.ndarray  # (count+1,)
    sizes: np.ndarray  # edge count of each cavity
    viscosities: np.ndarray


def batch_cavities(count=64, nmin=16, nmax=64, mu_min=1e-3, mu_max=1e-1, seed=2024, sizes=None,
                   lid_velocity=(1.0, 0.0, 0.0)):
    """Independent unit-cube cavities of uneven size (edge counts U{nmin..nmax})
    and log-uniform viscosities, concatenated node- and element-wise. Cavity m
    owns boundaries 2m (lid, z = 1) and 2m+1 (other walls), applied in that
    order so its lid-edge nodes carry zero wall velocity; its pressure-level
    node is its first node (the origin corner)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if sizes is None:
        sizes = rng.integers(nmin, nmax + 1, size=count)
    sizes = np.asarray(sizes, dtype=np.int64)
    visc = np.exp(rng.uniform(np.log(mu_min), np.log(mu_max), size=sizes.size))
    coords, conns, fe, fo, fb, mus, refs, noff = [], [], [], [], [], [], [], [0]
    eoff = 0
    for m, n in enumerate(sizes):
        c = cavity(int(n), lid_velocity=lid_velocity)
        coords.append(c.coords)
        conns.append(c.conn + noff[-1])
        fe.append(c.face_elem + eoff)
        fo.append(c.face_ord)
        fb.append(c.face_bnd + 2 * m)
        mus.append(np.full(c.nn, visc[m]))
        refs.append(noff[-1])
        noff.append(noff[-1] + c.nn)
        eoff += c.ne
    bv = np.tile(np.array([list(lid_velocity), [0.0, 0.0, 0.0]]), (sizes.size, 1))
    mesh = HexMesh(int(sizes.max()), int(sizes.max()), int(sizes.max()), np.concatenate(coords),
                   np.concatenate(conns).astype(np.int32), np.concatenate(fe).astype(np.int32),
                   np.concatenate(fo).astype(np.int32), np.concatenate(fb).astype(np.int32), bv,
                   meta={"kind": "cavity_batch", "count": int(sizes.size), "seed": seed})
    return CavityBatch(mesh, np.concatenate(mus), np.asarray(refs, np.int32), np.asarray(noff, np.int64), sizes,
                       visc)


# tet4 face ordinal -> element-local nodes, outward orientation
# (external/nalu/src/master_element/Tet4CVFEM.C:416-421)
TET_SIDE_NODES = np.array([[0, 1, 3], [1, 2, 3], [0, 3, 2], [0, 2, 1]], dtype=np.int32)

BND_FIXED_VALUE = 0
BND_ZERO_FLUX = 1


@dataclass
class TetMesh:
    """tet4 mesh with boundary faces (element, face ordinal, boundary index)."""

    n: int
    coords: np.ndarray  # (nn, 3) float64
    conn: np.ndarray  # (ne, 4) int32
    face_elem: np.ndarray
    face_ord: np.ndarray
    face_bnd: np.ndarray
    bnd_kind: np.ndarray  # (nbnd,) BND_FIXED_VALUE / BND_ZERO_FLUX
    bnd_value: np.ndarray  # (nbnd,) fixed values
    meta: dict = field(default_factory=dict)

    @property
    def nn(self) -> int:
        return self.coords.shape[0]

    @property
    def ne(self) -> int:
        return self.conn.shape[0]

    @property
    def nf(self) -> int:
        return self.face_elem.shape[0]


def kuhn_tets(n, perturb=0.0, seed=12345):
    """n^3 hex block on the unit cube, each hex split into the 6 Kuhn tets that
    share its (0,0,0)-(1,1,1) diagonal, so face diagonals match between
    neighbours. Node numbering as ``hex_block``; tet nodes are ordered for a
    positive Jacobian. Returns (coords, conn)."""
    coords, _ = hex_block(n, n, n)
    if perturb > 0.0:
        h = 1.0 / n
        rng = np.random.Generator(np.random.PCG64(seed))
        noise = rng.uniform(-perturb * h, perturb * h, size=coords.shape)
        idx = np.arange(coords.shape[0])
        i, j, k = idx % (n + 1), (idx // (n + 1)) % (n + 1), idx // ((n + 1) * (n + 1))
        interior = (i > 0) & (i < n) & (j > 0) & (j < n) & (k > 0) & (k < n)
        coords[interior] += noise[interior]
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    n0 = _node_id(i.ravel(), j.ravel(), k.ravel(), n, n).astype(np.int64)
    stride = np.array([1, n + 1, (n + 1) * (n + 1)], dtype=np.int64)
    tets = []
    for perm, sign in [((0, 1, 2), 1), ((1, 2, 0), 1), ((2, 0, 1), 1),
                       ((0, 2, 1), -1), ((2, 1, 0), -1), ((1, 0, 2), -1)]:
        p0 = n0
        p1 = p0 + stride[perm[0]]
        p2 = p1 + stride[perm[1]]
        p3 = n0 + stride.sum()
        tets.append(np.stack([p0, p1, p2, p3] if sign > 0 else [p0, p2, p1, p3], axis=1))
    conn = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int32)
    return coords, conn


def tet_boundary_faces(n, conn):
    """Boundary faces of a ``kuhn_tets`` block by side: {'x-': (elems, ords), ...},
    each sorted by (element, ordinal)."""
    nodes = conn[:, TET_SIDE_NODES]  # (ne, 4, 3)
    i = nodes % (n + 1)
    j = (nodes // (n + 1)) % (n + 1)
    k = nodes // ((n + 1) * (n + 1))
    out = {}
    for side, arr, val in [("x-", i, 0), ("x+", i, n), ("y-", j, 0), ("y+", j, n), ("z-", k, 0), ("z+", k, n)]:
        e, o = np.nonzero(np.all(arr == val, axis=2))
        out[side] = (e.astype(np.int32), o.astype(np.int32))
    return out


def conduction(n, sigma=1.0, seed=4242, perturb=0.0, t_left=0.0, t_right=1.0):
    """Steady heat conduction on the unit cube split into 6 n^3 tets.

    Boundary 0 (x = 0) holds ``t_left``, boundary 1 (x = 1) holds ``t_right``,
    boundary 2 (the other four faces) is zero-flux. Conductivity is lognormal
    per element (median 1, ``sigma``), projected to nodes as the
    volume-weighted mean of the adjacent elements (the reference keeps the
    diffusivity at nodes); the volumetric source is U[0, 1] per node. Returns
    (TetMesh, gamma_node, source_node, gamma_elem)."""
    coords, conn = kuhn_tets(n, perturb=perturb, seed=seed)
    faces = tet_boundary_faces(n, conn)
    fe, fo, fb = [], [], []
    for bnd, sides in enumerate([["x-"], ["x+"], ["y-", "y+", "z-", "z+"]]):
        for s in sides:
            e, o = faces[s]
            fe.append(e), fo.append(o), fb.append(np.full_like(e, bnd))
    mesh = TetMesh(n, coords, conn, np.concatenate(fe), np.concatenate(fo), np.concatenate(fb),
                   np.array([BND_FIXED_VALUE, BND_FIXED_VALUE, BND_ZERO_FLUX], np.int32),
                   np.array([t_left, t_right, 0.0]),
                   meta={"kind": "conduction", "n": n, "sigma": sigma, "seed": seed, "perturb": perturb})
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    gamma_e = np.exp(sigma * rng.standard_normal(conn.shape[0]))
    x = coords[conn]  # (ne, 4, 3)
    vol_e = np.einsum("ij,ij->i", x[:, 1] - x[:, 0], np.cross(x[:, 2] - x[:, 0], x[:, 3] - x[:, 0])) / 6.0
    flat = conn.ravel()
    wsum = np.bincount(flat, weights=np.repeat(vol_e, 4), minlength=coords.shape[0])
    gsum = np.bincount(flat, weights=np.repeat(vol_e * gamma_e, 4), minlength=coords.shape[0])
    gamma_n = gsum / wsum
    src = rng.uniform(0.0, 1.0, size=coords.shape[0])
    return mesh, gamma_n, src, gamma_e
