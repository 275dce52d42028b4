"""Q1 meshes for the particle path: generators, a UNV reader and vertex maps.

A mesh is the flat data the particle handler needs from deal.II's
Triangulation/DoFHandler (reference: ``src/pfem2particlehandler.cpp:84-92``
iterates active cells, ``src/pfem2particle.cpp:83-87`` copies
``cell->vertex_dof_index(i, 0)``):

* ``vertices``   (n_verts, dim) float64
* ``cells``      (n_cells, 2**dim) int32, deal.II lexicographic vertex order
  (vertex i sits at reference corner ((i>>0)&1, (i>>1)&1, (i>>2)&1))
* ``cell_dofs``  (n_cells, 2**dim) int32, the Q1 DoF of each cell vertex
* ``n_dofs``

The generators number cells and vertices the way
``GridGenerator::subdivided_hyper_rectangle`` does (x fastest), which is the
mesh of ``cases/PoiseuilleFlow3D/PoiseuilleFlow3D.cc:27-30``.
"""
from __future__ import annotations

import dataclasses
import io
import os
import tarfile

import numpy as np


@dataclasses.dataclass
class Mesh:
    dim: int
    vertices: np.ndarray
    cells: np.ndarray
    cell_dofs: np.ndarray
    n_dofs: int
    name: str = ""

    @property
    def n_cells(self) -> int:
        return int(self.cells.shape[0])

    @property
    def n_verts(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def nv(self) -> int:
        return 1 << self.dim

    def dof_coordinates(self) -> np.ndarray:
        """Coordinates of every DoF (the vertex it sits on)."""
        out = np.zeros((self.n_dofs, self.dim))
        out[self.cell_dofs.ravel()] = self.vertices[self.cells.ravel()]
        return out

    def renumber_dofs_first_touch(self) -> "Mesh":
        """DoFs numbered by first appearance in cell order, as a DoFHandler
        distributes them, instead of by vertex index."""
        order = {}
        flat = self.cells.ravel()
        perm = np.full(self.n_verts, -1, np.int64)
        nxt = 0
        for v in flat:
            if perm[v] < 0:
                perm[v] = nxt
                nxt += 1
        del order
        dofs = perm[self.cells].astype(np.int32)
        return dataclasses.replace(self, cell_dofs=dofs, n_dofs=int(nxt))


def _lex_cells(n):
    """Cells of a structured grid with n = (nx, ny[, nz]) cells, x fastest,
    vertex ids of a (nx+1)(ny+1)(nz+1) lattice, deal.II vertex order."""
    dim = len(n)
    nvx = [k + 1 for k in n]
    idx = np.indices(n[::-1]).reshape(dim, -1)[::-1]  # idx[d] = cell index along d, x fastest
    cells = np.zeros((idx.shape[1], 1 << dim), np.int64)
    for i in range(1 << dim):
        vid = np.zeros(idx.shape[1], np.int64)
        stride = 1
        for d in range(dim):
            vid += (idx[d] + ((i >> d) & 1)) * stride
            stride *= nvx[d]
        cells[:, i] = vid
    return cells.astype(np.int32)


def hyper_rectangle(p0, p1, reps, name="box") -> Mesh:
    """GridGenerator::subdivided_hyper_rectangle equivalent."""
    dim = len(reps)
    axes = [np.linspace(p0[d], p1[d], reps[d] + 1) for d in range(dim)]
    grid = np.meshgrid(*axes[::-1], indexing="ij")[::-1]
    verts = np.stack([g.ravel() for g in grid], axis=1).astype(np.float64)
    cells = _lex_cells(list(reps))
    return Mesh(dim, verts, cells, cells.copy(), verts.shape[0], name)


def perturbed_cube(n, length=2 * np.pi, amplitude=0.1, seed=0, name="perturbed_cube") -> Mesh:
    """n^3 hexes on [0, length]^3; interior vertices moved uniformly by up to
    +-amplitude*h per axis with numpy's PCG64 seeded by ``seed``."""
    m = hyper_rectangle((0.0, 0.0, 0.0), (length,) * 3, (n, n, n), name)
    h = length / n
    rng = np.random.default_rng(seed)
    v = m.vertices
    interior = np.all((v > 0.5 * h) & (v < length - 0.5 * h), axis=1)
    shift = rng.uniform(-amplitude * h, amplitude * h, size=v.shape)
    v = v.copy()
    v[interior] += shift[interior]
    return dataclasses.replace(m, vertices=v)


def _orient(dim, verts, cells):
    """Make every cell right-handed (positive Jacobian at its centre) by
    swapping the xi and eta directions of left-handed cells."""
    X = verts[cells]  # (nC, nv, dim)
    if dim == 2:
        e = (X[:, 1] + X[:, 3] - X[:, 0] - X[:, 2]) * 0.5
        f = (X[:, 2] + X[:, 3] - X[:, 0] - X[:, 1]) * 0.5
        det = e[:, 0] * f[:, 1] - e[:, 1] * f[:, 0]
        bad = det < 0
        cells[bad] = cells[bad][:, [0, 2, 1, 3]]
    else:
        J = np.zeros((cells.shape[0], 3, 3))
        for k in range(3):
            hi = [i for i in range(8) if (i >> k) & 1]
            lo = [i for i in range(8) if not (i >> k) & 1]
            J[:, :, k] = (X[:, hi].sum(1) - X[:, lo].sum(1)) / 4
        bad = np.linalg.det(J) < 0
        cells[bad] = cells[bad][:, [0, 2, 1, 3, 4, 6, 5, 7]]
    return cells


def turek_channel(n_t=96, n_r=48, n_x=480, name="turek_channel") -> Mesh:
    """Synthetic stand-in for the Turek benchmark mesh (channel
    [0,2.2]x[0,0.41], cylinder of radius 0.05 centred at (0.2,0.2); the
    reference's ``cases/TurekBenchmark`` meshes): an O-grid of 4*n_t*n_r
    curved quads between the cylinder and the square [0,0.41]^2, graded
    towards the wall, plus an n_x x n_t block downstream.  Default size
    64,512 quads; cells are non-affine."""
    L, H = 2.2, 0.41
    cx, cy, r = 0.2, 0.2, 0.05
    s = H
    # square boundary points, counter-clockwise starting at the lower-right
    # corner, n_t segments per side
    t = np.linspace(0.0, 1.0, n_t + 1)
    sides = [
        np.stack([np.full_like(t, s), t * s], 1),            # right: (s,0)->(s,s)
        np.stack([s - t * s, np.full_like(t, s)], 1),        # top: (s,s)->(0,s)
        np.stack([np.zeros_like(t), s - t * s], 1),          # left: (0,s)->(0,0)
        np.stack([t * s, np.zeros_like(t)], 1),              # bottom: (0,0)->(s,0)
    ]
    outer = np.concatenate([sd[:-1] for sd in sides], 0)  # 4 n_t points
    ang0 = np.arctan2(outer[:, 1] - cy, outer[:, 0] - cx)
    # circle points at the angles of the square points (monotone around)
    inner = np.stack([cx + r * np.cos(ang0), cy + r * np.sin(ang0)], 1)
    nring = outer.shape[0]
    # radial grading: geometric clustering at the wall
    g = np.linspace(0.0, 1.0, n_r + 1) ** 1.6
    ring = inner[None, :, :] * (1 - g)[:, None, None] + outer[None, :, :] * g[:, None, None]
    verts = [ring.reshape(-1, 2)]
    nid = lambda k, j: k * nring + (j % nring)
    cells = []
    for k in range(n_r):
        for j in range(nring):
            cells.append([nid(k, j), nid(k + 1, j), nid(k, j + 1), nid(k + 1, j + 1)])
    base = (n_r + 1) * nring
    # downstream block: columns x_1..x_nx (x_0 = s is the ring's right side)
    xs = s + (L - s) * np.linspace(0.0, 1.0, n_x + 1)[1:]
    ys = np.linspace(0.0, s, n_t + 1)
    bx, by = np.meshgrid(xs, ys, indexing="ij")
    verts.append(np.stack([bx.ravel(), by.ravel()], 1))
    right_ring = [nid(n_r, j) for j in range(n_t + 1)]  # j=0..n_t: (s,0)..(s,s)
    right_ring[n_t] = nid(n_r, n_t)

    def bid(i, j):  # i = column 0..n_x, j = row 0..n_t
        if i == 0:
            return right_ring[j]
        return base + (i - 1) * (n_t + 1) + j

    for i in range(n_x):
        for j in range(n_t):
            cells.append([bid(i, j), bid(i + 1, j), bid(i, j + 1), bid(i + 1, j + 1)])
    V = np.concatenate(verts, 0).astype(np.float64)
    C = np.asarray(cells, np.int32)
    C = _orient(2, V, C)
    return Mesh(2, V, C, C.copy(), V.shape[0], name)


def read_unv(src, dim=None) -> Mesh:
    """Read an I-DEAS universal mesh as GridIn::read_unv does for the
    reference (``src/pfem2solver.cpp:116-119``): dataset 2411 gives the nodes,
    2412 the elements (type 44 quads and 115 hexes become cells, type 11
    edges and 2467 groups are boundary data the particle path ignores).
    Node order of a UNV quad/hex is counter-clockwise per face; it is mapped
    to deal.II's lexicographic order and left-handed cells are flipped.
    Unused nodes are dropped.  ``src`` is a path, a text stream, or a .tgz
    archive path holding one .unv file."""
    if isinstance(src, (str, os.PathLike)):
        p = os.fspath(src)
        if p.endswith((".tgz", ".tar.gz")):
            with tarfile.open(p) as tf:
                mem = [m for m in tf.getmembers() if m.name.endswith(".unv")][0]
                text = tf.extractfile(mem).read().decode()
        else:
            with open(p) as f:
                text = f.read()
    else:
        text = src.read()
    lines = text.splitlines()
    i = 0
    nodes = {}
    elems = []
    n = len(lines)
    while i < n:
        tok = lines[i].strip()
        if tok == "-1" and i + 1 < n:
            ds = lines[i + 1].strip()
            i += 2
            if ds == "2411":
                while lines[i].strip() != "-1":
                    lab = int(lines[i].split()[0])
                    xyz = [float(w.replace("D", "E")) for w in lines[i + 1].split()]
                    nodes[lab] = xyz
                    i += 2
            elif ds == "2412":
                while lines[i].strip() != "-1":
                    head = lines[i].split()
                    etype = int(head[1])
                    nnode = int(head[5])
                    i += 1
                    if etype in (11, 21, 22, 24):  # beam-like: extra record line
                        i += 1
                    conn = []
                    while len(conn) < nnode:
                        conn += [int(w) for w in lines[i].split()]
                        i += 1
                    if etype in (44, 94, 115):
                        elems.append((etype, conn))
            else:
                while i < n and lines[i].strip() != "-1":
                    i += 1
            i += 1  # closing -1
            continue
        i += 1
    if not elems:
        raise ValueError("UNV file has no quad (44) or hex (115) elements")
    etype0 = elems[0][0]
    edim = 3 if etype0 == 115 else 2
    dim = dim or edim
    if dim != edim:
        raise ValueError(f"UNV elements are {edim}D, asked for {dim}D")
    ucd_to_lex = [0, 1, 3, 2] if dim == 2 else [0, 1, 3, 2, 4, 5, 7, 6]
    conn = np.asarray([c for t, c in elems if (t == 115) == (dim == 3)], np.int64)
    conn = conn[:, ucd_to_lex]
    used = np.unique(conn)
    labmap = {lab: k for k, lab in enumerate(used)}
    verts = np.asarray([nodes[lab][:dim] for lab in used], np.float64)
    cells = np.vectorize(labmap.__getitem__)(conn).astype(np.int32)
    cells = _orient(dim, verts, cells)
    return Mesh(dim, verts, cells, cells.copy(), verts.shape[0], "unv")


def read_unv_native(src, dim=None) -> Mesh:
    """read_unv through the library's C++ reader (pfem2gpu_read_unv, host
    only): the same mesh, for large files.  ``src`` is a .unv path or a .tgz
    archive holding one (extracted to a temporary file first)."""
    import ctypes as C
    import tempfile

    from . import _lib

    L = _lib.load()
    p = os.fspath(src)
    tmp = None
    if p.endswith((".tgz", ".tar.gz")):
        with tarfile.open(p) as tf:
            mem = [m for m in tf.getmembers() if m.name.endswith(".unv")][0]
            tmp = tempfile.NamedTemporaryFile(suffix=".unv", delete=False)
            tmp.write(tf.extractfile(mem).read())
            tmp.close()
            p = tmp.name
    try:
        nv, nc, dd = C.c_int64(), C.c_int64(), C.c_int32()
        path = p.encode()
        rc = L.pfem2gpu_read_unv(path, int(dim or 0), C.byref(dd), C.byref(nv), C.byref(nc), None, None, 0, 0)
        if rc != _lib.OK:
            raise ValueError(L.pfem2gpu_read_unv_error().decode())
        d = dd.value
        verts = np.empty((nv.value, d), np.float64)
        cells = np.empty((nc.value, 1 << d), np.int32)
        rc = L.pfem2gpu_read_unv(path, d, None, C.byref(nv), C.byref(nc), verts.ctypes.data_as(C.c_void_p),
                                 cells.ctypes.data_as(C.c_void_p), nv.value, nc.value)
        if rc != _lib.OK:
            raise ValueError(L.pfem2gpu_read_unv_error().decode())
    finally:
        if tmp is not None:
            os.unlink(tmp.name)
    return Mesh(d, verts, cells, cells.copy(), verts.shape[0], "unv")


def boundary_face_ids(mesh: Mesh, classify=None) -> np.ndarray:
    """Per cell and face (deal.II face numbering: face 2d has xi_d = 0, face
    2d+1 has xi_d = 1), the boundary id of a face no other cell shares, -1
    for interior faces.  ``classify(centre) -> id`` names the boundary part
    from the face centre; by default the id is the face number of the
    bounding box side the face lies on (as GridGenerator::hyper_rectangle
    with colorize), or 2*dim for a face inside the box (an obstacle)."""
    dim, nv = mesh.dim, mesh.nv
    faces = {}
    keys = np.zeros((mesh.n_cells, 2 * dim), dtype=object)
    for f in range(2 * dim):
        d, side = f // 2, f % 2
        loc = [i for i in range(nv) if ((i >> d) & 1) == side]
        fv = np.sort(mesh.cells[:, loc], axis=1)
        for c in range(mesh.n_cells):
            k = tuple(fv[c])
            keys[c, f] = k
            faces[k] = faces.get(k, 0) + 1
    lo, hi = mesh.vertices.min(0), mesh.vertices.max(0)
    span = np.maximum(hi - lo, 1e-300)
    out = np.full((mesh.n_cells, 2 * dim), -1, np.int32)
    for c in range(mesh.n_cells):
        for f in range(2 * dim):
            if faces[keys[c, f]] != 1:
                continue
            centre = mesh.vertices[list(keys[c, f])].mean(0)
            if classify is not None:
                out[c, f] = int(classify(centre))
                continue
            bid = 2 * dim
            for d in range(dim):
                if abs(centre[d] - lo[d]) <= 1e-9 * span[d]:
                    bid = 2 * d
                elif abs(centre[d] - hi[d]) <= 1e-9 * span[d]:
                    bid = 2 * d + 1
            out[c, f] = bid
    return out


def write_unv(mesh: Mesh, stream: io.TextIOBase):
    """Write a mesh as UNV datasets 2411/2412 (nodes and quad/hex cells)."""
    lex_to_ucd = [0, 1, 3, 2] if mesh.dim == 2 else [0, 1, 3, 2, 4, 5, 7, 6]
    w = stream.write
    w("    -1\n  2411\n")
    for k, x in enumerate(mesh.vertices):
        xyz = list(x) + [0.0] * (3 - mesh.dim)
        w(f"{k + 1:10d}         1         1        11\n")
        w("".join(f"{c:25.16E}" for c in xyz) + "\n")
    w("    -1\n    -1\n  2412\n")
    et = 44 if mesh.dim == 2 else 115
    for k, c in enumerate(mesh.cells):
        w(f"{k + 1:10d}{et:10d}         2         1         7{mesh.nv:10d}\n")
        w("".join(f"{int(c[j]) + 1:10d}" for j in lex_to_ucd) + "\n")
    w("    -1\n")


def vertex_maps(mesh: Mesh):
    """GridTools::vertex_to_cell_map and vertex_to_cell_centers_directions as
    used by ``initialize_maps`` (``src/pfem2particlehandler.cpp:320-324``):
    CSR offsets (n_verts+1), adjacent cells ascending, and the unit vector
    from the vertex to each adjacent cell's vertex-average centre, evaluated
    in vertex order so the values are reproducible bit for bit."""
    nC, nv, dim = mesh.n_cells, mesh.nv, mesh.dim
    pairs = np.stack([mesh.cells.ravel().astype(np.int64), np.repeat(np.arange(nC), nv)], 1)
    pairs = np.unique(pairs, axis=0)  # sorted by (vertex, cell); drops repeats
    counts = np.bincount(pairs[:, 0], minlength=mesh.n_verts)
    offsets = np.zeros(mesh.n_verts + 1, np.int64)
    np.cumsum(counts, out=offsets[1:])
    cells = pairs[:, 1]
    X = mesh.vertices
    ctr = np.zeros((nC, dim))
    for i in range(nv):
        ctr = ctr + X[mesh.cells[:, i]]
    ctr = ctr / float(nv)
    dirs = ctr[cells] - X[pairs[:, 0]]
    s = np.zeros(dirs.shape[0])
    for d in range(dim):
        s = s + dirs[:, d] * dirs[:, d]
    dirs = dirs / np.sqrt(s)[:, None]
    return offsets.astype(np.int32), cells.astype(np.int32), np.ascontiguousarray(dirs)


# --------------------------------------------------------------------------
# Velocity fields sampled at DoFs, component-major (one vector per component,
# like the reference's std::array<TrilinosWrappers::MPI::Vector, dim>).
# --------------------------------------------------------------------------

def field_at_dofs(mesh: Mesh, fn) -> np.ndarray:
    xy = mesh.dof_coordinates()
    u = np.asarray(fn(xy), np.float64)
    return np.ascontiguousarray(u.T.reshape(mesh.dim, mesh.n_dofs))


def channel_profile(umax=1.0, height=1.0):
    """u = 4 umax y (H - y) / H^2, v = 0 (zero on the walls)."""
    def fn(x):
        u = np.zeros_like(x)
        u[:, 0] = 4.0 * umax * x[:, 1] * (height - x[:, 1]) / (height * height)
        return u
    return fn


def duct_profile(umax=1.0):
    """u = 16 umax y(1-y) z(1-z) on the unit cross-section, v = w = 0."""
    def fn(x):
        u = np.zeros_like(x)
        u[:, 0] = 16.0 * umax * x[:, 1] * (1 - x[:, 1]) * x[:, 2] * (1 - x[:, 2])
        return u
    return fn


def taylor_green_3d():
    """u = (sin x cos y cos z, -cos x sin y cos z, 0): divergence-free."""
    def fn(x):
        u = np.zeros_like(x)
        u[:, 0] = np.sin(x[:, 0]) * np.cos(x[:, 1]) * np.cos(x[:, 2])
        u[:, 1] = -np.cos(x[:, 0]) * np.sin(x[:, 1]) * np.cos(x[:, 2])
        return u
    return fn


def cylinder_inflow(umax=1.5, height=0.41, center=(0.2, 0.2), radius=0.05):
    """Parabolic channel profile (``cases/TurekBenchmark/TurekBenchmark.cc:6-9``)
    set to zero inside and on the cylinder."""
    def fn(x):
        u = channel_profile(umax, height)(x)
        rr = (x[:, 0] - center[0]) ** 2 + (x[:, 1] - center[1]) ** 2
        u[rr <= radius * radius * (1 + 1e-9)] = 0.0
        return u
    return fn
