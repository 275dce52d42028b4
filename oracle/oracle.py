"""ctypes wrapper of the FP64 oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline leg.  The product never imports it.
PARITY UNPINNED: see pfem2_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")

ORDER_ID = 0
ORDER_VECTOR = 1
EULER = 0  # sub-step integrators (orc_params.integrator)
RK2 = 1


class Params(C.Structure):
    _fields_ = [
        ("q", C.c_int32 * 3),
        ("max_per_part", C.c_int32),
        ("substeps", C.c_int32),
        ("dt", C.c_double),
        ("removal_order", C.c_int32),
        ("removal_seed", C.c_uint32),
        ("n_threads", C.c_int32),
        ("integrator", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int64),
        ("lost", C.c_int64),
        ("removed", C.c_int64),
        ("seeded", C.c_int64),
        ("map_failures", C.c_int64),
        ("near_face", C.c_int64),
        ("searched", C.c_int64),
        ("nan_dofs", C.c_int64),
        ("next_id", C.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        P = C.c_void_p
        dp = np.ctypeslib.ndpointer(np.float64, flags="C")
        ip = np.ctypeslib.ndpointer(np.int32, flags="C")
        up = np.ctypeslib.ndpointer(np.uint32, flags="C")
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int, C.POINTER(Params)]
        L.orc_destroy.argtypes = [P]
        L.orc_set_mesh.argtypes = [P, C.c_int64, C.c_int64, C.c_int64, dp, ip, ip]
        L.orc_vertex_map_size.restype = C.c_int64
        L.orc_vertex_map_size.argtypes = [P]
        L.orc_get_vertex_maps.argtypes = [P, ip, ip, dp]
        for f in (L.orc_seed, L.orc_move, L.orc_project):
            f.argtypes = [P, dp]
        L.orc_correct.argtypes = [P, dp, dp]
        L.orc_n_particles.restype = C.c_int64
        L.orc_n_particles.argtypes = [P]
        L.orc_get_particles.argtypes = [P, up, ip, dp, dp, dp]
        L.orc_set_particles.argtypes = [P, C.c_int64, up, ip, dp, dp, dp, C.c_uint32]
        L.orc_get_stats.argtypes = [P, C.POINTER(Stats)]
        L.orc_reset_stats.argtypes = [P]
        L.orc_shape_values.argtypes = [C.c_int, dp, dp]
        L.orc_forward_map.argtypes = [C.c_int, dp, dp, dp]
        L.orc_inverse_map.argtypes = [C.c_int, dp, dp, dp]
        L.orc_window_forward.argtypes = [P, C.c_int, dp, P, P, C.c_int, dp]
        L.orc_window_particles.argtypes = [P, C.c_int, dp, P, P, ip, dp, dp, dp]
        L.orc_window_adjoint.argtypes = [P, C.c_int, dp, P, P, C.c_int, dp, P, P, P, P]
        L.orc_key.restype = C.c_uint32
        L.orc_key.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_fem_pattern.restype = C.c_int64
        L.orc_fem_pattern.argtypes = [C.c_int, C.c_int64, C.c_int64, ip, P, P]
        L.orc_fem_assemble.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int64, dp, ip, ip, ip, C.c_double,
                                       C.c_double, C.c_double, P, P, P, P, dp, dp]
        L.orc_fem_velocity_bc.argtypes = [C.c_int, C.c_int64, C.c_int64, dp, ip, ip, C.c_int, ip, C.c_int, ip, dp,
                                          C.c_double, C.c_double, dp, ip, dp]
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """FP64 restatement of pfem2ParticleHandler (src/pfem2particlehandler.h:17-71)."""

    def __init__(self, mesh, q, max_per_part, substeps, dt, removal_order=ORDER_ID, removal_seed=0,
                 n_threads=1, integrator=EULER):
        self.L = lib()
        self.dim = mesh.dim
        p = Params()
        for d in range(3):
            p.q[d] = q[d] if d < len(q) else 1
        p.max_per_part = max_per_part
        p.substeps = substeps
        p.dt = dt
        p.removal_order = removal_order
        p.removal_seed = removal_seed
        p.n_threads = n_threads
        p.integrator = integrator
        self.h = self.L.orc_create(self.dim, C.byref(p))
        if not self.h:
            raise ValueError("orc_create failed")
        self.mesh = mesh
        rc = self.L.orc_set_mesh(self.h, mesh.n_cells, mesh.n_verts, mesh.n_dofs, _c(mesh.vertices, np.float64),
                                 _c(mesh.cells, np.int32), _c(mesh.cell_dofs, np.int32))
        if rc:
            raise ValueError(f"orc_set_mesh failed: {rc}")

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def vertex_maps(self):
        tot = self.L.orc_vertex_map_size(self.h)
        off = np.zeros(self.mesh.n_verts + 1, np.int32)
        cells = np.zeros(max(tot, 1), np.int32)
        dirs = np.zeros((max(tot, 1), self.dim))
        self.L.orc_get_vertex_maps(self.h, off, cells, dirs)
        return off, cells[:tot], dirs[:tot]

    def _V(self, V):
        return _c(V, np.float64).reshape(-1)

    def seed(self, V):
        assert self.L.orc_seed(self.h, self._V(V)) == 0

    def correct(self, V, Vold):
        assert self.L.orc_correct(self.h, self._V(V), self._V(Vold)) == 0

    def move(self, V):
        assert self.L.orc_move(self.h, self._V(V)) == 0

    def project(self):
        out = np.zeros(self.dim * self.mesh.n_dofs)
        assert self.L.orc_project(self.h, out) == 0
        return out.reshape(self.dim, self.mesh.n_dofs)

    def step(self, V, Vold):
        self.correct(V, Vold)
        self.move(V)
        return self.project()

    def particles(self):
        n = self.L.orc_n_particles(self.h)
        ids = np.zeros(n, np.uint32)
        cell = np.zeros(n, np.int32)
        x = np.zeros((n, self.dim))
        xi = np.zeros((n, self.dim))
        v = np.zeros((n, self.dim))
        self.L.orc_get_particles(self.h, ids, cell, x, xi, v)
        return {"id": ids, "cell": cell, "x": x, "xi": xi, "v": v}

    def set_particles(self, P, next_id):
        n = len(P["id"])
        assert self.L.orc_set_particles(self.h, n, _c(P["id"], np.uint32), _c(P["cell"], np.int32),
                                        _c(P["x"], np.float64), _c(P["xi"], np.float64),
                                        _c(P["v"], np.float64), next_id) == 0

    def window_forward(self, K, V, Vold=None, v0=None, empty_policy=0):
        """K steps of correct (Vold given) + move without count correction
        from the current particles, then the projection; particles unchanged."""
        U = np.zeros(self.dim * self.mesh.n_dofs)
        vo = _c(Vold, np.float64) if Vold is not None else None
        v0c = _c(v0, np.float64) if v0 is not None else None
        rc = self.L.orc_window_forward(self.h, K, self._V(V), _vp(vo), _vp(v0c), empty_policy, U)
        assert rc == 0
        return U.reshape(self.dim, self.mesh.n_dofs)

    def window_particles(self, K, V, Vold=None, v0=None):
        """Final particle states of the window (cell -1: deleted), oracle order."""
        n = self.L.orc_n_particles(self.h)
        cell = np.zeros(max(n, 1), np.int32)
        x, xi, v = (np.zeros((max(n, 1), self.dim)) for _ in range(3))
        vo = _c(Vold, np.float64) if Vold is not None else None
        v0c = _c(v0, np.float64) if v0 is not None else None
        assert self.L.orc_window_particles(self.h, K, self._V(V), _vp(vo), _vp(v0c), cell, x, xi, v) == 0
        return {"cell": cell[:n], "x": x[:n], "xi": xi[:n], "v": v[:n]}

    def window_adjoint(self, K, V, gU, Vold=None, v0=None, empty_policy=0):
        """Forward + adjoint of the window: (U, g_v0 (n x dim), g_V, g_Vold)."""
        n = self.L.orc_n_particles(self.h)
        nd = self.dim * self.mesh.n_dofs
        U, gv0, gV, gVo = np.zeros(nd), np.zeros(max(n, 1) * self.dim), np.zeros(nd), np.zeros(nd)
        vo = _c(Vold, np.float64) if Vold is not None else None
        v0c = _c(v0, np.float64) if v0 is not None else None
        g = _c(gU, np.float64).reshape(-1)
        rc = self.L.orc_window_adjoint(self.h, K, self._V(V), _vp(vo), _vp(v0c), empty_policy, g,
                                       _vp(U), _vp(gv0), _vp(gV), _vp(gVo))
        assert rc == 0
        sh = (self.dim, self.mesh.n_dofs)
        return U.reshape(sh), gv0[: n * self.dim].reshape(n, self.dim), gV.reshape(sh), gVo.reshape(sh)

    def stats(self):
        s = Stats()
        self.L.orc_get_stats(self.h, C.byref(s))
        return s.as_dict()

    def reset_stats(self):
        self.L.orc_reset_stats(self.h)


def shape_values(dim, xi):
    N = np.zeros(1 << dim)
    lib().orc_shape_values(dim, _c(xi, np.float64), N)
    return N


def _pad(X, dim):
    Xp = np.zeros((1 << dim, 3))
    Xp[:, :dim] = X
    return Xp.reshape(-1)


def forward_map(X, xi):
    dim = X.shape[1]
    out = np.zeros(dim)
    lib().orc_forward_map(dim, _pad(X, dim), _c(xi, np.float64), out)
    return out


def inverse_map(X, p):
    dim = X.shape[1]
    out = np.zeros(dim)
    rc = lib().orc_inverse_map(dim, _pad(X, dim), _c(p, np.float64), out)
    return (out if rc == 0 else None)


def key(i, seed):
    return lib().orc_key(i, seed)


# --------------------------------------------------------------------------
# FEM systems' volume terms (src/pfem2fem.cpp:247-510), restated in
# fem_oracle.c: the checker of the library's device assembly.
# --------------------------------------------------------------------------
FEM_PREDICTION, FEM_PRESSURE, FEM_CORRECTION = 0, 1, 2


def fem_pattern(mesh):
    """CSR pattern (row_ptr, cols) of the Q1 DoF adjacency, columns ascending."""
    L = lib()
    cd = _c(mesh.cell_dofs, np.int32)
    nnz = L.orc_fem_pattern(mesh.dim, mesh.n_cells, mesh.n_dofs, cd, None, None)
    row_ptr = np.zeros(mesh.n_dofs + 1, np.int32)
    cols = np.zeros(max(nnz, 1), np.int32)
    L.orc_fem_pattern(mesh.dim, mesh.n_cells, mesh.n_dofs, cd, row_ptr.ctypes.data_as(C.c_void_p),
                      cols.ctypes.data_as(C.c_void_p))
    return row_ptr, cols[:nnz]


def fem_face_mask(face_ids, velocity_dirichlet=(), pressure_dirichlet=()):
    """Per cell: bit f = boundary face f outside the velocity Dirichlet set,
    bit 8 + f = outside the pressure Dirichlet set."""
    fid = np.asarray(face_ids)
    mask = np.zeros(fid.shape[0], np.uint16)
    for f in range(fid.shape[1]):
        b = fid[:, f] >= 0
        mask |= ((b & ~np.isin(fid[:, f], list(velocity_dirichlet))).astype(np.uint16) << f)
        mask |= ((b & ~np.isin(fid[:, f], list(pressure_dirichlet))).astype(np.uint16) << (8 + f))
    return mask


def fem_assemble(mesh, system, rho, mu, dt, U=None, U2=None, P=None, pattern=None, face_mask=None):
    """(A, rhs): A (matrices, nnz) on the pattern, rhs (right-hand sides, n_dofs)."""
    L = lib()
    row_ptr, cols = pattern if pattern is not None else fem_pattern(mesh)
    nnz = int(row_ptr[-1])
    nm = mesh.dim if system == FEM_PREDICTION else 1
    ns = 1 if system == FEM_PRESSURE else mesh.dim
    A = np.zeros((nm, nnz))
    rhs = np.zeros((ns, mesh.n_dofs))
    cellX = _c(mesh.vertices[mesh.cells], np.float64)
    keep = [None if a is None else _c(a, np.float64) for a in (U, U2, P)]
    fm = None if face_mask is None else _c(face_mask, np.uint16)
    rc = L.orc_fem_assemble(mesh.dim, system, mesh.n_cells, mesh.n_dofs, cellX, _c(mesh.cell_dofs, np.int32),
                            _c(row_ptr, np.int32), _c(cols, np.int32), rho, mu, dt,
                            *[None if a is None else a.ctypes.data_as(C.c_void_p) for a in keep],
                            None if fm is None else fm.ctypes.data_as(C.c_void_p), A, rhs)
    if rc:
        raise RuntimeError("pattern misses an entry")
    return A, rhs


def fem_constrain(row_ptr, cols, A, rhs, rows, values):
    """Dirichlet rows on an assembled system, restated: a constrained row
    keeps its diagonal alone and its right-hand side becomes A_rr g_r; every
    other row moves A_rc g_c of each constrained column (ascending) to its
    right-hand side and zeroes A_rc.  Right-hand side q uses matrix
    min(q, matrices - 1).  Returns new (A, rhs)."""
    A = np.array(A, dtype=np.float64)
    rhs = np.array(rhs, dtype=np.float64)
    values = np.asarray(values, np.float64)
    nm, ns, nd = A.shape[0], rhs.shape[0], rhs.shape[1]
    idx = -np.ones(nd, np.int64)
    idx[np.asarray(rows, np.int64)] = np.arange(len(rows))
    for r in range(nd):
        b, e = int(row_ptr[r]), int(row_ptr[r + 1])
        cs = cols[b:e]
        if idx[r] >= 0:
            for q in range(ns):
                m = min(q, nm - 1)
                diag = 0.0
                for k in range(b, e):
                    if cols[k] == r:
                        diag = float(A[m, k])
                rhs[q, r] = diag * float(values[q][idx[r]])
            for m in range(nm):
                A[m, b:e][cs != r] = 0.0
            continue
        hit = idx[cs] >= 0
        if not hit.any():
            continue
        for q in range(ns):
            m = min(q, nm - 1)
            s = float(rhs[q, r])
            for k in range(b, e):
                ic = idx[cols[k]]
                if ic >= 0:
                    s = s - float(A[m, k]) * float(values[q][ic])
            rhs[q, r] = s
        for m in range(nm):
            A[m, b:e][hit] = 0.0
    return A, rhs


def fem_velocity_bc(mesh, face_ids, velocity_dirichlet, velocity_bc, rho, dt, P):
    """velocity_prediction_bc restated: (rows, values (dim, n)) of the
    prediction's Dirichlet rows.  velocity_bc maps an id to its velocity."""
    L = lib()
    ids = np.asarray(sorted(velocity_bc), np.int32)
    vel = np.ascontiguousarray([velocity_bc[i] for i in ids], np.float64).reshape(-1)
    vd = np.asarray(list(velocity_dirichlet), np.int32)
    flags = np.zeros(mesh.n_dofs, np.int32)
    vals = np.zeros((mesh.dim, mesh.n_dofs))
    L.orc_fem_velocity_bc(mesh.dim, mesh.n_cells, mesh.n_dofs, _c(mesh.vertices[mesh.cells], np.float64),
                          _c(mesh.cell_dofs, np.int32), _c(face_ids, np.int32), len(vd), vd if len(vd) else
                          np.zeros(1, np.int32), len(ids), ids if len(ids) else np.zeros(1, np.int32),
                          vel if len(vel) else np.zeros(1), rho, dt, _c(P, np.float64), flags, vals)
    rows = np.nonzero(flags)[0].astype(np.int32)
    return rows, np.ascontiguousarray(vals[:, rows])
