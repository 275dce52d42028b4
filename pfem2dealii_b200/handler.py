"""Python mirror of pfem2ParticleHandler<dim> over the C ABI.

Method names and meaning follow src/pfem2particlehandler.h:17-71 of the
reference; the solver-owned inputs (parameters, mesh, the FEM velocity
vectors) are passed in explicitly instead of being fetched from a
pfem2Solver.  Velocity vectors are component-major arrays of shape
(dim, n_dofs), host numpy arrays or (for the *_device calls) CUDA tensors.
The *_device calls run on the handle's own CUDA stream and are ordered
against torch's current stream on both sides, so their tensors can be
produced and consumed by torch operations without further synchronisation.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import dataclasses
import json

import numpy as np

from . import _lib
from .mesh import Mesh, vertex_maps


@dataclasses.dataclass
class ParticleParams:
    """The particle keys of the reference's .prm file
    (src/pfem2parameterhandler.cpp:64-74, 40)."""

    particles_per_cell: tuple = (2, 2, 2)
    max_particles_per_cell_part: int = 2
    particle_integration_steps: int = 5
    time_step: float = 0.1
    removal_seed: int = 0
    empty_dof_policy: int = 0
    capacity: int = 0
    integrator: int = 0  # 0 Euler (the reference), 1 RK2 midpoint (opt-in)

    def to_c(self, dim):
        p = _lib.Params()
        q = list(self.particles_per_cell) + [1, 1, 1]
        for d in range(3):
            p.particles_per_cell[d] = int(q[d]) if d < dim else 1
        p.max_particles_per_cell_part = int(self.max_particles_per_cell_part)
        p.particle_integration_steps = int(self.particle_integration_steps)
        p.time_step = float(self.time_step)
        p.removal_seed = int(self.removal_seed)
        p.empty_dof_policy = int(self.empty_dof_policy)
        p.capacity = int(self.capacity)
        p.integrator = int(self.integrator)
        return p


def read_prm(path_or_text) -> ParticleParams:
    """Particle keys of a deal.II .prm file (subsections 'Particles' and
    'Computation parameters'), as read by src/pfem2parameterhandler.cpp:25-156."""
    text = path_or_text
    if "\n" not in path_or_text:
        with open(path_or_text) as f:
            text = f.read()
    sec = []
    vals = {}
    for raw in text.splitlines():
        line = raw.split("#")[0].strip()
        if not line:
            continue
        if line.startswith("subsection"):
            sec.append(line[len("subsection"):].strip())
        elif line == "end":
            sec.pop()
        elif line.startswith("set"):
            k, _, v = line[3:].partition("=")
            vals[(sec[-1] if sec else "", k.strip())] = v.strip()
    P = "Particles"
    q = [int(vals.get((P, f"Number of particles in the {a} direction"), 2)) for a in "xyz"]
    return ParticleParams(
        particles_per_cell=tuple(q),
        max_particles_per_cell_part=int(vals.get((P, "Maximum number of particles per cell part"), 2)),
        particle_integration_steps=int(vals.get((P, "Particle integration steps"), 5)),
        time_step=float(vals.get(("Computation parameters", "Time step"), 0.1)),
    )


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _host(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def project_noalloc(cell_dofs, cell, xi, v, out, empty_dof_policy=0, stream=None):
    """pfem2gpu_project_noalloc on CUDA tensors: cell_dofs (n_cells, 2^dim)
    int32, cell (n,) int32 ascending, xi and v (dim, n) float64, out
    (dim, n_dofs) float64.  Allocates no device memory; returns the number of
    DoFs no particle reaches."""
    import torch

    dim, n_dofs = out.shape
    n = cell.shape[0]
    dev = torch.device("cuda", torch.cuda.current_device())
    for name, t, dtype, shape in (("cell_dofs", cell_dofs, torch.int32, (cell_dofs.shape[0], 1 << dim)),
                                  ("cell", cell, torch.int32, (n,)), ("xi", xi, torch.float64, (dim, n)),
                                  ("v", v, torch.float64, (dim, n)), ("out", out, torch.float64, (dim, n_dofs))):
        if t.dtype != dtype or tuple(t.shape) != shape or not t.is_contiguous() or t.device != dev:
            raise ValueError(f"project_noalloc: {name} must be a contiguous {dtype} tensor of shape {shape} "
                             f"on {dev}, got {t.dtype} {tuple(t.shape)} on {t.device}")
    n_empty = C.c_int64(0)
    _lib.check(_lib.load().pfem2gpu_project_noalloc(
        dim, cell_dofs.shape[0], n_dofs, _ptr(cell_dofs), cell.shape[0], _ptr(cell), _ptr(xi), _ptr(v),
        int(empty_dof_policy), _ptr(out), C.byref(n_empty), stream))
    return n_empty.value


class ParticleHandler:
    """pfem2ParticleHandler<dim> on one B200.  precision: "fp64" (the
    reference's arithmetic) or "fp32"."""

    def __init__(self, dim: int, params: ParticleParams, precision: str = "fp64"):
        self.L = _lib.load()
        self.dim = dim
        self.params = params
        self.precision = precision
        h = C.c_void_p()
        prec = _lib.FP64 if precision == "fp64" else _lib.FP32
        _lib.check(self.L.pfem2gpu_create(dim, prec, C.byref(params.to_c(dim)), C.byref(h)))
        self.h = h
        self.mesh = None
        self._hs = None

    @contextlib.contextmanager
    def _torch_ordered(self):
        """Order a device call against torch's current stream: the handle's
        stream first waits for the work torch has queued (the tensors the
        call reads may still be being written), and torch's stream then waits
        for the call's work (the tensors it writes, and the reuse of freed
        tensor memory), so the *_device calls compose with torch operations
        like any torch operation."""
        import torch

        if self._hs is None:
            self._hs = torch.cuda.ExternalStream(self.stream_handle())
            self._ev = (torch.cuda.Event(), torch.cuda.Event())
        cur = torch.cuda.current_stream()
        self._ev[0].record(cur)
        self._hs.wait_event(self._ev[0])
        try:
            yield
        finally:
            self._ev[1].record(self._hs)
            cur.wait_event(self._ev[1])

    def close(self):
        if getattr(self, "h", None):
            self.L.pfem2gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        _lib.check(rc, self.h)

    # -- mesh -----------------------------------------------------------------
    def initialize_maps(self, mesh: Mesh, host_maps: bool = False):
        """Mesh upload plus initialize_maps (src/pfem2particlehandler.cpp:320-324).
        The vertex maps are built on the device, or, with host_maps, by
        mesh.vertex_maps and passed in."""
        assert mesh.dim == self.dim
        self.mesh = mesh
        self._keep = [
            _host(mesh.vertices, np.float64),
            _host(mesh.cells, np.int32),
            _host(mesh.cell_dofs, np.int32),
        ]
        maps = [None, None, None]
        if host_maps:
            off, cells, dirs = vertex_maps(mesh)
            maps = [_host(off, np.int32), _host(cells, np.int32), _host(dirs, np.float64)]
            self._keep += maps
        self._ck(self.L.pfem2gpu_set_mesh(self.h, mesh.n_cells, mesh.n_verts, mesh.n_dofs,
                                          *[_ptr(a) for a in self._keep[:3]], *[_ptr(a) for a in maps]))

    # -- the particle cycle ---------------------------------------------------
    def seed_particles(self, V):
        V = _host(V, np.float64)
        self._ck(self.L.pfem2gpu_seed(self.h, _ptr(V)))

    def correct_particle_velocity(self, V, Vold):
        V = _host(V, np.float64)
        Vold = _host(Vold, np.float64)
        self._ck(self.L.pfem2gpu_correct(self.h, _ptr(V), _ptr(Vold)))

    def correct_particle_velocity_from_projection(self, V):
        """correct_particle_velocity with Vold = the last projection, kept on
        the device (the reference's data flow: fem_step copies the projected
        velocity into the old solution, src/pfem2fem.cpp:523-524)."""
        V = _host(V, np.float64)
        self._ck(self.L.pfem2gpu_correct_from_projection(self.h, _ptr(V)))

    def move_particles(self, V=None):
        V = None if V is None else _host(V, np.float64)
        self._ck(self.L.pfem2gpu_move(self.h, _ptr(V)))

    def project_particle_fields(self):
        out = np.empty((self.dim, self.mesh.n_dofs))
        self._ck(self.L.pfem2gpu_project(self.h, _ptr(out)))
        return out

    def step(self, V, Vold):
        """One time step of the reference loop (src/pfem2solver.cpp:162-164)."""
        self.correct_particle_velocity(V, Vold)
        self.move_particles(None)
        return self.project_particle_fields()

    # device-resident variants (torch CUDA tensors, float64, shape (dim, n_dofs))
    def seed_particles_device(self, dV):
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_seed_device(self.h, _ptr(dV)))

    def correct_particle_velocity_device(self, dV, dVold):
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_correct_device(self.h, _ptr(dV), _ptr(dVold)))

    def move_particles_device(self, dV=None):
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_move_device(self.h, _ptr(dV)))

    def project_particle_fields_device(self, dout):
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_project_device(self.h, _ptr(dout)))

    def correct_particle_velocity_from_projection_device(self, dV):
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_correct_from_projection_device(self.h, _ptr(dV)))

    def step_solver(self, V):
        """One time step with the solver's data flow: correct with Vold = the
        last projection, move, project (host vectors)."""
        self.correct_particle_velocity_from_projection(V)
        self.move_particles(None)
        return self.project_particle_fields()

    def step_device(self, dV, dVold, dout):
        """correct + move + project on device vectors as one CUDA graph
        (dVold None: the last projection)."""
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_step_device(self.h, _ptr(dV), _ptr(dVold), _ptr(dout)))

    # -- differentiated window (no counterpart in the reference) -------------
    def window_forward_device(self, steps, checkpoint_every, dV, dVold=None, dv0=None, dU=None):
        """K steps of correct + move without count correction from the
        current particles, then the projection, on CUDA tensors: dV, dVold,
        dU (dim, n_dofs) float64, dv0 (n, dim) float64 or None.  The
        particles are not changed.  Returns dU."""
        if dU is None:
            import torch

            dU = torch.empty_like(dV)
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_window_forward_device(self.h, int(steps), int(checkpoint_every), _ptr(dV),
                                                           _ptr(dVold), _ptr(dv0), _ptr(dU)))
        return dU

    def window_backward_device(self, dgU, dg_v0=None, dg_V=None, dg_Vold=None):
        """Adjoint of the last window forward for dJ/dU = dgU (CUDA tensors)."""
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_window_backward_device(self.h, _ptr(dgU), _ptr(dg_v0), _ptr(dg_V),
                                                            _ptr(dg_Vold)))

    # -- the solver step's Q1 systems (src/pfem2fem.cpp:247-510, volume terms) ----
    FEM_PREDICTION, FEM_PRESSURE, FEM_CORRECTION = 0, 1, 2

    def fem_pattern(self):
        """CSR pattern (row_ptr, cols) of the system matrices."""
        n = C.c_int64()
        row_ptr = np.zeros(self.mesh.n_dofs + 1, np.int32)
        self._ck(self.L.pfem2gpu_fem_pattern(self.h, _ptr(row_ptr), None, 0, C.byref(n)))
        cols = np.zeros(max(n.value, 1), np.int32)
        self._ck(self.L.pfem2gpu_fem_pattern(self.h, _ptr(row_ptr), _ptr(cols), n.value, C.byref(n)))
        return row_ptr, cols[: n.value]

    def fem_set_boundary(self, face_ids, velocity_dirichlet=(), pressure_dirichlet=()):
        """Boundary ids per cell and face (mesh.boundary_face_ids) and the
        Dirichlet id sets; None clears (no face terms)."""
        if face_ids is None:
            self._ck(self.L.pfem2gpu_fem_set_boundary(self.h, None, 0, None, 0, None))
            return
        fid = _host(face_ids, np.int32)
        vd = np.asarray(list(velocity_dirichlet) or [0], np.int32)
        pd = np.asarray(list(pressure_dirichlet) or [0], np.int32)
        self._ck(self.L.pfem2gpu_fem_set_boundary(self.h, _ptr(fid), len(velocity_dirichlet), _ptr(vd),
                                                  len(pressure_dirichlet), _ptr(pd)))

    def fem_assemble(self, system, rho, mu, dt, U, U2=None, P=None):
        """One system on host arrays: (A (matrices, nnz), rhs (right-hand sides, n_dofs)).
        PREDICTION: U = solution V, U2 = old solution V; PRESSURE: U = predicted
        V; CORRECTION: U = predicted V, P = pressure."""
        n = C.c_int64()
        self._ck(self.L.pfem2gpu_fem_pattern(self.h, None, None, 0, C.byref(n)))
        nm = self.dim if system == self.FEM_PREDICTION else 1
        ns = 1 if system == self.FEM_PRESSURE else self.dim
        A = np.empty((nm, max(n.value, 1)))
        rhs = np.empty((ns, self.mesh.n_dofs))
        keep = [None if a is None else _host(a, np.float64) for a in (U, U2, P)]
        self._ck(self.L.pfem2gpu_fem_assemble(self.h, int(system), float(rho), float(mu), float(dt),
                                              *[_ptr(a) for a in keep], _ptr(A), _ptr(rhs)))
        return A[:, : n.value], rhs

    def fem_velocity_bc(self, rho, dt, P, velocity_bc):
        """velocity_prediction_bc: (rows, values (dim, n)) of the prediction's
        Dirichlet rows; velocity_bc maps a Dirichlet boundary id to its
        velocity vector."""
        P = _host(P, np.float64)
        ids = np.asarray(sorted(velocity_bc), np.int32)
        vel = np.ascontiguousarray([velocity_bc[i] for i in ids], np.float64).reshape(len(ids), self.dim)
        n = C.c_int64()
        args = (_ptr(ids) if len(ids) else None, _ptr(vel) if len(ids) else None)
        self._ck(self.L.pfem2gpu_fem_velocity_bc(self.h, float(rho), float(dt), _ptr(P), len(ids), *args, None,
                                                 None, 0, C.byref(n)))
        rows = np.zeros(max(n.value, 1), np.int32)
        vals = np.zeros((self.dim, max(n.value, 1)))
        self._ck(self.L.pfem2gpu_fem_velocity_bc(self.h, float(rho), float(dt), _ptr(P), len(ids), *args, _ptr(rows),
                                                 _ptr(vals), n.value, C.byref(n)))
        k = n.value
        return rows[:k], np.ascontiguousarray(vals.ravel()[: self.dim * k].reshape(self.dim, k))

    def fem_constrain(self, system, A, rhs, rows, values):
        """Dirichlet rows (pfem2gpu_fem_constrain) on host copies of an
        assembled system: returns the constrained (A, rhs).  values: one row
        of len(rows) values per right-hand side."""
        A = np.array(A, dtype=np.float64, order="C")
        rhs = np.array(rhs, dtype=np.float64, order="C")
        r = np.ascontiguousarray(rows, np.int32)
        v = np.ascontiguousarray(values, np.float64)
        self._ck(self.L.pfem2gpu_fem_constrain(self.h, int(system), len(r), _ptr(r) if len(r) else None,
                                               _ptr(v) if len(r) else None, _ptr(A), _ptr(rhs)))
        return A, rhs

    def vertex_maps(self):
        """The vertex -> cell maps in use: (offsets, cells, dirs (n, dim))."""
        off = np.zeros(self.mesh.n_verts + 1, np.int32)
        n = C.c_int64()
        self._ck(self.L.pfem2gpu_get_vertex_maps(self.h, _ptr(off), None, None, 0, C.byref(n)))
        k = max(n.value, 1)
        cells = np.zeros(k, np.int32)
        dirs = np.zeros((k, self.dim))
        self._ck(self.L.pfem2gpu_get_vertex_maps(self.h, _ptr(off), _ptr(cells), _ptr(dirs), k, C.byref(n)))
        return off, cells[: n.value], dirs[: n.value]

    def window_particles(self):
        """End states of the last window forward: cell (-1: deleted), xi, v."""
        n = C.c_int64()
        self._ck(self.L.pfem2gpu_window_size(self.h, C.byref(n)))
        k = max(n.value, 1)
        cell = np.zeros(k, np.int32)
        xi = np.zeros((k, self.dim))
        v = np.zeros((k, self.dim))
        self._ck(self.L.pfem2gpu_window_particles(self.h, _ptr(cell), _ptr(xi), _ptr(v), k, C.byref(n)))
        return {"cell": cell[: n.value], "xi": xi[: n.value], "v": v[: n.value]}

    def adjoint(self, steps, checkpoint_every, V, gU, Vold=None, v0=None):
        """Window forward + adjoint on host arrays: (U, g_v0 (n, dim), g_V, g_Vold)."""
        n = self.stats()["n_particles"]
        V = _host(V, np.float64)
        gU = _host(gU, np.float64)
        Vold = None if Vold is None else _host(Vold, np.float64)
        v0 = None if v0 is None else _host(v0, np.float64)
        U = np.empty((self.dim, self.mesh.n_dofs))
        gv0 = np.empty((max(n, 1), self.dim))
        gV = np.empty_like(U)
        gVo = np.empty_like(U)
        self._ck(self.L.pfem2gpu_adjoint(self.h, int(steps), int(checkpoint_every), _ptr(V), _ptr(Vold), _ptr(v0),
                                         _ptr(gU), _ptr(U), _ptr(gv0), _ptr(gV), _ptr(gVo)))
        return U, gv0[:n], gV, gVo

    # -- particle access ------------------------------------------------------
    def particles(self):
        """Host copy of the particles (begin()/end() of the reference)."""
        n = C.c_int64()
        self.L.pfem2gpu_get_particles(self.h, None, None, None, None, None, 0, C.byref(n))
        cap = max(n.value, 1)
        ids = np.zeros(cap, np.uint32)
        cell = np.zeros(cap, np.int32)
        x = np.zeros((cap, self.dim))
        xi = np.zeros((cap, self.dim))
        v = np.zeros((cap, self.dim))
        self._ck(self.L.pfem2gpu_get_particles(self.h, _ptr(ids), _ptr(cell), _ptr(x), _ptr(xi), _ptr(v), cap,
                                               C.byref(n)))
        k = n.value
        return {"id": ids[:k], "cell": cell[:k], "x": x[:k], "xi": xi[:k], "v": v[:k]}

    def set_particles(self, P, next_id):
        n = len(P["id"])
        arrs = [_host(P["id"], np.uint32), _host(P["cell"], np.int32), _host(P["x"], np.float64),
                _host(P["xi"], np.float64), _host(P["v"], np.float64)]
        self._ck(self.L.pfem2gpu_set_particles(self.h, n, *[_ptr(a) for a in arrs], next_id))

    # -- cell-range partitions (pfem2dealii_b200.shard) -----------------------
    def set_partition(self, cell_begin: int, cell_end: int):
        """Own the particles of cells [cell_begin, cell_end) only."""
        self._ck(self.L.pfem2gpu_set_partition(self.h, int(cell_begin), int(cell_end)))

    def move_exchange_begin(self, V=None) -> int:
        """Phase 1 of a partitioned move; returns the outbox size."""
        V = None if V is None else _host(V, np.float64)
        n = C.c_int64()
        self._ck(self.L.pfem2gpu_move_exchange_begin(self.h, _ptr(V), C.byref(n)))
        return n.value

    def move_outbox(self, n: int):
        """The n particles that ended the move in foreign cells (dict of
        id, cell, x, xi, v)."""
        P = {"id": np.zeros(n, np.uint32), "cell": np.zeros(n, np.int32), "x": np.zeros((n, self.dim)),
             "xi": np.zeros((n, self.dim)), "v": np.zeros((n, self.dim))}
        got = C.c_int64()
        self._ck(self.L.pfem2gpu_move_outbox(self.h, *[_ptr(P[k]) for k in ("id", "cell", "x", "xi", "v")], n,
                                             C.byref(got)))
        return P

    def move_inbox(self, P) -> int:
        """The particles sent to this handle's cells; returns the number of
        particles count correction will add."""
        arrs = [_host(P["id"], np.uint32), _host(P["cell"], np.int32), _host(P["x"], np.float64),
                _host(P["xi"], np.float64), _host(P["v"], np.float64)]
        ns = C.c_int64()
        self._ck(self.L.pfem2gpu_move_inbox(self.h, len(arrs[0]), *[_ptr(a) for a in arrs], C.byref(ns)))
        return ns.value

    def move_exchange_end(self, first_id: int, next_id: int):
        self._ck(self.L.pfem2gpu_move_exchange_end(self.h, int(first_id), int(next_id)))

    def get_partials(self, cells):
        """Projection partial sums of the listed cells, (n, 2^dim x 4)."""
        cells = _host(cells, np.int32)
        out = np.zeros((len(cells), 4 << self.dim))
        self._ck(self.L.pfem2gpu_get_partials(self.h, len(cells), _ptr(cells), _ptr(out)))
        return out

    def set_partials(self, cells, values):
        cells = _host(cells, np.int32)
        values = _host(values, np.float64)
        if values.shape != (len(cells), 4 << self.dim):
            raise ValueError(f"set_partials: values must have shape ({len(cells)}, {4 << self.dim})")
        self._ck(self.L.pfem2gpu_set_partials(self.h, len(cells), _ptr(cells), _ptr(values)))

    def pack_output_device(self, dout=None):
        """Float32 positions and velocities of the particles packed on the
        device (a CUDA tensor of 6 n floats: n x 3 positions, then n x 3
        velocities), the data of output_particle_solution.  Returns the
        tensor and n."""
        import torch

        n = self.stats()["n_particles"]
        if dout is None:
            dout = torch.empty(max(6 * n, 1), dtype=torch.float32, device="cuda")
        got = C.c_int64()
        with self._torch_ordered():
            self._ck(self.L.pfem2gpu_pack_output_device(self.h, _ptr(dout), dout.numel() // 6, C.byref(got)))
        return dout, got.value

    def output_particle_solution(self, timestep_number: int, directory: str = "."):
        """particles-NN.000.vtu plus particles-NN.pvtu
        (src/pfem2particlehandler.cpp:218-317, one rank)."""
        import os

        base = f"particles-{timestep_number:02d}"
        self._ck(self.L.pfem2gpu_write_vtu(self.h, os.path.join(directory, base + ".000.vtu").encode()))
        with open(os.path.join(directory, base + ".pvtu"), "w") as f:
            f.write('<?xml version="1.0" ?> \n<VTKFile type="PUnstructuredGrid" version="0.1" '
                    'byte_order="LittleEndian">\n  <PUnstructuredGrid GhostLevel="0">\n'
                    '    <PPointData Scalars="scalars">\n'
                    '      <PDataArray type="Float32" Name="velocity" NumberOfComponents="3" format="ascii"/>\n'
                    '      <PDataArray type="Float32" Name="subdomain" format="ascii"/>\n'
                    '    </PPointData>\n    <PPoints>\n'
                    '      <PDataArray type="Float32" NumberOfComponents="3"/>\n    </PPoints>\n'
                    f'    <Piece Source="{base}.000.vtu"/>  </PUnstructuredGrid>\n</VTKFile>\n')

    # -- diagnostics ----------------------------------------------------------
    def stats(self):
        s = _lib.Stats()
        self._ck(self.L.pfem2gpu_get_stats(self.h, C.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        self._ck(self.L.pfem2gpu_reset_stats(self.h))

    def synchronize(self):
        self._ck(self.L.pfem2gpu_synchronize(self.h))

    def stream_handle(self) -> int:
        p = C.c_void_p()
        self._ck(self.L.pfem2gpu_get_stream(self.h, C.byref(p)))
        return p.value or 0

    def profile(self, on: bool):
        self._ck(self.L.pfem2gpu_profile(self.h, 1 if on else 0))

    def profile_report(self):
        buf = C.create_string_buffer(1 << 16)
        self._ck(self.L.pfem2gpu_profile_report(self.h, buf, 1 << 16))
        return json.loads(buf.value.decode())

    def launch_count(self) -> int:
        c = C.c_uint64()
        self._ck(self.L.pfem2gpu_launch_count(self.h, C.byref(c)))
        return c.value
