"""pfem2ParticleHandler<dim> partitioned by cells over the ranks of a
torch.distributed process group, one GPU per rank.

The reference distributes the triangulation's cells over MPI ranks (p4est),
keeps each rank's particles in its own cells, sends the particles that a
relocation finds in another rank's cells to that rank (send_recv_particles,
src/pfem2particlehandler.cpp:480-502,507-618) and sums the projection over
the ghost cells of each DoF (project_particle_fields, :202-205,
compress(VectorOperation::add)).  Here every rank holds the whole mesh and
the whole nodal velocity (the FEM solve stays replicated, as the velocity is
an input of the path), owns the particles of a contiguous range of cells, and
exchanges after each move:

* the particles whose move ended in another rank's cells (outbox -> inbox),
  before count correction, so that each cell's particles, their order and
  their ids are those of one unpartitioned handle;
* the seed counts, scanned over the ranks in cell order, so the new
  particles get the ids an unpartitioned run hands out;
* the projection partial sums of the cells that share a DoF with another
  rank's cells (the halo), so each rank's projection is exact on the DoFs of
  its own cells; the full projection is assembled from each DoF's lowest
  owning rank.

In the FP64 form the result is bit-identical to one unpartitioned handle.
The exchange runs on the host over the process group (gloo on CPU tensors,
NCCL on CUDA tensors): its volume is the crossing particles and the halo
cells' partial sums, a small part of a step's particle data.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .handler import ParticleHandler, ParticleParams
from .mesh import Mesh


# ---------------------------------------------------------------------------
# Host logic of the partition (numpy only, no device and no communication).
# ---------------------------------------------------------------------------
def cell_bounds(n_cells: int, world: int) -> np.ndarray:
    """Contiguous cell ranges of `world` ranks: rank r owns
    [bounds[r], bounds[r + 1]); sizes differ by at most one cell."""
    if world < 1:
        raise ValueError("world must be >= 1")
    return np.array([(r * n_cells) // world for r in range(world + 1)], dtype=np.int64)


def owner_of_cells(cells, bounds) -> np.ndarray:
    """Rank owning each cell."""
    return np.searchsorted(bounds, np.asarray(cells, dtype=np.int64), side="right") - 1


def halo_cells(cell_dofs: np.ndarray, n_dofs: int, begin: int, end: int) -> np.ndarray:
    """Cells outside [begin, end) that share a DoF with a cell inside it
    (the ghost cells of the reference's partition), ascending."""
    mark = np.zeros(n_dofs, dtype=bool)
    mark[cell_dofs[begin:end].ravel()] = True
    touch = mark[cell_dofs].any(axis=1)
    touch[begin:end] = False
    return np.nonzero(touch)[0].astype(np.int32)


def dof_owners(cell_dofs: np.ndarray, n_dofs: int, bounds) -> np.ndarray:
    """Lowest rank owning a cell around each DoF (the DoF's owner)."""
    world = len(bounds) - 1
    own = np.full(n_dofs, world, dtype=np.int64)
    rank = owner_of_cells(np.arange(cell_dofs.shape[0]), bounds)
    np.minimum.at(own, cell_dofs.ravel(), np.repeat(rank, cell_dofs.shape[1]))
    return own


def halo_plan(cell_dofs: np.ndarray, n_dofs: int, bounds, rank: int):
    """The halo exchange of `rank`: the cells whose partial sums it receives
    (its halo, ascending) and, per peer, the own cells whose partial sums it
    sends (that peer's halo cells inside this rank's range, ascending)."""
    world = len(bounds) - 1
    b, e = int(bounds[rank]), int(bounds[rank + 1])
    recv = halo_cells(cell_dofs, n_dofs, b, e)
    send = []
    for q in range(world):
        if q == rank:
            send.append(np.zeros(0, np.int32))
            continue
        hq = halo_cells(cell_dofs, n_dofs, int(bounds[q]), int(bounds[q + 1]))
        send.append(hq[(hq >= b) & (hq < e)])
    return recv, send


def seed_ids(n_seeds, rank: int, next_id: int):
    """Ids of a move's new particles: (first_id, next_id) of `rank` given
    every rank's seed count (ranks in cell order) and the ids handed out
    before the move."""
    n = [int(s) for s in n_seeds]
    return next_id + sum(n[:rank]), next_id + sum(n)


@dataclass
class Particles:
    """Host particle records: id (n,), cell (n,), x, xi, v (n, dim)."""

    id: np.ndarray
    cell: np.ndarray
    x: np.ndarray
    xi: np.ndarray
    v: np.ndarray

    @staticmethod
    def empty(dim):
        return Particles(np.zeros(0, np.uint32), np.zeros(0, np.int32), np.zeros((0, dim)), np.zeros((0, dim)),
                         np.zeros((0, dim)))

    def __len__(self):
        return len(self.id)

    def take(self, sel):
        return Particles(self.id[sel], self.cell[sel], self.x[sel], self.xi[sel], self.v[sel])

    @staticmethod
    def concat(parts, dim):
        parts = [p for p in parts if len(p)]
        if not parts:
            return Particles.empty(dim)
        return Particles(*[np.concatenate([getattr(p, f) for p in parts]) for f in ("id", "cell", "x", "xi", "v")])


def route(p: Particles, bounds):
    """Split particles by the rank owning their cell."""
    world = len(bounds) - 1
    own = owner_of_cells(p.cell, bounds)
    return [p.take(own == q) for q in range(world)]


# ---------------------------------------------------------------------------
# Communication: every rank sends one object per peer, host side.
# ---------------------------------------------------------------------------
class TorchComm:
    """Exchange over a torch.distributed process group (gloo or NCCL; NCCL
    moves the pickled objects through the current CUDA device)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def allgather(self, obj):
        out = [None] * self.world
        self.dist.all_gather_object(out, obj, group=self.group)
        return out

    def exchange(self, per_peer):
        """per_peer[q] goes to rank q; returns what every rank sent to this
        one, by source rank."""
        got = self.allgather(per_peer)
        return [got[q][self.rank] for q in range(self.world)]


class LocalComm:
    """The exchange of a one-rank run (no process group)."""

    rank, world = 0, 1

    def allgather(self, obj):
        return [obj]

    def exchange(self, per_peer):
        return [per_peer[0]]


# ---------------------------------------------------------------------------
# The partitioned handler.
# ---------------------------------------------------------------------------
def _particles(P) -> Particles:
    return Particles(P["id"], P["cell"], P["x"], P["xi"], P["v"])


class ShardedParticleHandler:
    """pfem2ParticleHandler<dim> with its cells split over the ranks of
    `comm` (a TorchComm, or LocalComm for one rank): one ParticleHandler per
    rank on that rank's current CUDA device.  Method names and meaning follow
    ParticleHandler; nodal vectors are full (dim, n_dofs) host arrays on every
    rank, and project_particle_fields returns the full projection on every
    rank.  `handler` is the rank's ParticleHandler (made here by default)."""

    def __init__(self, dim: int, params: ParticleParams, precision: str = "fp64", comm=None, handler=None):
        self.comm = comm if comm is not None else LocalComm()
        self.rank, self.world = self.comm.rank, self.comm.world
        self.dim = dim
        self.precision = precision
        self.ph = handler if handler is not None else ParticleHandler(dim, params, precision)
        self.mesh = None
        self.next_id = 0
        self.exchanged = 0  # particles this rank sent, all moves

    def close(self):
        self.ph.close()

    def initialize_maps(self, mesh: Mesh, host_maps: bool = False):
        self.ph.initialize_maps(mesh, host_maps)
        self.mesh = mesh
        self.bounds = cell_bounds(mesh.n_cells, self.world)
        self.begin, self.end = int(self.bounds[self.rank]), int(self.bounds[self.rank + 1])
        self.ph.set_partition(self.begin, self.end)
        cd = np.asarray(mesh.cell_dofs)
        self.halo_recv, self.halo_send = halo_plan(cd, mesh.n_dofs, self.bounds, self.rank)
        owners = dof_owners(cd, mesh.n_dofs, self.bounds)
        self.dof_by_rank = [np.nonzero(owners == q)[0] for q in range(self.world)]
        self.dof_owned = self.dof_by_rank[self.rank]

    # -- the particle cycle ---------------------------------------------------
    def seed_particles(self, V):
        self.ph.seed_particles(V)
        self.next_id = int(self.ph.stats()["next_id"])

    def correct_particle_velocity(self, V, Vold):
        self.ph.correct_particle_velocity(V, Vold)

    def correct_particle_velocity_from_projection(self, V):
        self.ph.correct_particle_velocity_from_projection(V)

    def move_particles(self, V=None):
        """move_particles (:142-171) with send_recv_particles (:507-618)."""
        n = self.ph.move_exchange_begin(V)
        out = _particles(self.ph.move_outbox(n))
        self.exchanged += n
        inbox = Particles.concat(self.comm.exchange(route(out, self.bounds)), self.dim)
        n_seeds = self.ph.move_inbox(vars(inbox))
        first, nxt = seed_ids(self.comm.allgather(n_seeds), self.rank, self.next_id)
        self.ph.move_exchange_end(first, nxt)
        self.next_id = nxt

    def _exchange_halo(self):
        send = [(cells, self.ph.get_partials(cells)) for cells in self.halo_send]
        got = self.comm.exchange(send)
        cells = np.concatenate([c for c, _ in got]).astype(np.int32)
        vals = np.concatenate([b for _, b in got]).reshape(len(cells), 4 << self.dim)
        self.ph.set_partials(cells, vals)

    def project_particle_fields(self):
        """project_particle_fields (:174-215): this rank's projection with its
        halo's partial sums, each DoF taken from its owner."""
        self._exchange_halo()
        mine = self.ph.project_particle_fields()
        parts = self.comm.allgather(np.ascontiguousarray(mine[:, self.dof_owned]))
        out = np.empty_like(mine)
        for q in range(self.world):
            out[:, self.dof_by_rank[q]] = parts[q]
        return out

    def step(self, V, Vold):
        self.correct_particle_velocity(V, Vold)
        self.move_particles(None)
        return self.project_particle_fields()

    def step_solver(self, V):
        """One step of the solver's data flow: Vold = the last projection."""
        self.correct_particle_velocity_from_projection(V)
        self.move_particles(None)
        return self.project_particle_fields()

    # -- access ---------------------------------------------------------------
    def local_particles(self):
        return self.ph.particles()

    def particles(self):
        """All particles on every rank, in the unpartitioned handle's order
        (rank ranges are contiguous and ascending)."""
        parts = self.comm.allgather(self.ph.particles())
        return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}

    def stats(self):
        """Counters summed over the ranks (next_id is the common one)."""
        s = self.comm.allgather(self.ph.stats())
        out = {k: sum(d[k] for d in s) for k in s[0] if isinstance(s[0][k], (int, float))}
        out["next_id"] = self.next_id
        out["exchanged"] = sum(self.comm.allgather(self.exchanged))
        return out
