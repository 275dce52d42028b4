"""Host logic of the cell-partitioned handler (pfem2dealii_b200.shard), no
GPU: the partition helpers, the halo identity of the projection, and the
whole exchange choreography of ShardedParticleHandler over two and three
gloo ranks, driven through a numpy stand-in of the partitioned C handle
(StandIn below) and compared with one unpartitioned stand-in."""
import os
import random
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from pfem2dealii_b200 import mesh as M  # noqa: E402
from pfem2dealii_b200 import shard as S  # noqa: E402


def small_mesh(dim):
    if dim == 2:
        return M.hyper_rectangle((0.0, 0.0), (3.0, 1.0), (9, 4))
    return M.hyper_rectangle((0.0, 0.0, 0.0), (2.0, 1.0, 1.0), (6, 3, 3))


# ---------------------------------------------------------------------------
# partition helpers
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n,world", [(10, 1), (10, 3), (7, 7), (5, 8), (0, 2)])
def test_cell_bounds_cover_in_order(n, world):
    b = S.cell_bounds(n, world)
    assert b[0] == 0 and b[-1] == n and len(b) == world + 1
    sizes = np.diff(b)
    assert (sizes >= 0).all() and sizes.max() - sizes.min() <= 1
    cells = np.arange(n)
    own = S.owner_of_cells(cells, b)
    for r in range(world):
        assert ((own == r) == ((cells >= b[r]) & (cells < b[r + 1]))).all()


@pytest.mark.parametrize("dim", [2, 3])
def test_halo_cells_match_brute_force(dim):
    m = small_mesh(dim)
    cd = m.cell_dofs
    for world in (2, 3):
        b = S.cell_bounds(m.n_cells, world)
        for r in range(world):
            lo, hi = int(b[r]), int(b[r + 1])
            own_dofs = set(cd[lo:hi].ravel().tolist())
            want = [c for c in range(m.n_cells) if not lo <= c < hi and own_dofs & set(cd[c].tolist())]
            assert S.halo_cells(cd, m.n_dofs, lo, hi).tolist() == want


@pytest.mark.parametrize("dim", [2, 3])
def test_dof_owner_and_halo_plan(dim):
    m = small_mesh(dim)
    cd = m.cell_dofs
    world = 3
    b = S.cell_bounds(m.n_cells, world)
    own = S.dof_owners(cd, m.n_dofs, b)
    for d in range(m.n_dofs):
        cells = np.nonzero((cd == d).any(axis=1))[0]
        assert own[d] == S.owner_of_cells(cells, b).min()
    plans = [S.halo_plan(cd, m.n_dofs, b, r) for r in range(world)]
    for r in range(world):
        recv = plans[r][0]
        sent_to_r = np.sort(np.concatenate([plans[q][1][r] for q in range(world)]))
        assert sent_to_r.tolist() == recv.tolist()


def test_seed_ids_scan():
    assert S.seed_ids([3, 0, 5], 0, 100) == (100, 108)
    assert S.seed_ids([3, 0, 5], 1, 100) == (103, 108)
    assert S.seed_ids([3, 0, 5], 2, 100) == (103, 108)
    assert S.seed_ids([], 0, 7) == (7, 7)


@pytest.mark.parametrize("dim", [2, 3])
def test_projection_from_own_and_halo_cells_is_exact(dim):
    """Each DoF's sum over its cells needs only the partials of the cells
    around it: a rank that has its own cells' and its halo's partials gets
    the same values, bit for bit, on the DoFs it owns."""
    m = small_mesh(dim)
    cd = m.cell_dofs
    nv = cd.shape[1]
    rng = np.random.default_rng(3)
    part = rng.normal(size=(m.n_cells, nv, 2))
    part[..., 1] = np.abs(part[..., 1]) + 0.1

    def project(P):
        num = np.zeros(m.n_dofs)
        den = np.zeros(m.n_dofs)
        for c in range(m.n_cells):  # ascending cell order, as the device gather
            np.add.at(num, cd[c], P[c, :, 0])
            np.add.at(den, cd[c], P[c, :, 1])
        with np.errstate(invalid="ignore"):  # DoFs away from a rank's cells: 0/0
            return num / den

    full = project(part)
    world = 3
    b = S.cell_bounds(m.n_cells, world)
    own = S.dof_owners(cd, m.n_dofs, b)
    out = np.full(m.n_dofs, np.nan)
    for r in range(world):
        lo, hi = int(b[r]), int(b[r + 1])
        keep = np.zeros(m.n_cells, bool)
        keep[lo:hi] = True
        keep[S.halo_cells(cd, m.n_dofs, lo, hi)] = True
        mine = project(np.where(keep[:, None, None], part, 0.0))
        out[own == r] = mine[own == r]
    assert np.array_equal(out, full)


# ---------------------------------------------------------------------------
# the choreography, against a numpy stand-in of the partitioned C handle
# ---------------------------------------------------------------------------
class StandIn:
    """The partitioned C handle's contract in numpy, on a toy dynamics: a
    move shifts each particle by (id mod 3) cells (mod n_cells) and drops ids
    divisible by 11 in cell 0; count correction gives every own cell left
    empty one new particle (ids first_id + 1, ... in cell order); a cell's
    order is stayers (old order), arrivals by id, new particles; partial sums
    per cell and vertex are (sum v (j+1), count (j+1))."""

    def __init__(self, dim):
        self.dim = dim

    def initialize_maps(self, mesh, host_maps=False):
        self.m = mesh
        self.b, self.e = 0, mesh.n_cells
        self.over = {}

    def set_partition(self, b, e):
        self.b, self.e = b, e

    def close(self):
        pass

    def seed_particles(self, V):
        cells = np.repeat(np.arange(self.b, self.e), 2)
        n = len(cells)
        ids = (cells * 2 + np.tile([1, 2], self.e - self.b)).astype(np.uint32)
        vel = V[:, self.m.cell_dofs[cells, 0]].T.copy()
        self.P = S.Particles(ids, cells.astype(np.int32), np.zeros((n, self.dim)), np.full((n, self.dim), 0.5), vel)
        self.next_id = self.m.n_cells * 2
        self.Vlast = None

    def stats(self):
        return {"next_id": self.next_id, "n_particles": len(self.P)}

    def correct_particle_velocity_from_projection(self, V):
        d = self.m.cell_dofs[self.P.cell, 0]
        self.P.v = self.P.v + 0.25 * (V[:, d] - self.Vlast[:, d]).T

    def move_exchange_begin(self, V=None):
        P = self.P
        keep = ~((P.id % 11 == 0) & (P.cell == 0))
        P = P.take(keep)
        new = ((P.cell.astype(np.int64) + P.id % 3) % self.m.n_cells).astype(np.int32)
        self.stay = S.Particles(P.id, new, P.x, P.xi, P.v)
        self.moved = new != P.cell
        mine = (new >= self.b) & (new < self.e)
        self.out = self.stay.take(~mine)
        self.stay_mask = mine
        self.kept = self.stay.take(mine)
        self.kept_moved = self.moved[mine]
        return len(self.out)

    def move_outbox(self, n):
        assert n == len(self.out)
        return vars(self.out)

    def move_inbox(self, P):
        P = S._particles(P)
        assert ((P.cell >= self.b) & (P.cell < self.e)).all()
        self.arr = S.Particles.concat([self.kept.take(self.kept_moved), P], self.dim)
        self.stayers = self.kept.take(~self.kept_moved)
        present = set(self.stayers.cell.tolist()) | set(self.arr.cell.tolist())
        self.empty = [c for c in range(self.b, self.e) if c not in present]
        return len(self.empty)

    def move_exchange_end(self, first, nxt):
        parts = []
        for k, c in enumerate(range(self.b, self.e)):
            st = self.stayers.take(self.stayers.cell == c)
            ar = self.arr.take(self.arr.cell == c)
            ar = ar.take(np.argsort(ar.id, kind="stable"))
            parts += [st, ar]
            if c in self.empty:
                i = self.empty.index(c)
                parts.append(S.Particles(np.array([first + 1 + i], np.uint32), np.array([c], np.int32),
                                         np.zeros((1, self.dim)), np.full((1, self.dim), 0.5),
                                         np.ones((1, self.dim))))
        self.P = S.Particles.concat(parts, self.dim)
        self.next_id = nxt
        self.over = {}

    def _partials(self, c):
        nv = self.m.cell_dofs.shape[1]
        out = np.zeros(4 * nv)
        sel = self.P.cell == c
        for j in range(nv):
            out[4 * j:4 * j + self.dim] = self.P.v[sel].sum(axis=0) * (j + 1)
            out[4 * j + 3] = sel.sum() * (j + 1)
        return out

    def get_partials(self, cells):
        nv = self.m.cell_dofs.shape[1]
        return np.array([self._partials(c) for c in cells]).reshape(len(cells), 4 * nv)

    def set_partials(self, cells, vals):
        for c, v in zip(cells, vals):
            self.over[int(c)] = v

    def project_particle_fields(self):
        cd = self.m.cell_dofs
        num = np.zeros((self.dim, self.m.n_dofs))
        den = np.zeros(self.m.n_dofs)
        for c in range(self.m.n_cells):
            p = self.over.get(c) if not self.b <= c < self.e else self._partials(c)
            if p is None:
                continue
            for j in range(cd.shape[1]):
                num[:, cd[c, j]] += p[4 * j:4 * j + self.dim]
                den[cd[c, j]] += p[4 * j + 3]
        with np.errstate(invalid="ignore", divide="ignore"):
            self.Vlast = num / den
        return self.Vlast

    def particles(self):
        return {k: np.array(v) for k, v in vars(self.P).items()}


def run_choreography(comm, dim, steps=6):
    m = small_mesh(dim)
    V = np.stack([np.linspace(1.0, 2.0, m.n_dofs)] * dim)
    h = S.ShardedParticleHandler(dim, None, comm=comm, handler=StandIn(dim))
    h.initialize_maps(m)
    h.seed_particles(V)
    out = []
    U = h.project_particle_fields()
    for k in range(steps):
        U = h.step_solver(V * (1.0 + 0.1 * k))
        out.append((U, h.particles(), h.stats()))
    return out


def _rank(rank, world, port, dim, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = run_choreography(S.TorchComm(), dim)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dim,world", [(2, 2), (3, 3)])
def test_sharded_choreography_matches_one_handle_gloo(dim, world):
    want = run_choreography(S.LocalComm(), dim)
    port = 29500 + random.randint(0, 3000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, dim, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        got = dict(out)
    moved = 0
    for r in range(world):
        for (Uw, Pw, sw), (Ug, Pg, sg) in zip(want, got[r]):
            np.testing.assert_array_equal(Ug, Uw)
            for k in Pw:
                np.testing.assert_array_equal(Pg[k], Pw[k])
            assert sg["next_id"] == sw["next_id"] and sg["n_particles"] == sw["n_particles"]
            moved = sg["exchanged"]
    assert moved > 0  # particles did cross between ranks
