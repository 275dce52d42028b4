"""Cell-partitioned handlers on the GPU against one unpartitioned handle.

Two or three ranks (gloo process group, every rank's handle on cuda:0: the
exchange is host-driven, no kernel waits on another rank) run the solver's
data flow on a swirling field that carries particles across the partition
boundaries; their particles (gathered in cell order) and projections equal
one handle's bit for bit, in the FP64 and the FP32 form."""
import os
import random

import numpy as np
import pytest
import torch.multiprocessing as mp

from pfem2dealii_b200 import _lib
from pfem2dealii_b200 import mesh as M

from . import cases

pytestmark = pytest.mark.gpu

STEPS = 8


def swirl_case(dim):
    """A field with a transverse part, so particles cross the y-bands (2D)
    and z-slabs (3D) that contiguous cell ranges of a box mesh form."""
    if dim == 2:
        c = cases.channel(32, 12, dt=0.03)
    else:
        c = cases.duct(24, 6, 8, dt=0.01)

    def fn(x):
        u = np.zeros_like(x)
        u[:, 0] = 0.5 + 0.3 * np.cos(np.pi * x[:, 1])
        u[:, -1] = 0.6 * np.sin(np.pi * x[:, 0] / 2.0)
        if dim == 3:
            u[:, 1] = 0.2 * np.cos(np.pi * x[:, 2])
        return u

    c.V = M.field_at_dofs(c.mesh, fn)
    return c


def run(h, c, steps=STEPS):
    h.initialize_maps(c.mesh)
    h.seed_particles(c.V)
    U = h.project_particle_fields()
    out = [(U, h.particles())]
    for k in range(steps):
        U = h.step_solver(c.V * (1.0 + 0.05 * k))
        out.append((U, h.particles()))
    return out, h.stats()


def _rank(rank, world, port, dim, precision, out):
    import datetime

    import torch
    import torch.distributed as dist

    from pfem2dealii_b200.shard import ShardedParticleHandler, TorchComm

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        c = swirl_case(dim)
        h = ShardedParticleHandler(dim, cases.params(c), precision, comm=TorchComm())
        res, st = run(h, c)
        if rank == 0:
            out["res"] = res
        out[f"stats{rank}"] = st
        out[f"local{rank}"] = h.local_particles()["cell"]
        out[f"range{rank}"] = (h.begin, h.end)
        h.close()
    finally:
        dist.destroy_process_group()


def reference_run(dim, precision):
    from pfem2dealii_b200.handler import ParticleHandler

    c = swirl_case(dim)
    h = ParticleHandler(dim, cases.params(c), precision)
    res, st = run(h, c)
    h.close()
    return res, st


@pytest.mark.parametrize("dim,world,precision", [(2, 2, "fp64"), (2, 3, "fp32"), (3, 2, "fp64"), (3, 2, "fp32")])
def test_partitioned_equals_one_handle(dim, world, precision):
    want, wst = reference_run(dim, precision)
    port = 29500 + random.randint(0, 3000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, dim, precision, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(600)
            assert p.exitcode == 0
        got = dict(out)
    for k, ((Uw, Pw), (Ug, Pg)) in enumerate(zip(want, got["res"])):
        np.testing.assert_array_equal(Ug, Uw, err_msg=f"projection, step {k}")
        for key in Pw:
            np.testing.assert_array_equal(Pg[key], Pw[key], err_msg=f"particles' {key}, step {k}")
    st = got["stats0"]
    assert st["n_particles"] == wst["n_particles"] and st["next_id"] == wst["next_id"]
    assert st["exchanged"] > 100  # particles did cross between ranks
    for r in range(world):
        b, e = got[f"range{r}"]
        cells = got[f"local{r}"]
        assert ((cells >= b) & (cells < e)).all()


def test_one_rank_partition_equals_one_handle():
    from pfem2dealii_b200.shard import ShardedParticleHandler

    want, _ = reference_run(2, "fp64")
    c = swirl_case(2)
    got, _ = run(ShardedParticleHandler(2, cases.params(c), "fp64"), c)
    for (Uw, Pw), (Ug, Pg) in zip(want, got):
        np.testing.assert_array_equal(Ug, Uw)
        for key in Pw:
            np.testing.assert_array_equal(Pg[key], Pw[key])


def test_partition_errors():
    from pfem2dealii_b200.handler import ParticleHandler

    c = swirl_case(2)
    nC = c.mesh.n_cells
    h = ParticleHandler(2, cases.params(c))
    h.initialize_maps(c.mesh)
    with pytest.raises(_lib.Pfem2GpuError):
        h.set_partition(5, 2)
    with pytest.raises(_lib.Pfem2GpuError):
        h.set_partition(0, nC + 1)
    h.set_partition(0, nC // 2)
    h.seed_particles(c.V)
    assert set(np.unique(h.particles()["cell"]).tolist()) == set(range(nC // 2))
    with pytest.raises(_lib.Pfem2GpuError):
        h.set_partition(0, nC)  # after particles exist
    with pytest.raises(_lib.Pfem2GpuError):
        h.move_particles(c.V)  # a partitioned handle moves through the exchange
    with pytest.raises(_lib.Pfem2GpuError):
        h.move_inbox({"id": [], "cell": [], "x": np.zeros((0, 2)), "xi": np.zeros((0, 2)), "v": np.zeros((0, 2))})
    n = h.move_exchange_begin(c.V)
    P = h.move_outbox(n)
    assert ((P["cell"] >= nC // 2) & (P["cell"] < nC)).all()
    with pytest.raises(_lib.Pfem2GpuError):
        h.project_particle_fields()  # inside the move
    bad = {"id": np.array([7], np.uint32), "cell": np.array([nC - 1], np.int32), "x": np.zeros((1, 2)),
           "xi": np.full((1, 2), 0.5), "v": np.zeros((1, 2))}
    with pytest.raises(_lib.Pfem2GpuError):
        h.move_inbox(bad)  # a foreign cell
    h.move_inbox({k: v[:0] for k, v in bad.items()})
    h.move_exchange_end(10**6, 10**6 + 10)
    assert h.stats()["next_id"] == 10**6 + 10
    with pytest.raises(ValueError):
        h.set_partials([0, 1], np.zeros((1, 16)))
    p = h.get_partials([0, 1, nC - 1])
    assert p.shape == (3, 16) and np.all(p[2] == 0)
    h.set_partials([nC - 1], p[:1])
    assert np.array_equal(h.get_partials([nC - 1]), p[:1])
    h.close()
