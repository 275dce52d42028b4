"""bench.py under torchrun runs one replica per rank; its whole-job figures
are the max of the ranks' times and the sum of their particle-steps.  Two
gloo ranks on the CPU check that reduction (no GPU needed)."""
import os
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    ms, ps = bench.reduce_over_ranks(10.0 + rank, 1000 * (rank + 1), world, "cpu")
    out[rank] = (ms, ps)
    dist.destroy_process_group()


def test_reduce_over_ranks_two_gloo_ranks():
    import random

    world = 2
    port = 29500 + random.randint(0, 2000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1] == (11.0, 3000.0)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_over_ranks(3.5, 42, 1, "cpu") == (3.5, 42.0)
