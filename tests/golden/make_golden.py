"""Generates the golden fixtures of tests/golden/ from the FP64 oracle.

The reference itself cannot be built or run here (it needs deal.II >= 9.4
with p4est, Trilinos and MPI) and ships no golden vectors, so these
fixtures are the oracle's own outputs on small seeded cases: they pin the
oracle against regressions (tests/test_golden.py, CPU) and the CUDA FP64
form against them bit for bit (tests/test_golden.py, GPU), without running
the oracle at test time.  Parity with the reference stays unpinned.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests import cases  # noqa: E402


def snapshot(o, prefix, out):
    P = o.particles()
    order = np.argsort(P["id"], kind="stable")
    for k in ("id", "cell", "x", "xi", "v"):
        out[f"{prefix}{k}"] = P[k][order]
    st = o.stats()
    out[f"{prefix}stats"] = np.array([st[k] for k in STAT_KEYS], np.int64)


STAT_KEYS = ("n_particles", "lost", "removed", "seeded", "searched", "map_failures", "near_face", "nan_dofs",
             "next_id")

CASES = {
    # name: (case factory, steps, snapshot steps)
    "channel": (lambda: cases.channel(16, 4, q=(4, 4), maxpp=2, S=4, dt=0.047), 12, (1, 6, 12)),
    "duct": (lambda: cases.duct(8, 4, 4, q=(3, 3, 3), maxpp=2, S=3, dt=0.03), 6, (1, 6)),
    "cylinder": (lambda: cases.cylinder(12, 6, 20, q=(4, 4), maxpp=2, S=3, dt=5e-3), 6, (6,)),
    "cube": (lambda: cases.cube(4, q=(2, 2, 2), maxpp=1, S=3, dt=0.05), 4, (4,)),
}


def make(name):
    factory, steps, snaps = CASES[name]
    c = factory()
    o = cases.oracle_for(c)
    out = {"steps": np.array(steps), "snaps": np.array(snaps)}
    o.seed(c.V)
    snapshot(o, "s0_", out)
    for s in range(1, steps + 1):
        U = o.step(c.V, c.Vold)
        if s in snaps:
            snapshot(o, f"s{s}_", out)
            out[f"s{s}_U"] = U
    # the differentiated window from the final state
    K = 3
    U = o.window_forward(K, c.V, c.Vold)
    rng = np.random.default_rng(5)
    finite = np.where(np.all(np.isfinite(U), 0))[0]
    probe = rng.choice(finite, min(8, len(finite)), replace=False)
    gU = np.zeros_like(U)
    gU[:, probe] = 2.0 * (U[:, probe] - (U[:, probe] + 0.01))
    Uw, gv0, gV, gVo = o.window_adjoint(K, c.V, gU, Vold=c.Vold)
    P = o.particles()
    order = np.argsort(P["id"], kind="stable")
    out.update({"win_K": np.array(K), "win_gU": gU, "win_U": Uw, "win_gv0": gv0[order], "win_gV": gV,
                "win_gVold": gVo})
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


if __name__ == "__main__":
    from oracle import oracle

    oracle.build()
    for n in CASES:
        make(n)
        print(n, os.path.getsize(os.path.join(HERE, f"{n}.npz")), "bytes")
