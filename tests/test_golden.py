"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py
from the FP64 oracle on small seeded cases: channel, duct, cylinder, cube).

CPU: the oracle still produces them bit for bit (a regression pin on the
checker itself).  GPU: the CUDA FP64 form reproduces every snapshot (ids,
cells, positions, reference coordinates, velocities, counters) bit for bit,
the projected velocity to 1e-12 and the window adjoint to 1e-10, from the
fixtures alone.
"""
import os

import numpy as np
import pytest

from . import cases
from .golden.make_golden import CASES, STAT_KEYS

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with np.load(os.path.join(HERE, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def by_id(P):
    o = np.argsort(P["id"], kind="stable")
    return {k: v[o] for k, v in P.items()}


def check_snapshot(G, prefix, P, st, exact=True):
    P = by_id(P)
    for k in ("id", "cell", "x", "xi", "v"):
        assert np.array_equal(G[prefix + k], P[k]), (prefix, k)
    assert np.array_equal(G[prefix + "stats"], np.array([st[k] for k in STAT_KEYS], np.int64)), prefix


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_golden(name):
    G = load(name)
    factory, steps, snaps = CASES[name]
    c = factory()
    o = cases.oracle_for(c)
    o.seed(c.V)
    check_snapshot(G, "s0_", o.particles(), o.stats())
    for s in range(1, steps + 1):
        U = o.step(c.V, c.Vold)
        if s in snaps:
            check_snapshot(G, f"s{s}_", o.particles(), o.stats())
            assert np.array_equal(G[f"s{s}_U"], U, equal_nan=True)
    K = int(G["win_K"])
    Uw, gv0, gV, gVo = o.window_adjoint(K, c.V, G["win_gU"], Vold=c.Vold)
    order = np.argsort(o.particles()["id"], kind="stable")
    assert np.array_equal(G["win_U"], Uw, equal_nan=True)
    assert np.array_equal(G["win_gv0"], gv0[order])
    assert np.array_equal(G["win_gV"], gV) and np.array_equal(G["win_gVold"], gVo)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_fp64_reproduces_golden(name):
    from pfem2dealii_b200.handler import ParticleHandler

    G = load(name)
    factory, steps, snaps = CASES[name]
    c = factory()
    g = ParticleHandler(c.mesh.dim, cases.params(c), "fp64")
    g.initialize_maps(c.mesh)
    g.seed_particles(c.V)
    check_snapshot(G, "s0_", g.particles(), g.stats())
    for s in range(1, steps + 1):
        U = g.step(c.V, c.Vold)
        if s in snaps:
            check_snapshot(G, f"s{s}_", g.particles(), g.stats())
            Ug = G[f"s{s}_U"]
            assert np.array_equal(np.isnan(Ug), np.isnan(U))
            m = np.isfinite(Ug)
            assert np.max(np.abs(Ug[m] - U[m])) <= 1e-12 * np.max(np.abs(Ug[m]))
    K = int(G["win_K"])
    Uw, gv0, gV, gVo = g.adjoint(K, 2, c.V, G["win_gU"], Vold=c.Vold)
    order = np.argsort(g.particles()["id"], kind="stable")
    m = np.isfinite(G["win_U"])
    assert np.array_equal(np.isnan(G["win_U"]), np.isnan(Uw))
    assert np.max(np.abs(G["win_U"][m] - Uw[m])) <= 1e-12 * np.max(np.abs(G["win_U"][m]))
    assert rel(gv0[order], G["win_gv0"]) <= 1e-10
    assert rel(gV, G["win_gV"]) <= 1e-10 and rel(gVo, G["win_gVold"]) <= 1e-10
    g.close()
