"""Failure detection at the boundary: bad input is refused with a status code
before any device work, and the handle stays as it was.

The reference stops on bad input with deal.II assertions
(src/pfem2particlehandler.cpp:515-519) and otherwise lets NaN propagate;
here every refused call returns its code, the counters and particles are
unchanged, and the next valid call gives the same result as a handle that
never saw the bad one.  The failures are made on the host (wrong sizes,
values and states); no test makes a kernel fault or wait."""
import numpy as np
import pytest

from pfem2dealii_b200 import _lib
from pfem2dealii_b200.handler import ParticleHandler, ParticleParams

from . import cases

pytestmark = pytest.mark.gpu


def small_case():
    return cases.channel(16, 4, dt=0.02)


def handler(case, **kw):
    g = ParticleHandler(case.mesh.dim, cases.params(case, **kw), "fp64")
    g.initialize_maps(case.mesh)
    return g


def code_of(fn, *a):
    with pytest.raises(_lib.Pfem2GpuError) as e:
        fn(*a)
    return e.value.code


def test_capacity_below_the_seeded_particles():
    """params.capacity is a limit: seeding more particles than it allows is
    PFEM2GPU_ERR_CAPACITY, with nothing seeded; particles that fit can still
    be set."""
    c = small_case()
    n_seed = c.mesh.n_cells * 16
    g = handler(c, capacity=n_seed // 2)
    assert code_of(g.seed_particles, c.V) == _lib.ERR_CAPACITY
    assert g.stats()["n_particles"] == 0
    ref = handler(c)
    ref.seed_particles(c.V)
    P = ref.particles()
    k = n_seed // 4
    sub = {key: val[:k] for key, val in P.items()}
    g.set_particles(sub, int(P["id"].max()))
    assert g.stats()["n_particles"] == k
    assert code_of(g.set_particles, P, int(P["id"].max())) == _lib.ERR_CAPACITY
    assert g.stats()["n_particles"] == k
    g.close()
    ref.close()


def test_set_particles_bad_input_leaves_the_particles():
    c = small_case()
    g = handler(c)
    g.seed_particles(c.V)
    g.step(c.V, c.Vold)
    before, st = g.particles(), g.stats()
    nid = st["next_id"]
    for field, value, code in (("cell", c.mesh.n_cells, _lib.ERR_ARG), ("cell", -1, _lib.ERR_ARG),
                               ("xi", 1.5, _lib.ERR_ARG), ("xi", np.nan, _lib.ERR_ARG),
                               ("v", np.inf, _lib.ERR_ARG), ("x", np.nan, _lib.ERR_ARG)):
        bad = {k: v.copy() for k, v in before.items()}
        bad[field][len(bad[field]) // 2] = value
        assert code_of(g.set_particles, bad, nid) == code, (field, value)
        after = g.particles()
        for k in before:
            assert np.array_equal(before[k], after[k]), (field, k)
        assert g.stats() == st
    g.close()


def test_non_finite_nodal_velocity_is_refused():
    """NaN or Inf in the FEM velocity given to seed, correct or move:
    PFEM2GPU_ERR_ARG before anything is copied; the following valid steps
    equal those of a handle that never saw the bad calls, bit for bit."""
    c = small_case()
    bad = c.V.copy()
    bad[1, 7] = np.nan
    g = handler(c)
    assert code_of(g.seed_particles, bad) == _lib.ERR_ARG
    assert g.stats()["n_particles"] == 0
    g.seed_particles(c.V)
    ref = handler(c)
    ref.seed_particles(c.V)
    bad[1, 7] = np.inf
    for k in range(3):
        assert code_of(g.correct_particle_velocity, bad, c.Vold) == _lib.ERR_ARG
        assert code_of(g.move_particles, bad) == _lib.ERR_ARG
        Vg = g.step(c.V, c.Vold)
        Vr = ref.step(c.V, c.Vold)
        assert np.array_equal(Vg, Vr, equal_nan=True)
    Pg, Pr = g.particles(), ref.particles()
    for k in Pg:
        assert np.array_equal(Pg[k], Pr[k])
    assert g.stats() == ref.stats()
    g.close()
    ref.close()


def test_calls_out_of_order():
    c = small_case()
    g = handler(c)
    assert code_of(g.move_particles, c.V) == _lib.ERR_STATE
    assert code_of(g.project_particle_fields) == _lib.ERR_STATE
    assert code_of(g.correct_particle_velocity_from_projection, c.V) == _lib.ERR_STATE
    g.seed_particles(c.V)
    assert code_of(g.seed_particles, c.V) == _lib.ERR_STATE  # seeding twice
    assert code_of(g.correct_particle_velocity_from_projection, c.V) == _lib.ERR_STATE  # no projection yet
    g.project_particle_fields()
    g.correct_particle_velocity_from_projection(c.V)
    g.close()
    h = ParticleHandler(2, ParticleParams(particles_per_cell=(2, 2)), "fp64")
    assert code_of(h.seed_particles, c.V) == _lib.ERR_STATE  # no mesh
    h.close()
