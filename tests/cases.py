"""Test workloads: meshes, velocity fields and particle parameters of the
benchmark configurations (reduced sizes for the oracle, full sizes for
property tests), built identically for the oracle and the GPU handler."""
from __future__ import annotations

import dataclasses
import os

import numpy as np

from pfem2dealii_b200 import mesh as M


@dataclasses.dataclass
class Case:
    name: str
    mesh: M.Mesh
    V: np.ndarray
    Vold: np.ndarray
    q: tuple
    max_per_part: int
    substeps: int
    dt: float


def channel(nx=64, ny=16, q=(4, 4), maxpp=2, S=4, dt=0.01, old_scale=0.9):
    """2D channel [0,4]x[0,1], parabolic inflow u = 4y(1-y)."""
    m = M.hyper_rectangle((0.0, 0.0), (4.0, 1.0), (nx, ny), "channel")
    V = M.field_at_dofs(m, M.channel_profile(1.0, 1.0))
    return Case("channel", m, V, old_scale * V, q, maxpp, S, dt)


def duct(nx=128, ny=32, nz=32, q=(3, 3, 3), maxpp=2, S=3, dt=2e-3, old_scale=0.9):
    """3D duct [0,8]x[0,1]^2, u = 16 y(1-y) z(1-z)."""
    m = M.hyper_rectangle((0.0, 0.0, 0.0), (8.0, 1.0, 1.0), (nx, ny, nz), "duct")
    V = M.field_at_dofs(m, M.duct_profile(1.0))
    return Case("duct", m, V, old_scale * V, q, maxpp, S, dt)


def cylinder(n_t=96, n_r=48, n_x=480, q=(4, 4), maxpp=2, S=3, dt=5e-4, old_scale=0.9):
    """2D channel with a cylinder (synthetic Turek-like mesh), Umax = 1.5."""
    m = M.turek_channel(n_t, n_r, n_x)
    V = M.field_at_dofs(m, M.cylinder_inflow(1.5))
    return Case("cylinder", m, V, old_scale * V, q, maxpp, S, dt)


MESH3 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "Mesh3.tgz")


def turek_mesh3(q=(4, 4), maxpp=2, S=3, dt=5e-4, old_scale=0.9):
    """The reference's Turek benchmark mesh (cases/TurekBenchmark/Mesh3.tgz:
    60,450 quads around a cylinder of radius 0.05 at (0.2, 0.2) in the
    2.2 x 0.41 channel) with the parabolic inflow of Umax 1.5
    (cases/TurekBenchmark/TurekBenchmark.cc:6-9), zero on the walls and the
    cylinder."""
    m = M.read_unv_native(MESH3)
    V = M.field_at_dofs(m, M.cylinder_inflow(1.5))
    return Case("turek_mesh3", m, V, old_scale * V, q, maxpp, S, dt)


def noisy_start(case, sigma=0.01, seed=0):
    """The case's seeded particles (FP64 form) with N(0, sigma) added to each
    velocity component, drawn in id order: the initial particle velocities
    of the Turek configuration.  Returns (particles, next_id) for
    ParticleHandler.set_particles."""
    from pfem2dealii_b200.handler import ParticleHandler

    g = ParticleHandler(case.mesh.dim, params(case), "fp64")
    g.initialize_maps(case.mesh)
    g.seed_particles(case.V)
    P = g.particles()
    nid = g.stats()["next_id"]
    g.close()
    order = np.argsort(P["id"])
    P["v"] = P["v"].copy()
    P["v"][order] += np.random.default_rng(seed).normal(0.0, sigma, size=P["v"].shape)
    return P, nid


def cube(n=80, q=(4, 4, 4), maxpp=2, S=3, dt=1e-3, amplitude=0.1, seed=0, old_scale=0.9):
    """Perturbed [0,2pi]^3 cube, Taylor-Green-type divergence-free field."""
    m = M.perturbed_cube(n, amplitude=amplitude, seed=seed)
    V = M.field_at_dofs(m, M.taylor_green_3d())
    return Case("cube", m, V, old_scale * V, q, maxpp, S, dt)


def params(case: Case, **kw):
    from pfem2dealii_b200.handler import ParticleParams

    return ParticleParams(particles_per_cell=case.q, max_particles_per_cell_part=case.max_per_part,
                          particle_integration_steps=case.substeps, time_step=case.dt, **kw)


def oracle_for(case: Case, **kw):
    from oracle.oracle import Oracle

    return Oracle(case.mesh, case.q, case.max_per_part, case.substeps, case.dt, **kw)


def by_id(P):
    o = np.argsort(P["id"], kind="stable")
    return {k: v[o] for k, v in P.items()}
