"""Parity of the CUDA particle path (through the C ABI) with the FP64 oracle.

FP64 form: bit-exact.  Ids, cells, positions, reference coordinates and
velocities of every particle, and the lost/removed/seeded/searched counters,
equal the oracle's after every step; projected velocities agree to 1e-12
relative (only the summation order differs).  The oracle runs in id removal
order, the deterministic order the GPU implements.
FP32 form: relative L2 error against the FP64 oracle <= 1e-4 (projected
velocity) and <= 1e-5 (positions of particles alive in both).
"""
import numpy as np
import pytest

from oracle.oracle import ORDER_ID, ORDER_VECTOR
from pfem2dealii_b200 import mesh as M
from pfem2dealii_b200.handler import ParticleHandler

from . import cases
from .cases import by_id

pytestmark = pytest.mark.gpu

STAT_KEYS = ("lost", "removed", "seeded", "searched", "map_failures", "near_face", "n_particles", "next_id")
V_RTOL_FP64 = 1e-12
V_RTOL_FP32 = 1e-4
X_RTOL_FP32 = 1e-5


def make(case, precision="fp64", oracle_kw=None, **pkw):
    o = cases.oracle_for(case, **(oracle_kw or {}))
    g = ParticleHandler(case.mesh.dim, cases.params(case, **pkw), precision)
    g.initialize_maps(case.mesh)
    return o, g


def assert_same_particles(Po, Pg, exact=True):
    a, b = by_id(Po), by_id(Pg)
    assert np.array_equal(a["id"], b["id"])
    assert np.array_equal(a["cell"], b["cell"])
    for k in ("x", "xi", "v"):
        if exact:
            assert np.array_equal(a[k], b[k]), (k, np.max(np.abs(a[k] - b[k])))


def rel_l2(a, b):
    m = np.isfinite(a) & np.isfinite(b)
    return np.linalg.norm((a - b)[m]) / max(np.linalg.norm(a[m]), 1e-300)


def assert_v_close(Vo, Vg, rtol):
    assert np.array_equal(np.isnan(Vo), np.isnan(Vg))
    m = np.isfinite(Vo)
    scale = max(np.max(np.abs(Vo[m])), 1e-300) if m.any() else 1.0
    assert np.max(np.abs(Vo[m] - Vg[m])) <= rtol * scale


def run_fp64(case, steps, check_every=1, **pkw):
    o, g = make(case, **pkw)
    o.seed(case.V)
    g.seed_particles(case.V)
    assert_same_particles(o.particles(), g.particles())
    for s in range(steps):
        Vo = o.step(case.V, case.Vold)
        Vg = g.step(case.V, case.Vold)
        if (s + 1) % check_every == 0 or s == steps - 1:
            assert_same_particles(o.particles(), g.particles())
            so, sg = o.stats(), g.stats()
            for k in STAT_KEYS:
                assert so[k] == sg[k], (s, k, so[k], sg[k])
            assert so["nan_dofs"] == sg["nan_dofs"]
            assert_v_close(Vo, Vg, V_RTOL_FP64)
    return o, g


def test_fp64_channel_config_bit_exact():
    """2D channel 64x16, 16 ppc, max 2 per part, 4 sub-steps, dt 0.01, 100
    steps (the reference-size CPU case)."""
    o, g = run_fp64(cases.channel(), 100, check_every=10)
    st = g.stats()
    assert st["lost"] > 0 and st["seeded"] > 0 and st["searched"] > 0 and st["near_face"] > 0


def test_fp64_solver_data_flow_bit_exact():
    """The reference's data flow (src/pfem2solver.cpp:162-165 with fem_step
    copying the projection into the old solution, src/pfem2fem.cpp:523-524):
    every step corrects with Vold = the previous projection.  The host path
    (pfem2gpu_correct_from_projection, only V uploaded) and the device step
    (pfem2gpu_step_device with dVold NULL) both equal the oracle given the
    same Vold (the GPU's previous projection, which it keeps on the device),
    bit for bit; the projections agree to 1e-12 as everywhere (their
    summation orders differ), and the two GPU paths agree bit for bit."""
    import torch

    c = cases.channel(32, 8, dt=0.02)
    o, g = make(c)
    _, gd = make(c)
    o.seed(c.V)
    g.seed_particles(c.V)
    gd.seed_particles(c.V)
    Vo = o.project()
    Vg = g.project_particle_fields()
    dV = torch.from_numpy(np.ascontiguousarray(c.V)).cuda()
    dout = torch.empty_like(dV)
    gd.project_particle_fields_device(dout)
    assert_v_close(Vo, Vg, V_RTOL_FP64)
    for s in range(12):
        Vo = o.step(c.V, Vg)
        Vg = g.step_solver(c.V)
        gd.step_device(dV, None, dout)
        assert_same_particles(o.particles(), g.particles())
        assert_v_close(Vo, Vg, V_RTOL_FP64)
        assert np.array_equal(Vg, dout.cpu().numpy())
    assert_same_particles(o.particles(), gd.particles())
    # before any projection there is no previous one to correct from
    _, g2 = make(c)
    g2.seed_particles(c.V)
    with pytest.raises(Exception):
        g2.correct_particle_velocity_from_projection(c.V)
    for h in (g, gd, g2):
        h.close()


def test_fp64_duct_bit_exact():
    c = cases.duct(32, 8, 8, dt=0.05)
    o, g = run_fp64(c, 12)
    assert g.stats()["searched"] > 1000


def test_fp64_cylinder_unstructured_bit_exact():
    c = cases.cylinder(16, 8, 40, dt=0.01)
    o, g = run_fp64(c, 15)
    st = g.stats()
    assert st["searched"] > 0 and st["nan_dofs"] >= 0


def test_fp64_perturbed_cube_many_particles_per_cell():
    """64 particles per cell: cells span several warp passes; non-affine
    hexes exercise the 3D Newton inverse."""
    c = cases.cube(6, q=(4, 4, 4), dt=0.1)
    run_fp64(c, 6)


def test_fp64_many_arrivals_and_cells_beyond_64_particles():
    """64 particles per cell and a time step that carries particles across
    much of a cell: more than 32 arrivals into a cell (the overflow list
    beyond the per-cell arrival slots: up to 55 in this case) and cells of
    more than 64 old slots plus arrivals (the write pass's three-round and
    general paths)."""
    c = cases.channel(32, 8, q=(8, 8), maxpp=5, dt=0.1)
    run_fp64(c, 8)


@pytest.mark.parametrize("q,maxpp", [((6, 6), 1), ((7, 7), 0)])
def test_fp64_cells_of_33_to_64_particles(q, maxpp):
    """36 or 49 particles per cell: the write pass's two-round path (more
    than one warp's worth of particles), with arrivals and removals."""
    c = cases.channel(32, 8, q=q, maxpp=maxpp, dt=0.03)
    o, g = run_fp64(c, 10)
    st = g.stats()
    assert st["searched"] > 0


def test_fp64_first_touch_dofs_and_removal_seed():
    c = cases.channel(16, 8, q=(3, 2), dt=0.05)
    c.mesh = c.mesh.renumber_dofs_first_touch()
    c.V = M.field_at_dofs(c.mesh, M.channel_profile())
    c.Vold = 0.5 * c.V
    o, g = make(c, oracle_kw={"removal_seed": 987654321}, removal_seed=987654321)
    o.seed(c.V)
    g.seed_particles(c.V)
    for _ in range(10):
        Vo, Vg = o.step(c.V, c.Vold), g.step(c.V, c.Vold)
    assert_same_particles(o.particles(), g.particles())
    assert_v_close(Vo, Vg, V_RTOL_FP64)


@pytest.mark.parametrize("maxpp", [0, -1, 5])
def test_fp64_count_cap_variants(maxpp):
    c = cases.channel(16, 4, q=(2, 2), maxpp=maxpp, dt=0.1)
    run_fp64(c, 5)


def _crowd(case, cell, n, rng):
    """n particles crowded into one cell part plus a regular seeding."""
    X = case.mesh.vertices[case.mesh.cells[cell]]
    from oracle.oracle import forward_map

    xi = rng.uniform(0.01, 0.2, size=(n, case.mesh.dim))
    x = np.array([forward_map(X, z) for z in xi])
    return {"id": np.arange(1, n + 1, dtype=np.uint32), "cell": np.full(n, cell, np.int32), "x": x, "xi": xi,
            "v": rng.normal(size=(n, case.mesh.dim))}


def test_fp64_overfull_part_beyond_key_cache():
    """300 particles in one part (more than the per-warp key cache)."""
    c = cases.channel(8, 4, q=(4, 4), maxpp=2, dt=0.0)
    rng = np.random.default_rng(5)
    P = _crowd(c, 9, 300, rng)
    o, g = make(c)
    o.set_particles(P, 300)
    g.set_particles(P, 300)
    assert_same_particles(o.particles(), g.particles())
    Vo, Vg = o.step(c.V, c.V), g.step(c.V, c.V)
    so, sg = o.stats(), g.stats()
    assert so["removed"] == sg["removed"] == 297 and so["seeded"] == sg["seeded"] == 15
    assert_same_particles(o.particles(), g.particles())
    assert_v_close(Vo, Vg, V_RTOL_FP64)
    assert np.isnan(Vg).any()  # DoFs far from the crowded cell have no weight


def test_fp64_correct_then_project_without_move():
    c = cases.duct(8, 4, 4, dt=0.01)
    o, g = make(c)
    o.seed(c.V)
    g.seed_particles(c.V)
    o.correct(c.V, c.Vold)
    g.correct_particle_velocity(c.V, c.Vold)
    assert_v_close(o.project(), g.project_particle_fields(), V_RTOL_FP64)
    assert_same_particles(o.particles(), g.particles())


def test_fp64_project_after_removals_ignores_empty_slots():
    """A step that removes particles leaves empty slots in the cell's range;
    a correct + project with no move in between must not count them."""
    c = cases.channel(8, 4, q=(4, 4), maxpp=2, dt=0.0)
    P = _crowd(c, 9, 300, np.random.default_rng(6))
    o, g = make(c)
    o.set_particles(P, 300)
    g.set_particles(P, 300)
    o.step(c.V, c.V)
    g.step(c.V, c.V)
    assert g.stats()["removed"] == 297
    o.correct(c.V, 0.5 * c.V)
    g.correct_particle_velocity(c.V, 0.5 * c.V)
    assert_v_close(o.project(), g.project_particle_fields(), V_RTOL_FP64)
    assert_same_particles(o.particles(), g.particles())


def test_fp64_empty_dof_policy_keeps_input():
    c = cases.channel(8, 4, dt=0.0)
    P = _crowd(c, 0, 5, np.random.default_rng(1))
    _, g = make(c, empty_dof_policy=1)
    g.set_particles(P, 5)
    g.move_particles(c.V)
    Vg = g.project_particle_fields()
    assert not np.isnan(Vg).any()
    far = np.setdiff1d(np.arange(c.mesh.n_dofs), c.mesh.cell_dofs[0])
    assert np.array_equal(Vg[:, far], c.V[:, far])


def test_vector_order_oracle_agrees_on_counts():
    """The reference's own (vector) removal order picks other survivors but
    the same per-cell counts, seeds and losses as the GPU."""
    c = cases.channel(32, 8, q=(3, 3), maxpp=1, dt=0.02)
    o, g = make(c, oracle_kw={"removal_order": ORDER_VECTOR})
    o.seed(c.V)
    g.seed_particles(c.V)
    o.step(c.V, c.Vold)
    g.step(c.V, c.Vold)
    a, b = o.particles(), g.particles()
    assert np.array_equal(np.bincount(a["cell"], minlength=c.mesh.n_cells),
                          np.bincount(b["cell"], minlength=c.mesh.n_cells))
    for k in ("lost", "removed", "seeded"):
        assert o.stats()[k] == g.stats()[k]


@pytest.mark.parametrize("which", ["channel", "duct", "cylinder", "cube"])
def test_fp32_error_against_fp64_oracle(which):
    # the cube seeds 64 particles per cell: its write pass stages by plain loads
    c = {"channel": lambda: cases.channel(),
         "duct": lambda: cases.duct(32, 8, 8, dt=0.02),
         "cylinder": lambda: cases.cylinder(24, 12, 60, dt=2e-3),
         "cube": lambda: cases.cube(6, q=(4, 4, 4), dt=0.05)}[which]()
    o, g = make(c, precision="fp32")
    o.seed(c.V)
    g.seed_particles(c.V)
    for _ in range(20):
        Vo = o.step(c.V, c.Vold)
        Vg = g.step(c.V, c.Vold)
    assert np.array_equal(np.isnan(Vo), np.isnan(Vg)) or rel_l2(Vo, Vg) < V_RTOL_FP32
    assert rel_l2(Vo, Vg) <= V_RTOL_FP32
    a, b = by_id(o.particles()), by_id(g.particles())
    common, ia, ib = np.intersect1d(a["id"], b["id"], return_indices=True)
    assert len(common) >= 0.99 * len(a["id"])
    assert rel_l2(a["x"][ia], b["x"][ib]) <= X_RTOL_FP32
    assert abs(len(a["id"]) - len(b["id"])) <= 0.01 * len(a["id"])


def test_vtu_output(tmp_path):
    c = cases.channel(8, 4, q=(2, 2))
    _, g = make(c)
    g.seed_particles(c.V)
    g.output_particle_solution(3, str(tmp_path))
    text = (tmp_path / "particles-03.000.vtu").read_text()
    assert 'NumberOfPoints="128"' in text and "<VTKFile" in text
    assert (tmp_path / "particles-03.pvtu").exists()


@pytest.mark.parametrize("which", ["duct", "cube"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_step_device_graph_replay(precision, which):
    """pfem2gpu_step_device (eager first call, captured second, replayed
    afterwards) gives the oracle's particles, bit-exact in FP64; a new output
    pointer re-captures; the result matches the separate host calls."""
    import torch

    c = cases.duct(32, 8, 8, dt=0.05) if which == "duct" else cases.cube(6, q=(4, 4, 4), dt=0.05)
    o, g = make(c, precision)
    _, h = make(c, precision)
    o.seed(c.V)
    g.seed_particles(c.V)
    h.seed_particles(c.V)
    dV = torch.tensor(c.V, device="cuda")
    dVo = torch.tensor(c.Vold, device="cuda")
    outs = [torch.empty_like(dV), torch.empty_like(dV)]
    for s in range(8):
        Vo = o.step(c.V, c.Vold)
        Vh = h.step(c.V, c.Vold)
        out = outs[s // 5]
        g.step_device(dV, dVo, out)
        g.synchronize()  # the handler's stream is not torch's current stream
        Vg = out.cpu().numpy()
        if precision == "fp64":
            assert_same_particles(o.particles(), g.particles())
            so, sg = o.stats(), g.stats()
            for k in STAT_KEYS:
                assert so[k] == sg[k], (s, k, so[k], sg[k])
            assert_v_close(Vo, Vg, V_RTOL_FP64)
        else:
            assert rel_l2(Vo, Vg) <= V_RTOL_FP32
        assert np.array_equal(np.isnan(Vh), np.isnan(Vg))
        m = np.isfinite(Vh)
        assert np.array_equal(Vh[m], Vg[m])
        assert_same_particles(h.particles(), g.particles())


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("which", ["channel", "duct", "cylinder"])
def test_pack_output_matches_particles(precision, which):
    """pfem2gpu_pack_output_device: the live particles' positions and
    velocities as Float32, in get_particles order (empty slots skipped:
    the runs include removals and losses)."""
    import torch

    c = {"channel": lambda: cases.channel(16, 4, q=(4, 4), maxpp=0, dt=0.03),
         "duct": lambda: cases.duct(16, 4, 4, maxpp=0, dt=0.05),
         "cylinder": lambda: cases.cylinder(24, 12, 60, dt=4e-3)}[which]()
    _, g = make(c, precision)
    g.seed_particles(c.V)
    for _ in range(4):
        g.step(c.V, c.Vold)
    assert g.stats()["removed"] > 0 or which == "cylinder"
    out, n = g.pack_output_device()
    g.synchronize()
    P = g.particles()
    assert n == len(P["id"])
    o = out.cpu().numpy()
    dim = c.mesh.dim
    x = o[: 3 * n].reshape(n, 3)
    v = o[3 * n: 6 * n].reshape(n, 3)
    assert np.array_equal(x[:, :dim], P["x"].astype(np.float32))
    assert np.array_equal(v[:, :dim], P["v"].astype(np.float32))
    if dim == 2:
        assert not x[:, 2].any() and not v[:, 2].any()


def _maps_case(which):
    if which == "cube_big":
        return cases.cube(n=96)
    return getattr(cases, which)()


@pytest.mark.parametrize("which", ["channel", "duct", "cylinder", "cube", "cube_big"])
def test_device_vertex_maps_equal_host_builder(which):
    """initialize_maps built on the device (src/pfem2particlehandler.cpp:320-324):
    offsets and ascending cells equal mesh.vertex_maps, the unit directions
    bit for bit."""
    case = _maps_case(which)
    g = ParticleHandler(case.mesh.dim, cases.params(case), "fp64")
    g.initialize_maps(case.mesh)
    off, cells, dirs = g.vertex_maps()
    o2, c2, d2 = M.vertex_maps(case.mesh)
    assert np.array_equal(off, o2)
    assert np.array_equal(cells, c2)
    assert dirs.shape == d2.shape and dirs.tobytes() == d2.tobytes()
    g.close()


def test_given_vertex_maps_kept_and_runs_identical():
    """Maps passed by the caller are used as given; a run on them equals the
    run on device-built maps bit for bit."""
    case = cases.cylinder()
    runs = []
    for host_maps in (True, False):
        g = ParticleHandler(case.mesh.dim, cases.params(case), "fp64")
        g.initialize_maps(case.mesh, host_maps=host_maps)
        if host_maps:
            off, cells, dirs = g.vertex_maps()
            o2, c2, d2 = M.vertex_maps(case.mesh)
            assert np.array_equal(off, o2) and np.array_equal(cells, c2) and dirs.tobytes() == d2.tobytes()
        g.seed_particles(case.V)
        for _ in range(5):
            U = g.step(case.V, case.Vold)
        runs.append((by_id(g.particles()), U))
        g.close()
    (a, Ua), (b, Ub) = runs
    for k in ("id", "cell", "x", "xi", "v"):
        assert np.array_equal(a[k], b[k]), k
    assert Ua.tobytes() == Ub.tobytes()


def test_device_vertex_maps_collapsed_cell():
    """A cell listing one vertex twice counts it once (the map is a set per
    vertex), as GridTools::vertex_to_cell_map does."""
    verts = np.array([[0, 0], [1, 0], [0, 1], [1, 1], [2, 0], [2, 1]], np.float64)
    cells = np.array([[0, 1, 2, 3], [1, 4, 3, 3]], np.int32)
    m = M.Mesh(2, verts, cells, cells.copy(), verts.shape[0], "collapsed")
    g = ParticleHandler(2, cases.params(cases.channel()), "fp64")
    g.initialize_maps(m)
    off, cl, dirs = g.vertex_maps()
    o2, c2, d2 = M.vertex_maps(m)
    assert np.array_equal(off, o2) and np.array_equal(cl, c2) and dirs.tobytes() == d2.tobytes()
    assert off[4] - off[3] == 2
    g.close()


# The opt-in RK2 sub-step (PFEM2GPU_RK2; the reference has Euler only): the
# FP64 form equals the oracle's RK2 bit for bit, on affine and non-affine
# meshes; the FP32 form stays within the FP32 tolerances of the oracle.
RK2 = {"oracle_kw": {"integrator": 1}, "integrator": 1}


@pytest.mark.parametrize("which", ["channel", "cylinder", "cube"])
def test_fp64_rk2_bit_exact(which):
    c = {"channel": lambda: cases.channel(32, 8, dt=0.02),
         "cylinder": lambda: cases.cylinder(16, 8, 40, dt=0.01),
         "cube": lambda: cases.cube(5, q=(3, 3, 3), dt=0.1)}[which]()
    o, g = run_fp64(c, 10, **RK2)
    assert g.stats()["searched"] > 0


@pytest.mark.parametrize("which", ["channel", "cylinder", "duct"])
def test_fp32_rk2_error_against_fp64_oracle(which):
    c = {"channel": lambda: cases.channel(),
         "cylinder": lambda: cases.cylinder(24, 12, 60, dt=2e-3),
         "duct": lambda: cases.duct(32, 8, 8, dt=0.02)}[which]()
    o, g = make(c, precision="fp32", **RK2)
    o.seed(c.V)
    g.seed_particles(c.V)
    for _ in range(20):
        Vo = o.step(c.V, c.Vold)
        Vg = g.step(c.V, c.Vold)
    assert rel_l2(Vo, Vg) <= V_RTOL_FP32
    a, b = by_id(o.particles()), by_id(g.particles())
    common, ia, ib = np.intersect1d(a["id"], b["id"], return_indices=True)
    assert len(common) >= 0.99 * len(a["id"])
    assert rel_l2(a["x"][ia], b["x"][ib]) <= X_RTOL_FP32


def test_rk2_differs_from_euler_and_window_refuses_it():
    import torch

    c = cases.channel(16, 4, dt=0.05)
    out = {}
    for integ in (0, 1):
        _, g = make(c, integrator=integ)
        g.seed_particles(c.V)
        out[integ] = g.step(c.V, c.Vold)
        if integ == 1:
            dV = torch.from_numpy(np.ascontiguousarray(c.V)).cuda()
            with pytest.raises(Exception):
                g.window_forward_device(2, 1, dV)
        g.close()
    assert not np.array_equal(out[0], out[1], equal_nan=True)
