"""Known-answer tests of the FP64 oracle (CPU).

The reference ships no tests or golden data, so the oracle is pinned by
mathematics: Q1 reproduction, exact Euler transport on affine cells,
partition of unity in the projection, the seeding pattern, the count cap
(max+1 survivors per part, src/pfem2particlehandler.cpp:372), the
relocation's search confined to the cells around the closest vertex, and
inverse/forward map round trips.
"""
import io
import os

import numpy as np
import pytest

from oracle.oracle import ORDER_ID, ORDER_VECTOR, Oracle, forward_map, inverse_map, key, shape_values
from pfem2dealii_b200 import mesh as M

from . import cases


def test_shape_partition_and_linear_reproduction():
    rng = np.random.default_rng(1)
    for dim in (2, 3):
        corners = np.array([[(i >> d) & 1 for d in range(dim)] for i in range(1 << dim)], float)
        a = rng.normal(size=dim)
        for _ in range(50):
            xi = rng.uniform(0, 1, dim)
            N = shape_values(dim, xi)
            assert abs(N.sum() - 1) < 1e-15
            # multilinear field reproduced: f = a.xi + xi0*xi1
            f = corners @ a + corners[:, 0] * corners[:, 1]
            assert abs(N @ f - (a @ xi + xi[0] * xi[1])) < 1e-14


def _random_cell(rng, dim, jitter):
    X = np.array([[(i >> d) & 1 for d in range(dim)] for i in range(1 << dim)], float)
    return X + rng.uniform(-jitter, jitter, X.shape)


@pytest.mark.parametrize("dim", [2, 3])
def test_inverse_map_round_trip(dim):
    rng = np.random.default_rng(dim)
    for _ in range(200):
        X = _random_cell(rng, dim, 0.2) * rng.uniform(0.01, 10) + rng.normal(size=dim)
        xi = rng.uniform(0, 1, dim)
        p = forward_map(X, xi)
        back = inverse_map(X, p)
        assert back is not None
        assert np.max(np.abs(back - xi)) < 1e-10


def test_inverse_map_outside_point():
    X = np.array([[0, 0], [1, 0], [0, 1], [1, 1]], float)
    back = inverse_map(X, np.array([1.5, 0.25]))
    assert back is not None and abs(back[0] - 1.5) < 1e-14  # affine: exact, outside
    X3 = _random_cell(np.random.default_rng(0), 3, 0.1)
    p = forward_map(X3, np.array([1.2, 0.5, -0.1]))
    b = inverse_map(X3, p)
    assert b is not None and np.allclose(b, [1.2, 0.5, -0.1], atol=1e-9)


def test_key_is_identity_without_seed_and_bijective_with_seed():
    assert [key(i, 0) for i in range(5)] == [0, 1, 2, 3, 4]
    ks = {key(i, 12345) for i in range(20000)}
    assert len(ks) == 20000


def _channel(nx=16, ny=4):
    return M.hyper_rectangle((0.0, 0.0), (4.0, 1.0), (nx, ny))


def test_seeding_pattern():
    m = _channel()
    V = M.field_at_dofs(m, M.channel_profile())
    o = Oracle(m, (4, 3), 2, 4, 0.01)
    o.seed(V)
    P = o.particles()
    assert len(P["id"]) == m.n_cells * 12
    assert np.array_equal(P["id"], np.arange(1, m.n_cells * 12 + 1))
    assert np.array_equal(np.bincount(P["cell"]), np.full(m.n_cells, 12))
    xi = P["xi"][:12]
    exp = np.array([[(i + 0.5) / 4, (j + 0.5) / 3] for i in range(4) for j in range(3)])  # x outermost
    assert np.allclose(xi, exp, atol=1e-15)
    # location = F(xi) and velocity = interpolated V
    X = m.vertices[m.cells[P["cell"]]]
    xq = np.einsum("pi,pid->pd", np.array([shape_values(2, z) for z in P["xi"]]), X)
    assert np.allclose(P["x"], xq, atol=1e-14)
    N = np.array([shape_values(2, z) for z in P["xi"]])
    vq = np.einsum("pi,dpi->pd", N, V[:, m.cell_dofs[P["cell"]]])
    assert np.allclose(P["v"], vq, atol=1e-15)


@pytest.mark.parametrize("dim", [2, 3])
def test_uniform_flow_is_exact_on_affine_cells(dim):
    if dim == 2:
        m = M.hyper_rectangle((0.0, 0.0), (2.0, 1.0), (8, 4))
        u = np.array([0.3, -0.1])
    else:
        m = M.hyper_rectangle((0.0, 0.0, 0.0), (2.0, 1.0, 1.0), (6, 3, 3))
        u = np.array([0.3, -0.1, 0.05])
    V = np.repeat(u[:, None], m.n_dofs, axis=1)
    o = Oracle(m, (2,) * dim, 100, 3, 0.05)
    o.seed(V)
    P0 = o.particles()
    o.move(V)
    P1 = o.particles()
    alive = np.isin(P0["id"], P1["id"])
    x0 = P0["x"][alive][np.argsort(P0["id"][alive])]
    x1 = P1["x"][np.isin(P1["id"], P0["id"])]
    x1 = x1[np.argsort(P1["id"][np.isin(P1["id"], P0["id"])])]
    assert np.allclose(x1, x0 + u * 0.05, atol=1e-13)
    # relocated reference coordinates are consistent with the positions
    X = m.vertices[m.cells[P1["cell"]]]
    xq = np.einsum("pi,pid->pd", np.array([shape_values(dim, z) for z in P1["xi"]]), X)
    assert np.allclose(xq, P1["x"], atol=1e-13)
    assert np.all((P1["xi"] >= 0) & (P1["xi"] <= 1))


@pytest.mark.parametrize("shift, survivors", [(0.7, "neighbour"), (1.7, "none")])
def test_relocation_searches_only_the_closest_vertex_patch(shift, survivors):
    """One particle per cell at its centre, a uniform flow along x moving each
    by `shift` cells in one sub-step.  0.7 cells: every particle leaves its
    cell through the face ahead and is found in the next cell, which holds
    the vertices of that face (src/pfem2particlehandler.cpp:413-503 with
    src/pfem2particle.cpp:186-211); the last column leaves the mesh.  1.7
    cells: the particle lands two cells ahead, outside the cells around the
    closest vertex of its old cell, and is deleted although it is inside
    the mesh: the reference searches no further."""
    nx, ny, h = 8, 2, 0.5
    m = M.hyper_rectangle((0.0, 0.0), (nx * h, ny * h), (nx, ny))
    u = shift * h / 0.1
    V = np.repeat(np.array([u, 0.0])[:, None], m.n_dofs, axis=1)
    o = Oracle(m, (1, 1), 100, 1, 0.1)
    o.seed(V)
    P0 = o.particles()
    o.move(V)
    P1 = o.particles()
    st = o.stats()
    if survivors == "neighbour":
        assert st["lost"] == ny
        assert len(P1["id"]) == (nx - 1) * ny
        for i, c in zip(P1["id"], P1["cell"]):
            c0 = P0["cell"][P0["id"] == i][0]
            x0 = m.vertices[m.cells[c0]].mean(0)
            xc = m.vertices[m.cells[c]]
            assert np.all(xc.min(0) <= x0 + [shift * h, 0.0]) and np.all(x0 + [shift * h, 0.0] <= xc.max(0))
            assert np.isclose(xc.min(0)[0] - x0[0], 0.5 * h)  # the next cell along x
        assert np.allclose(P1["xi"][:, 0], 0.2, atol=1e-12)
    else:
        assert len(P1["id"]) == 0
        assert st["lost"] == nx * ny


def test_projection_partition_of_unity():
    m = M.turek_channel(n_t=16, n_r=8, n_x=40)
    c = np.array([0.7, -0.2])
    V = np.repeat(c[:, None], m.n_dofs, axis=1)
    o = Oracle(m, (2, 2), 2, 1, 1e-3)
    o.seed(V)
    Vp = o.project()
    assert np.allclose(Vp, V, atol=1e-14)


def test_count_cap_keeps_max_plus_one():
    # all particles squeezed into one cell part: max/part = 2 keeps 3
    m = _channel(4, 2)
    V = np.zeros((2, m.n_dofs))
    o = Oracle(m, (4, 4), 2, 1, 0.0)
    n = 10
    X = m.vertices[m.cells[5]]
    xi = np.tile([[0.1, 0.1]], (n, 1))
    x = np.array([forward_map(X, z) for z in xi])
    P = {"id": np.arange(1, n + 1, dtype=np.uint32), "cell": np.full(n, 5, np.int32), "x": x, "xi": xi,
         "v": np.zeros((n, 2))}
    for order in (ORDER_ID, ORDER_VECTOR):
        o = Oracle(m, (4, 4), 2, 1, 0.0, removal_order=order)
        o.set_particles(P, n)
        o.move(V)
        Q = o.particles()
        st = o.stats()
        assert st["removed"] == 7 and st["seeded"] == 15
        assert np.sum(Q["cell"] == 5) == 3 + 15
        assert set(np.unique(Q["cell"])) == {5}  # empty cells are never reseeded
        kept = sorted(Q["id"][Q["id"] <= n])
        if order == ORDER_ID:
            assert kept == [1, 2, 3]
        else:
            # swap-with-back: 1,2,3 counted, 4 replaced by 10 (removed), 9, 8, ...
            assert kept == [1, 2, 3]
        new = np.sort(Q["id"][Q["id"] > n])
        assert np.array_equal(new, np.arange(n + 1, n + 16))


def test_vector_and_id_order_agree_on_counts():
    m = _channel(32, 8)
    V = M.field_at_dofs(m, M.channel_profile())
    res = []
    for order in (ORDER_ID, ORDER_VECTOR):
        o = Oracle(m, (3, 3), 1, 4, 0.02, removal_order=order)
        o.seed(V)
        o.step(V, 0.9 * V)
        P = o.particles()
        res.append((np.bincount(P["cell"], minlength=m.n_cells), o.stats()))
    assert np.array_equal(res[0][0], res[1][0])
    for k in ("lost", "removed", "seeded", "n_particles"):
        assert res[0][1][k] == res[1][1][k]


def test_closed_divergence_free_flow_loses_nothing():
    m = M.perturbed_cube(6, amplitude=0.1, seed=0)
    V = M.field_at_dofs(m, M.taylor_green_3d())
    o = Oracle(m, (2, 2, 2), 2, 3, 0.05)
    o.seed(V)
    for _ in range(5):
        o.step(V, V)
    assert o.stats()["lost"] == 0


def test_vertex_maps_match_host_builder():
    for m in (_channel(8, 3), M.perturbed_cube(3), M.turek_channel(8, 4, 10)):
        o = Oracle(m, (2,) * m.dim, 2, 1, 0.1)
        off, cells, dirs = o.vertex_maps()
        off2, cells2, dirs2 = M.vertex_maps(m)
        assert np.array_equal(off, off2) and np.array_equal(cells, cells2)
        assert np.array_equal(dirs, dirs2)  # bit-exact


def test_threaded_oracle_matches_serial_state():
    m = M.perturbed_cube(5, amplitude=0.1, seed=3)
    V = M.field_at_dofs(m, M.taylor_green_3d())
    outs = []
    for nt in (1, 4):
        o = Oracle(m, (2, 2, 2), 1, 3, 0.1, n_threads=nt)
        o.seed(V)
        for _ in range(3):
            Vp = o.step(V, 0.5 * V)
        outs.append((o.particles(), Vp))
    a, b = outs
    for k in ("id", "cell", "x", "xi", "v"):
        assert np.array_equal(a[0][k], b[0][k])
    assert np.allclose(a[1], b[1], rtol=1e-13, atol=1e-13)


def test_unv_round_trip():
    m = M.turek_channel(8, 4, 10)
    buf = io.StringIO()
    M.write_unv(m, buf)
    buf.seek(0)
    r = M.read_unv(buf)
    assert r.n_cells == m.n_cells and r.n_verts == m.n_verts
    assert np.allclose(r.vertices, m.vertices, rtol=0, atol=1e-15)
    assert np.array_equal(r.cells, m.cells)


MESH3 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "Mesh3.tgz")


def test_reference_turek_mesh_reads():
    """The reference's Turek benchmark mesh (cases/TurekBenchmark/Mesh3.tgz,
    committed as a fixture)."""
    m = M.read_unv(MESH3)
    assert m.n_cells == 60450 and m.n_verts == 61075
    assert np.allclose(m.vertices.min(0), [0, 0]) and np.allclose(m.vertices.max(0), [2.2, 0.41])


@pytest.mark.parametrize("which", ["channel", "cylinder", "cube"])
def test_oracle_window_adjoint_central_differences(which):
    """The oracle's adjoint of the differentiated window against central
    differences of its own window forward (h = 1e-6), along random directions
    of the starting particle velocities, V and Vold.  The time steps are not
    dyadic: on these uniform grids a dyadic step can land a particle exactly
    on a cell face, where J has a kink (the projection weights are only
    piecewise smooth) and central differences average the two sides."""
    c = {"channel": lambda: cases.channel(16, 4, S=2, dt=0.047),
         "cylinder": lambda: cases.cylinder(n_t=12, n_r=6, n_x=20, dt=5e-3),
         "cube": lambda: cases.cube(n=4, q=(2, 2, 2), dt=5e-2)}[which]()
    o = cases.oracle_for(c)
    o.seed(c.V)
    o.step(c.V, c.Vold)
    K = 3
    P = o.particles()
    U = o.window_forward(K, c.V, c.Vold)
    rng = np.random.default_rng(1)
    finite = np.where(np.all(np.isfinite(U), 0))[0]
    probe = rng.choice(finite, 8, replace=False)
    T = U[:, probe] + 0.01
    J = lambda Ux: float(np.sum((Ux[:, probe] - T) ** 2))  # noqa: E731
    gU = np.zeros_like(U)
    gU[:, probe] = 2 * (U[:, probe] - T)
    U2, gv0, gV, gVo = o.window_adjoint(K, c.V, gU, Vold=c.Vold)
    assert np.array_equal(U2, U, equal_nan=True)
    h = 1e-6
    for name in ("v0", "V", "Vold"):
        d = rng.standard_normal(P["v"].shape if name == "v0" else c.V.shape)
        if name == "v0":
            Jp = J(o.window_forward(K, c.V, c.Vold, v0=P["v"] + h * d))
            Jm = J(o.window_forward(K, c.V, c.Vold, v0=P["v"] - h * d))
            ana = np.sum(gv0 * d)
        elif name == "V":
            Jp, Jm = J(o.window_forward(K, c.V + h * d, c.Vold)), J(o.window_forward(K, c.V - h * d, c.Vold))
            ana = np.sum(gV * d)
        else:
            Jp, Jm = J(o.window_forward(K, c.V, c.Vold + h * d)), J(o.window_forward(K, c.V, c.Vold - h * d))
            ana = np.sum(gVo * d)
        fd = (Jp - Jm) / (2 * h)
        assert abs(fd - ana) <= 1e-6 * abs(fd), (name, fd, ana)


def _unv_file(tmp_path, m, name):
    p = tmp_path / name
    with open(p, "w") as f:
        M.write_unv(m, f)
    return str(p)


@pytest.mark.parametrize("which", ["channel2d", "turek", "box3d", "cube3d"])
def test_native_unv_reader_matches_python(tmp_path, which):
    """pfem2gpu_read_unv (the library's C++ reader, host only) gives the same
    vertices and cells as mesh.read_unv."""
    m = {"channel2d": lambda: M.hyper_rectangle((0, 0), (4, 1), (16, 4)),
         "turek": lambda: M.turek_channel(8, 4, 10),
         "box3d": lambda: M.hyper_rectangle((0, 0, 0), (2, 1, 1), (4, 3, 2)),
         "cube3d": lambda: M.perturbed_cube(5)}[which]()
    p = _unv_file(tmp_path, m, which + ".unv")
    a = M.read_unv(p)
    b = M.read_unv_native(p)
    assert b.dim == a.dim == m.dim
    assert np.array_equal(a.vertices, b.vertices)
    assert np.array_equal(a.cells, b.cells)
    assert np.array_equal(b.cells, m.cells)


def test_native_unv_reader_flips_left_handed_cells(tmp_path):
    """Cells written with their first two directions swapped (negative
    Jacobian) come back right-handed, as in the Python reader."""
    m = M.hyper_rectangle((0, 0, 0), (1, 1, 1), (2, 2, 2))
    bad = m.cells.copy()
    bad[::2] = bad[::2][:, [0, 2, 1, 3, 4, 6, 5, 7]]
    mb = M.Mesh(3, m.vertices, bad, bad.copy(), m.n_verts, "flipped")
    p = _unv_file(tmp_path, mb, "flipped.unv")
    b = M.read_unv_native(p)
    assert np.array_equal(b.cells, M.read_unv(p).cells)
    assert np.array_equal(b.cells, m.cells)


def test_native_unv_reader_errors(tmp_path):
    from pfem2dealii_b200 import _lib
    import ctypes as C

    L = _lib.load()
    nv, nc = C.c_int64(), C.c_int64()
    assert L.pfem2gpu_read_unv(b"/nonexistent.unv", 0, None, C.byref(nv), C.byref(nc), None, None, 0, 0) != 0
    assert b"cannot open" in L.pfem2gpu_read_unv_error()
    p = _unv_file(tmp_path, M.hyper_rectangle((0, 0), (1, 1), (2, 2)), "q.unv")
    assert L.pfem2gpu_read_unv(p.encode(), 3, None, C.byref(nv), C.byref(nc), None, None, 0, 0) != 0
    assert b"2D" in L.pfem2gpu_read_unv_error()


MESH2 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "Mesh2.tgz")


def test_native_unv_reader_reference_mesh2():
    """The mesh the reference's own Turek case reads (cases/TurekBenchmark/
    Mesh2.tgz, its input_data.prm: `Mesh file name = Mesh2.unv`), committed
    as a fixture: both readers agree and give the 2.2 x 0.41 channel."""
    a = M.read_unv(MESH2)
    b = M.read_unv_native(MESH2)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.cells, b.cells)
    assert a.n_cells == 19700 and a.n_verts == 20060
    assert np.allclose(a.vertices.min(0), [0, 0]) and np.allclose(a.vertices.max(0), [2.2, 0.41])


def test_uniform_flow_on_the_reference_turek_case():
    """Mesh2 with the particle settings of the reference's Turek case
    (input_data.prm: 2 x 2 particles per cell, at most 5 per part, 3
    integration steps, time step 0.001) in a uniform field u = (1, -0.2):
    every particle carries u, so each projected DoF is u up to rounding
    (partition of unity), and every particle that stays in the mesh moves by
    exactly u dt in the FP64 position, whatever the cell's shape."""
    m = M.read_unv_native(MESH2)
    u = np.array([1.0, -0.2])
    V = np.repeat(u[:, None], m.n_dofs, axis=1)
    o = Oracle(m, (2, 2), 5, 3, 1e-3)
    o.seed(V)
    Vold = o.project()
    for _ in range(3):
        P0 = o.particles()
        Vold = o.step(V, Vold)
        P1 = o.particles()
        common, i0, i1 = np.intersect1d(P0["id"], P1["id"], return_indices=True)
        assert len(common) > 0.99 * len(P0["id"])
        assert np.allclose(P1["x"][i1] - P0["x"][i0], u * 1e-3, rtol=0, atol=1e-15)
        assert np.all((P1["xi"] >= 0) & (P1["xi"] <= 1))
        assert np.allclose(P1["v"], u, rtol=0, atol=1e-15)
        f = np.isfinite(Vold[0])
        assert f.mean() > 0.99
        assert np.allclose(Vold[:, f], u[:, None], rtol=0, atol=1e-14)


def test_native_unv_reader_reference_mesh():
    a = M.read_unv(MESH3)
    b = M.read_unv_native(MESH3)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.cells, b.cells)


def _rotation_error(integrator, S, T=0.4):
    """Largest position error after time T of particles in the solid-body
    rotation u = (-(y - 1/2), x - 1/2) on an 8x8 unit square, taken as one
    time step of S sub-steps.  The Q1 field reproduces the linear velocity
    exactly, so the error is the integrator's alone."""
    from oracle.oracle import Oracle

    m = M.hyper_rectangle((0.0, 0.0), (1.0, 1.0), (8, 8))
    xy = m.dof_coordinates()
    V = np.ascontiguousarray(np.stack([-(xy[:, 1] - 0.5), xy[:, 0] - 0.5]))
    o = Oracle(m, (4, 4), 100, S, T, integrator=integrator)
    o.seed(V)
    P0 = o.particles()
    x0 = {int(i): x for i, x in zip(P0["id"], P0["x"])}
    o.move(V)
    P = o.particles()
    c, s = np.cos(T), np.sin(T)
    err = 0.0
    for i, x in zip(P["id"], P["x"]):
        if int(i) not in x0:
            continue  # seeded by count correction
        r = x0[int(i)] - 0.5
        if np.hypot(*r) > 0.3:
            continue  # may leave the square
        ex = np.array([c * r[0] - s * r[1], s * r[0] + c * r[1]]) + 0.5
        err = max(err, float(np.max(np.abs(x - ex))))
    return err


def test_rk2_substeps_are_second_order():
    """The opt-in RK2 sub-step (midpoint rule in the particle's own cell; the
    reference has Euler only): halving the sub-step divides the error by 4,
    against 2 for Euler, the reference's integrator."""
    from oracle.oracle import EULER, RK2

    e = {k: [_rotation_error(k, S) for S in (8, 16, 32)] for k in (EULER, RK2)}
    for a, b in zip(e[EULER], e[EULER][1:]):
        assert 1.8 < a / b < 2.2, e[EULER]
    for a, b in zip(e[RK2], e[RK2][1:]):
        assert 3.6 < a / b < 4.4, e[RK2]
    assert e[RK2][-1] < 1e-2 * e[EULER][-1]


def test_window_refuses_rk2():
    from oracle.oracle import RK2, Oracle

    c = cases.channel(8, 4)
    o = Oracle(c.mesh, c.q, c.max_per_part, c.substeps, c.dt, integrator=RK2)
    o.seed(c.V)
    with pytest.raises(Exception):
        o.window_forward(2, c.V)
