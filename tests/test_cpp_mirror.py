"""The C++ mirror of pfem2ParticleHandler (include/pfem2gpu_handler.hpp),
driven through the reference's call sequence by tests/cpp/handler_driver.cpp:
it compiles and links against libpfem2gpu.so, reports a missing device as an
exception, and on a GPU gives the oracle's particles bit for bit (FP64 form).
"""
import os
import subprocess

import numpy as np
import pytest

from pfem2dealii_b200 import _lib

from . import cases
from .cases import by_id

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.dirname(_lib.LIB_PATH)


def _compile(tmp_path):
    exe = str(tmp_path / "handler_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "handler_driver.cpp"), "-L", LIBDIR, "-lpfem2gpu",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _write_input(path, case, steps, precision=0):
    m = case.mesh
    q = list(case.q) + [1] * (3 - len(case.q))
    hd = np.array([m.dim, precision, m.n_cells, m.n_verts, m.n_dofs, steps, *q, case.max_per_part, case.substeps],
                  np.int64)
    with open(path, "wb") as f:
        f.write(hd.tobytes())
        f.write(np.float64(case.dt).tobytes())
        for a, t in ((m.vertices, np.float64), (m.cells, np.int32), (m.cell_dofs, np.int32), (case.V, np.float64),
                     (case.Vold, np.float64)):
            f.write(np.ascontiguousarray(a, t).tobytes())


def _read_output(path, case, steps):
    dim, nD = case.mesh.dim, case.mesh.n_dofs
    raw = open(path, "rb").read()
    off = steps * dim * nD * 8
    V = np.frombuffer(raw[:off], np.float64).reshape(steps, dim, nD)
    n = int(np.frombuffer(raw[off:off + 8], np.int64)[0])
    off += 8
    P = {}
    for k, t, w in (("id", np.uint32, 1), ("cell", np.int32, 1), ("x", np.float64, dim), ("xi", np.float64, dim),
                    ("v", np.float64, dim)):
        a = np.frombuffer(raw[off:off + n * w * np.dtype(t).itemsize], t)
        off += a.nbytes
        P[k] = a.reshape(n, w) if w > 1 else a
    return V, P


def test_cpp_mirror_builds_and_reports_no_device(tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    exe = _compile(tmp_path)
    c = cases.channel(8, 4)
    _write_input(tmp_path / "in.bin", c, 1)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 10 + 6, (r.returncode, r.stderr)  # PFEM2GPU_ERR_NODEVICE, thrown as pfem2gpu::Error
    assert "no CUDA device" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["channel", "duct"])
def test_cpp_mirror_matches_oracle(tmp_path, which):
    c = cases.channel(32, 8, dt=0.02) if which == "channel" else cases.duct(16, 6, 6, dt=0.05)
    steps = 6
    exe = _compile(tmp_path)
    _write_input(tmp_path / "in.bin", c, steps)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    V, P = _read_output(tmp_path / "out.bin", c, steps)
    o = cases.oracle_for(c)
    o.seed(c.V)
    for s in range(steps):
        Vo = o.step(c.V, c.Vold)
        assert np.array_equal(np.isnan(Vo), np.isnan(V[s]))
        m = np.isfinite(Vo)
        assert np.max(np.abs(Vo[m] - V[s][m])) <= 1e-12 * np.max(np.abs(Vo[m]))
    a, b = by_id(o.particles()), by_id(P)
    for k in ("id", "cell", "x", "xi", "v"):
        assert np.array_equal(a[k], b[k].reshape(a[k].shape)), k


def test_cpp_read_unv_matches_python(tmp_path):
    """pfem2gpu::read_unv of the C++ mirror (host only, no device needed)
    gives mesh.read_unv's vertices and cells, each vertex its own DoF."""
    from pfem2dealii_b200 import mesh as M

    exe = str(tmp_path / "unv_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "unv_driver.cpp"), "-L", LIBDIR, "-lpfem2gpu",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for m in (M.turek_channel(8, 4, 10), M.perturbed_cube(4)):
        src = str(tmp_path / "m.unv")
        with open(src, "w") as f:
            M.write_unv(m, f)
        out = str(tmp_path / "m.bin")
        r = subprocess.run([exe, src, out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        raw = open(out, "rb").read()
        dim, nv, nc, nd = np.frombuffer(raw[:32], np.int64)
        o = 32
        verts = np.frombuffer(raw[o:o + nv * dim * 8], np.float64).reshape(nv, dim)
        o += nv * dim * 8
        cells = np.frombuffer(raw[o:o + nc * (1 << dim) * 4], np.int32).reshape(nc, 1 << dim)
        o += nc * (1 << dim) * 4
        dofs = np.frombuffer(raw[o:], np.int32).reshape(nc, 1 << dim)
        ref = M.read_unv(src)
        assert dim == ref.dim and nd == nv
        assert np.array_equal(verts, ref.vertices) and np.array_equal(cells, ref.cells)
        assert np.array_equal(dofs, cells)
    r = subprocess.run([exe, str(tmp_path / "missing.unv"), str(tmp_path / "x.bin")], capture_output=True, text=True)
    assert r.returncode == 3 and "cannot open" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cylinder", "cube"])
def test_cpp_fem_systems_match_oracle(tmp_path, which):
    """pfem2gpu::FemSystems, driven as pfem2Fem calls its assembly methods
    (setup_system, then prediction, pressure, correction with boundary
    ids), gives the oracle's pattern, matrices and right-hand sides bit for
    bit."""
    from oracle import oracle as O
    from pfem2dealii_b200 import mesh as M

    m = M.turek_channel(24, 12, 60) if which == "cylinder" else M.perturbed_cube(6)
    fid = M.boundary_face_ids(m)
    vd, pd = ((0, 2, 3, 4), (1,)) if which == "cylinder" else ((0, 1, 2, 3), (4, 5))
    rng = np.random.default_rng(5)
    U, U2, P = rng.standard_normal((m.dim, m.n_dofs)), rng.standard_normal((m.dim, m.n_dofs)), \
        rng.standard_normal(m.n_dofs)
    rho, mu, dt = 1.3, 0.01, 0.02
    exe = str(tmp_path / "fem_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "fem_driver.cpp"), "-L", LIBDIR, "-lpfem2gpu",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    src, dst = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(src, "wb") as f:
        f.write(np.array([m.dim, m.n_cells, m.n_verts, m.n_dofs, len(vd), len(pd)], np.int64).tobytes())
        f.write(np.array([rho, mu, dt], np.float64).tobytes())
        for a, t in ((m.vertices, np.float64), (m.cells, np.int32), (m.cell_dofs, np.int32), (fid, np.int32),
                     (np.array(vd), np.int32), (np.array(pd), np.int32), (U, np.float64), (U2, np.float64),
                     (P, np.float64)):
            f.write(np.ascontiguousarray(a, t).tobytes())
    r = subprocess.run([exe, src, dst], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = open(dst, "rb").read()
    nnz = int(np.frombuffer(raw[:8], np.int64)[0])
    o = 8
    rp = np.frombuffer(raw[o:o + 4 * (m.n_dofs + 1)], np.int32)
    o += 4 * (m.n_dofs + 1)
    cols = np.frombuffer(raw[o:o + 4 * nnz], np.int32)
    o += 4 * nnz
    orp, ocols = O.fem_pattern(m)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
    mask = O.fem_face_mask(fid, vd, pd)
    for system, nm, ns, kw in ((O.FEM_PREDICTION, m.dim, m.dim, dict(U=U, U2=U2)), (O.FEM_PRESSURE, 1, 1, dict(U=U)),
                               (O.FEM_CORRECTION, 1, m.dim, dict(U=U, P=P))):
        A = np.frombuffer(raw[o:o + 8 * nm * nnz], np.float64).reshape(nm, nnz)
        o += 8 * nm * nnz
        rhs = np.frombuffer(raw[o:o + 8 * ns * m.n_dofs], np.float64).reshape(ns, m.n_dofs)
        o += 8 * ns * m.n_dofs
        Ao, ro = O.fem_assemble(m, system, rho, mu, dt, pattern=(orp, ocols), face_mask=mask, **kw)
        assert A.tobytes() == Ao.tobytes() and rhs.tobytes() == ro.tobytes(), system
        if system == O.FEM_PREDICTION:
            Apred, rpred = Ao, ro
    nr = int(np.frombuffer(raw[o:o + 8], np.int64)[0])
    o += 8
    rows = np.frombuffer(raw[o:o + 4 * nr], np.int32)
    o += 4 * nr
    vals = np.frombuffer(raw[o:o + 8 * m.dim * nr], np.float64).reshape(m.dim, nr)
    o += 8 * m.dim * nr
    bc = {i: (1.0,) + (0.0,) * (m.dim - 1) for i in vd}
    ro_, vo_ = O.fem_velocity_bc(m, fid, vd, bc, rho, dt, P)
    assert np.array_equal(rows, ro_) and vals.tobytes() == vo_.tobytes()
    A = np.frombuffer(raw[o:o + 8 * m.dim * nnz], np.float64).reshape(m.dim, nnz)
    o += 8 * m.dim * nnz
    rhs = np.frombuffer(raw[o:o + 8 * m.dim * m.n_dofs], np.float64).reshape(m.dim, m.n_dofs)
    Ac, rc = O.fem_constrain(orp, ocols, Apred, rpred, rows, vals)
    assert A.tobytes() == Ac.tobytes() and rhs.tobytes() == rc.tobytes()


def _compile_shard(tmp_path):
    exe = str(tmp_path / "shard_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "shard_driver.cpp"), "-L", LIBDIR, "-lpfem2gpu",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_shard_driver_builds(tmp_path):
    """The partitioned move of the C++ mirror (set_partition, the three
    exchange phases, halo partials) compiles against the header and the
    library (no device needed)."""
    _compile_shard(tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("which,parts,precision", [("channel", 3, 0), ("duct", 2, 0), ("duct", 2, 1)])
def test_cpp_partitions_equal_one_handle(tmp_path, which, parts, precision):
    """P partitioned handles driven from C++ as P MPI ranks would drive them
    (exchange in memory), next to one unpartitioned handle: particles and
    assembled projections equal bit for bit at every step, FP64 and FP32."""
    from pfem2dealii_b200 import mesh as M

    c = cases.channel(32, 12, dt=0.03) if which == "channel" else cases.duct(24, 6, 8, dt=0.01)

    def swirl(x):
        u = np.zeros_like(x)
        u[:, 0] = 0.5 + 0.3 * np.cos(np.pi * x[:, 1])
        u[:, -1] = 0.6 * np.sin(np.pi * x[:, 0] / 2.0)
        return u

    c.V = M.field_at_dofs(c.mesh, swirl)
    exe = _compile_shard(tmp_path)
    _write_input(tmp_path / "in.bin", c, 8, precision)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(parts)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert int(r.stdout.strip()) > 100  # particles crossed between partitions
