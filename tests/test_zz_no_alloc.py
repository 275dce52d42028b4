"""pfem2gpu_project_noalloc: the projection that allocates no device memory.

Collected last on purpose (file name), so that it also runs after every other
GPU test has used the device in this process.  The FP64 handle's
pfem2gpu_project of the same particles is the comparison: equal bit for bit
(same sums in the same order), on two calls in a row.
"""
import ctypes as C

import numpy as np
import pytest

from pfem2dealii_b200 import _lib
from pfem2dealii_b200.handler import ParticleHandler, project_noalloc

from . import cases

pytestmark = pytest.mark.gpu


def _handle_after_steps(case, steps, precision="fp64"):
    g = ParticleHandler(case.mesh.dim, cases.params(case), precision)
    g.initialize_maps(case.mesh)
    g.seed_particles(case.V)
    for _ in range(steps):
        g.step(case.V, case.Vold)
    return g


def _device_particles(P, dim):
    import torch

    cell = torch.tensor(P["cell"], dtype=torch.int32, device="cuda")
    xi = torch.tensor(np.ascontiguousarray(P["xi"].T), device="cuda")
    v = torch.tensor(np.ascontiguousarray(P["v"].T), device="cuda")
    return cell, xi, v


def _same(a, b):
    return np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[np.isfinite(a)], b[np.isfinite(b)])


@pytest.mark.parametrize("which", ["channel", "duct", "cylinder"])
def test_noalloc_equals_handle_projection_twice(which):
    import torch

    c = {"channel": lambda: cases.channel(dt=0.01), "duct": lambda: cases.duct(16, 6, 6, dt=0.05),
         "cylinder": lambda: cases.cylinder(12, 6, 24, dt=0.01)}[which]()
    g = _handle_after_steps(c, 4)
    Vh = g.project_particle_fields()
    P = g.particles()
    assert np.all(np.diff(P["cell"]) >= 0)
    cell, xi, v = _device_particles(P, c.mesh.dim)
    cd = torch.tensor(c.mesh.cell_dofs, dtype=torch.int32, device="cuda")
    out = torch.empty((c.mesh.dim, c.mesh.n_dofs), dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(7.0)
        n_empty = project_noalloc(cd, cell, xi, v, out)
        torch.cuda.synchronize()
        Vn = out.cpu().numpy()
        assert _same(Vh, Vn)
        assert n_empty == g.stats()["nan_dofs"]


def test_noalloc_keep_policy_and_empty_input():
    import torch

    c = cases.channel(8, 4, dt=0.0)
    cd = torch.tensor(c.mesh.cell_dofs, dtype=torch.int32, device="cuda")
    e32 = torch.empty(0, dtype=torch.int32, device="cuda")
    e64 = torch.empty((c.mesh.dim, 0), dtype=torch.float64, device="cuda")
    out = torch.tensor(c.V, device="cuda")
    assert project_noalloc(cd, e32, e64, e64, out, empty_dof_policy=1) == c.mesh.n_dofs
    assert np.array_equal(out.cpu().numpy(), c.V)
    assert project_noalloc(cd, e32, e64, e64, out) == c.mesh.n_dofs
    assert np.isnan(out.cpu().numpy()).all()


def test_noalloc_rejects_bad_input_and_oversize():
    import torch

    L = _lib.load()
    c = cases.channel(8, 4, dt=0.0)
    g = _handle_after_steps(c, 0)
    P = g.particles()
    cell, xi, v = _device_particles(P, 2)
    cd = torch.tensor(c.mesh.cell_dofs, dtype=torch.int32, device="cuda")
    out = torch.empty((2, c.mesh.n_dofs), dtype=torch.float64, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    n = len(P["cell"])

    def call(n_cells=c.mesh.n_cells, n_dofs=c.mesh.n_dofs, cells=cell, dofs=cd):
        return L.pfem2gpu_project_noalloc(2, n_cells, n_dofs, p(dofs), n, p(cells), p(xi), p(v), 0, p(out), None,
                                          None)

    assert call() == _lib.OK
    # a mesh larger than the static scratch is refused before any launch
    assert call(n_cells=(1 << 31) // 4 - 1, n_dofs=1 << 26) == _lib.ERR_SCRATCH
    # particle cells out of order, or out of range, and DoFs out of range: ERR_ARG after the call
    rev = torch.flip(cell, [0]).contiguous()
    assert call(cells=rev) == _lib.ERR_ARG
    bad = cell.clone()
    bad[-1] = c.mesh.n_cells
    assert call(cells=bad) == _lib.ERR_ARG
    bad_dofs = cd.clone()
    bad_dofs[0, 0] = -1
    assert call(dofs=bad_dofs) == _lib.ERR_ARG
    # and a good call afterwards still gives the handle's result
    assert call() == _lib.OK
    torch.cuda.synchronize()
    assert _same(g.project_particle_fields(), out.cpu().numpy())
