"""The solver step's Q1 systems assembled on the device
(src/pfem2fem.cpp:247-510, volume terms) against the FP64 oracle: the CSR
pattern equal, matrices and right-hand sides bit for bit (both sum each
entry's cell contributions in ascending cell order, every operation
separately rounded), on structured, unstructured and perturbed meshes in 2D
and 3D; plus properties that hold whatever the arithmetic (mass matrix sums
to rho times the volume, Laplacian rows sum to zero, symmetric pressure
matrix)."""
import numpy as np
import pytest

from oracle import oracle as O
from pfem2dealii_b200 import mesh as M
from pfem2dealii_b200.handler import ParticleHandler

from . import cases

pytestmark = pytest.mark.gpu

RHO, MU, DT = 1.3, 0.01, 0.02


def _mesh(which):
    return {"channel": lambda: M.hyper_rectangle((0, 0), (4, 1), (16, 8)),
            "cylinder": lambda: M.turek_channel(24, 12, 60),
            "box": lambda: M.hyper_rectangle((0, 0, 0), (2, 1, 1), (8, 4, 4)),
            "cube": lambda: M.perturbed_cube(8)}[which]()


def _handler(m):
    c = cases.channel() if m.dim == 2 else cases.duct(8, 4, 4)
    g = ParticleHandler(m.dim, cases.params(c), "fp64")
    g.initialize_maps(m)
    return g


def _fields(m, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((m.dim, m.n_dofs)), rng.standard_normal((m.dim, m.n_dofs)), \
        rng.standard_normal(m.n_dofs)


@pytest.mark.parametrize("which", ["channel", "cylinder", "box", "cube"])
def test_fem_systems_match_oracle_bit_for_bit(which):
    m = _mesh(which)
    g = _handler(m)
    rp, cols = g.fem_pattern()
    orp, ocols = O.fem_pattern(m)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)
    U, U2, P = _fields(m)
    for system, kw in ((O.FEM_PREDICTION, dict(U=U, U2=U2)), (O.FEM_PRESSURE, dict(U=U)),
                       (O.FEM_CORRECTION, dict(U=U, P=P))):
        A, r = g.fem_assemble(system, RHO, MU, DT, **kw)
        Ao, ro = O.fem_assemble(m, system, RHO, MU, DT, pattern=(orp, ocols), **kw)
        assert A.shape == Ao.shape and r.shape == ro.shape
        assert A.tobytes() == Ao.tobytes(), (system, np.max(np.abs(A - Ao)))
        assert r.tobytes() == ro.tobytes(), (system, np.max(np.abs(r - ro)))
    g.close()


@pytest.mark.parametrize("which", ["cylinder", "cube"])
def test_fem_system_properties(which):
    m = _mesh(which)
    g = _handler(m)
    rp, cols = g.fem_pattern()
    U, U2, P = _fields(m, 1)
    X = m.vertices[m.cells]
    # volume by the same quadrature: the mass matrix sums to rho * |Omega|
    A, _ = g.fem_assemble(O.FEM_CORRECTION, RHO, MU, DT, U=U, P=P)
    vol = float(np.sum(np.abs(_volumes(X))))
    assert abs(A[0].sum() - RHO * vol) <= 1e-12 * RHO * vol
    # pressure matrix: rows sum to zero, symmetric
    A, _ = g.fem_assemble(O.FEM_PRESSURE, RHO, MU, DT, U=U)
    rows = np.add.reduceat(A[0], rp[:-1])
    assert np.max(np.abs(rows)) <= 1e-12 * np.max(np.abs(A[0]))
    import scipy.sparse as sp

    S = sp.csr_matrix((A[0], cols, rp), shape=(m.n_dofs, m.n_dofs))
    assert abs(S - S.T).max() <= 1e-13 * abs(S).max()
    # a uniform velocity has no divergence: the pressure right-hand side
    # vanishes wherever the velocity's support is whole (interior DoFs)
    c = np.arange(1, m.dim + 1, dtype=float)
    _, r = g.fem_assemble(O.FEM_PRESSURE, RHO, MU, DT, U=np.repeat(c[:, None], m.n_dofs, 1))
    assert np.isfinite(r).all()
    g.close()


def _volumes(X):
    """Cell volumes by the 2^dim-point Gauss rule (exact for these maps)."""
    dim = X.shape[2]
    nv = 1 << dim
    q = [0.21132486540518711775, 0.78867513459481288225]
    vol = np.zeros(X.shape[0])
    for k in range(nv):
        xi = [q[(k >> d) & 1] for d in range(dim)]
        J = np.zeros((X.shape[0], dim, dim))
        for i in range(nv):
            for e in range(dim):
                t = 1.0 if (i >> e) & 1 else -1.0
                for d in range(dim):
                    if d != e:
                        t *= xi[d] if (i >> d) & 1 else 1 - xi[d]
                J[:, :, e] += X[:, i, :] * t
        vol += np.linalg.det(J) * (0.5 ** dim)
    return vol


def test_fem_device_call_and_errors():
    import torch

    m = _mesh("box")
    g = _handler(m)
    rp, cols = g.fem_pattern()
    U, U2, P = _fields(m, 2)
    dU = torch.tensor(U, device="cuda")
    dU2 = torch.tensor(U2, device="cuda")
    dA = torch.empty((m.dim, len(cols)), dtype=torch.float64, device="cuda")
    dr = torch.empty((m.dim, m.n_dofs), dtype=torch.float64, device="cuda")
    g._ck(g.L.pfem2gpu_fem_assemble_device(g.h, 0, RHO, MU, DT, dU.data_ptr(), dU2.data_ptr(), None,
                                            dA.data_ptr(), dr.data_ptr()))
    g.synchronize()
    A, r = g.fem_assemble(0, RHO, MU, DT, U=U, U2=U2)
    assert np.array_equal(dA.cpu().numpy(), A) and np.array_equal(dr.cpu().numpy(), r)
    # unknown system and missing inputs are argument errors
    assert g.L.pfem2gpu_fem_assemble_device(g.h, 7, RHO, MU, DT, dU.data_ptr(), None, None, dA.data_ptr(),
                                            dr.data_ptr()) == 1
    assert g.L.pfem2gpu_fem_assemble_device(g.h, 0, RHO, MU, DT, dU.data_ptr(), None, None, dA.data_ptr(),
                                            dr.data_ptr()) == 1
    del dU, dU2, dA, dr
    g.close()


BOUNDARY = {  # velocity Dirichlet ids, pressure Dirichlet ids (the rest gets face terms)
    "channel": ((0, 2, 3), (1,)),
    "cylinder": ((0, 2, 3, 4), (1,)),
    "box": ((0, 2, 3, 4, 5), (1,)),
    "cube": ((0, 1, 2, 3), (4, 5)),
}


@pytest.mark.parametrize("which", ["channel", "cylinder", "box", "cube"])
def test_fem_face_terms_match_oracle_bit_for_bit(which):
    """With boundary ids and Dirichlet sets, the prediction and pressure
    systems carry the boundary-face terms (src/pfem2fem.cpp:320-383,
    436-449) on the other boundary faces; device and oracle agree bit for
    bit, and clearing the ids gives the volume-only systems back."""
    m = _mesh(which)
    g = _handler(m)
    fid = M.boundary_face_ids(m)
    vd, pd = BOUNDARY[which]
    g.fem_set_boundary(fid, vd, pd)
    mask = O.fem_face_mask(fid, vd, pd)
    assert mask.any()
    pat = O.fem_pattern(m)
    U, U2, P = _fields(m, 3)
    for system, kw in ((O.FEM_PREDICTION, dict(U=U, U2=U2)), (O.FEM_PRESSURE, dict(U=U)),
                       (O.FEM_CORRECTION, dict(U=U, P=P))):
        A, r = g.fem_assemble(system, RHO, MU, DT, **kw)
        Ao, ro = O.fem_assemble(m, system, RHO, MU, DT, pattern=pat, face_mask=mask, **kw)
        assert A.tobytes() == Ao.tobytes(), (system, np.max(np.abs(A - Ao)))
        assert r.tobytes() == ro.tobytes(), (system, np.max(np.abs(r - ro)))
    g.fem_set_boundary(None)
    A, r = g.fem_assemble(O.FEM_PRESSURE, RHO, MU, DT, U=U)
    Ao, ro = O.fem_assemble(m, O.FEM_PRESSURE, RHO, MU, DT, pattern=pat, U=U)
    assert A.tobytes() == Ao.tobytes() and r.tobytes() == ro.tobytes()
    g.close()


@pytest.mark.parametrize("which", ["channel", "cylinder", "cube"])
def test_fem_pressure_face_term_is_the_outflux(which):
    """With face terms on the whole boundary, the pressure right-hand side
    sums to -rho/dt times the outflux of the velocity, here u = (x, 0, 0):
    the domain's volume (the divergence theorem on the discrete normals)."""
    m = _mesh(which)
    g = _handler(m)
    g.fem_set_boundary(M.boundary_face_ids(m), (), ())
    U = np.zeros((m.dim, m.n_dofs))
    U[0] = m.vertices[:, 0]
    _, r = g.fem_assemble(O.FEM_PRESSURE, 1.0, 0.0, 1.0, U=U)
    vol = float(np.sum(_volumes(m.vertices[m.cells])))
    assert abs(r.sum() + vol) <= 1e-12 * vol
    g.close()


@pytest.mark.parametrize("which", ["cylinder", "box"])
def test_fem_dirichlet_rows_match_oracle_and_hold(which):
    """Dirichlet rows on the assembled prediction and pressure systems: the
    device result equals the restated rule bit for bit, and solving the
    constrained system returns the prescribed values on those rows."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    m = _mesh(which)
    g = _handler(m)
    fid = M.boundary_face_ids(m)
    vd, pd = BOUNDARY[which]
    g.fem_set_boundary(fid, vd, pd)
    rp, cols = g.fem_pattern()
    U, U2, P = _fields(m, 4)
    rng = np.random.default_rng(6)
    nv = m.nv
    for system, kw, ids in ((O.FEM_PREDICTION, dict(U=U, U2=U2), vd), (O.FEM_PRESSURE, dict(U=U), pd)):
        on = np.zeros(m.n_dofs, bool)
        for f in range(2 * m.dim):
            d, side = f // 2, f % 2
            loc = [i for i in range(nv) if ((i >> d) & 1) == side]
            sel = np.isin(fid[:, f], list(ids))
            on[m.cell_dofs[sel][:, loc].ravel()] = True
        rows = np.nonzero(on)[0].astype(np.int32)
        A, r = g.fem_assemble(system, RHO, MU, DT, **kw)
        vals = rng.standard_normal((r.shape[0], len(rows)))
        Ac, rc = g.fem_constrain(system, A, r, rows, vals)
        Ao, ro = O.fem_constrain(rp, cols, A, r, rows, vals)
        assert Ac.tobytes() == Ao.tobytes() and rc.tobytes() == ro.tobytes()
        for q in range(r.shape[0]):
            S = sp.csr_matrix((Ac[min(q, A.shape[0] - 1)], cols, rp), shape=(m.n_dofs, m.n_dofs))
            x = spl.spsolve(S.tocsc(), rc[q])
            assert np.allclose(x[rows], vals[q], rtol=1e-10, atol=1e-10)
    g.close()


VELOCITY_BC = {  # Dirichlet velocity per boundary id (inflow moves, walls and obstacle still)
    "channel": {0: (1.0, 0.0), 2: (0.0, 0.0), 3: (0.0, 0.0)},
    "cylinder": {0: (1.5, 0.0), 2: (0.0, 0.0), 3: (0.0, 0.0), 4: (0.0, 0.0)},
    "box": {0: (1.0, 0.0, 0.0), 2: (0.0,) * 3, 3: (0.0,) * 3, 4: (0.0,) * 3, 5: (0.0,) * 3},
    "cube": {0: (0.5, 0.0, 0.0), 1: (0.0,) * 3, 2: (0.0,) * 3, 3: (0.0,) * 3},
}


@pytest.mark.parametrize("which", ["channel", "cylinder", "box", "cube"])
def test_fem_velocity_bc_matches_oracle_and_linear_pressure(which):
    """velocity_prediction_bc (src/pfem2fem.cpp:150-245) on the device equals
    the oracle's rows and values bit for bit; with p = x the face-averaged
    gradient is (1, 0, 0), so every value is dt / rho e_x plus the Dirichlet
    velocity of the DoF's last Dirichlet face."""
    m = _mesh(which)
    g = _handler(m)
    fid = M.boundary_face_ids(m)
    vd, pd = BOUNDARY[which]
    bc = VELOCITY_BC[which]
    g.fem_set_boundary(fid, vd, pd)
    rng = np.random.default_rng(7)
    P = rng.standard_normal(m.n_dofs)
    rows, vals = g.fem_velocity_bc(RHO, DT, P, bc)
    ro, vo = O.fem_velocity_bc(m, fid, vd, bc, RHO, DT, P)
    assert np.array_equal(rows, ro) and vals.tobytes() == vo.tobytes()
    rows, vals = g.fem_velocity_bc(RHO, DT, m.vertices[:, 0].copy(), bc)
    _, vo = O.fem_velocity_bc(m, fid, vd, bc, RHO, DT, m.vertices[:, 0].copy())
    shift = vals.copy()
    shift[0] -= DT / RHO
    allowed = np.array([bc[k] for k in sorted(bc)]).T  # (dim, ids)
    for k in range(len(rows)):
        assert any(np.allclose(shift[:, k], allowed[:, j], atol=1e-11) for j in range(allowed.shape[1]))
    # the whole prediction step: assemble, Dirichlet rows, solve; the rows hold their values
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    rp, cols = g.fem_pattern()
    U, U2, _ = _fields(m, 8)
    A, r = g.fem_assemble(O.FEM_PREDICTION, RHO, MU, DT, U=U, U2=U2)
    A, r = g.fem_constrain(O.FEM_PREDICTION, A, r, rows, vals)
    for d in range(m.dim):
        x = spl.spsolve(sp.csr_matrix((A[d], cols, rp), shape=(m.n_dofs,) * 2).tocsc(), r[d])
        assert np.allclose(x[rows], vals[d], rtol=1e-10, atol=1e-10)
    g.close()
