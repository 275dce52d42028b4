// Drives pfem2gpu::FemSystems<dim> (include/pfem2gpu_handler.hpp) through
// pfem2Fem's call sequence: setup_system, then the three assemblies, with
// boundary ids.  Input (little-endian): int64 dim, n_cells, n_verts, n_dofs,
// n_vel, n_p; double rho, mu, dt; vertices (f64), cell_vertices, cell_dofs,
// face_ids (i32, n_cells x 2 dim), velocity ids (i32), pressure ids (i32),
// U, U2 (f64, dim x n_dofs), P (f64).  Output: int64 nnz, row_ptr, cols
// (i32), then for prediction, pressure, correction: A then rhs (f64); then
// the prediction's Dirichlet rows (int64 n, rows, values) and the constrained
// prediction A and rhs.
#include <cstdio>
#include <vector>

#include "pfem2gpu_handler.hpp"

template <typename T>
static bool rd(FILE* f, std::vector<T>& v, size_t n)
{
    v.resize(n);
    return fread(v.data(), sizeof(T), n, f) == n;
}

template <int dim>
static int run(const std::vector<int64_t>& hd, const std::vector<double>& coef, FILE* in, FILE* out)
{
    const int64_t nC = hd[1], nV = hd[2], nD = hd[3];
    pfem2gpu::Mesh m;
    m.n_cells = nC;
    m.n_verts = nV;
    m.n_dofs = nD;
    std::vector<int32_t> fid, vid, pid;
    std::vector<double> U, U2, P;
    if (!rd(in, m.vertices, nV * dim) || !rd(in, m.cell_vertices, nC << dim) || !rd(in, m.cell_dofs, nC << dim) ||
        !rd(in, fid, nC * 2 * dim) || !rd(in, vid, hd[4]) || !rd(in, pid, hd[5]) || !rd(in, U, dim * nD) ||
        !rd(in, U2, dim * nD) || !rd(in, P, nD))
        return 2;
    pfem2gpu_params prm{};
    for (int d = 0; d < 3; ++d) prm.particles_per_cell[d] = 2;
    prm.max_particles_per_cell_part = 2;
    prm.particle_integration_steps = 1;
    prm.time_step = coef[2];
    pfem2gpu::ParticleHandler<dim> particles(prm, PFEM2GPU_FP64);
    particles.set_mesh(m);
    pfem2gpu::FemSystems<dim> fem(particles, coef[0], coef[1]);
    std::vector<int32_t> row_ptr, cols;
    fem.setup_system(row_ptr, cols);
    fem.set_boundary(fid, vid, pid);
    const int64_t nnz = fem.nnz();
    fwrite(&nnz, 8, 1, out);
    fwrite(row_ptr.data(), 4, row_ptr.size(), out);
    fwrite(cols.data(), 4, cols.size(), out);
    std::vector<double> A(dim * nnz), rhs(dim * nD);
    fem.assemble_velocity_prediction(coef[2], U.data(), U2.data(), A.data(), rhs.data());
    fwrite(A.data(), 8, dim * nnz, out);
    fwrite(rhs.data(), 8, dim * nD, out);
    fem.assemble_pressure_equation(coef[2], U.data(), A.data(), rhs.data());
    fwrite(A.data(), 8, nnz, out);
    fwrite(rhs.data(), 8, nD, out);
    fem.assemble_velocity_correction(coef[2], U.data(), P.data(), A.data(), rhs.data());
    fwrite(A.data(), 8, nnz, out);
    fwrite(rhs.data(), 8, dim * nD, out);
    // the prediction's boundary values (every velocity-Dirichlet id moves with
    // velocity (1, 0, 0)) and the constrained prediction system
    std::vector<double> idv(vid.size() * dim, 0.0);
    for (size_t k = 0; k < vid.size(); ++k) idv[k * dim] = 1.0;
    std::vector<int32_t> rows;
    std::vector<double> vals;
    fem.velocity_prediction_bc(coef[2], P.data(), vid, idv, rows, vals);
    fem.assemble_velocity_prediction(coef[2], U.data(), U2.data(), A.data(), rhs.data());
    fem.apply_dirichlet(PFEM2GPU_FEM_PREDICTION, rows, vals, A.data(), rhs.data());
    const int64_t nr = (int64_t)rows.size();
    fwrite(&nr, 8, 1, out);
    fwrite(rows.data(), 4, rows.size(), out);
    fwrite(vals.data(), 8, vals.size(), out);
    fwrite(A.data(), 8, dim * nnz, out);
    fwrite(rhs.data(), 8, dim * nD, out);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    FILE* in = fopen(argv[1], "rb");
    FILE* out = fopen(argv[2], "wb");
    if (!in || !out) return 2;
    std::vector<int64_t> hd(6);
    std::vector<double> coef(3);
    if (fread(hd.data(), 8, 6, in) != 6 || fread(coef.data(), 8, 3, in) != 3) return 2;
    try {
        const int rc = hd[0] == 2 ? run<2>(hd, coef, in, out) : run<3>(hd, coef, in, out);
        fclose(out);
        return rc;
    } catch (const pfem2gpu::Error& e) {
        fprintf(stderr, "%s\n", e.what());
        return 10 + e.code;
    }
}
