// Drives pfem2gpu::ParticleHandler<dim> through the reference's call sequence
// (src/pfem2solver.cpp:155-164: seed, initialize_maps, then per step
// correct, move, project) on a case read from a binary file, and writes the
// projected velocity of every step and the final particles.
//
// Input (little-endian): int64 dim, precision, n_cells, n_verts, n_dofs,
// steps, q0, q1, q2, max_per_part, substeps; double time_step; then
// vertices (f64), cell_vertices (i32), cell_dofs (i32), V, Vold (f64,
// component-major).  Output: steps x dim x n_dofs f64, then int64 n, and
// id (u32), cell (i32), x, xi, v (f64, n x dim).  Exit status 10 + code on a
// pfem2gpu error.
#include <cstdio>
#include <vector>

#include "pfem2gpu_handler.hpp"

template <typename T>
static bool rd(FILE* f, std::vector<T>& v, size_t n)
{
    v.resize(n);
    return fread(v.data(), sizeof(T), n, f) == n;
}

template <typename T>
static void wr(FILE* f, const T* p, size_t n)
{
    fwrite(p, sizeof(T), n, f);
}

template <int dim>
static int run(const std::vector<int64_t>& hd, double dt, FILE* in, FILE* out)
{
    const int64_t nC = hd[2], nV = hd[3], nD = hd[4], steps = hd[5];
    pfem2gpu_params prm{};
    for (int d = 0; d < 3; ++d) prm.particles_per_cell[d] = (int32_t)hd[6 + d];
    prm.max_particles_per_cell_part = (int32_t)hd[9];
    prm.particle_integration_steps = (int32_t)hd[10];
    prm.time_step = dt;
    pfem2gpu::Mesh m;
    m.n_cells = nC;
    m.n_verts = nV;
    m.n_dofs = nD;
    std::vector<double> V, Vold;
    if (!rd(in, m.vertices, nV * dim) || !rd(in, m.cell_vertices, nC << dim) || !rd(in, m.cell_dofs, nC << dim) ||
        !rd(in, V, dim * nD) || !rd(in, Vold, dim * nD)) {
        fprintf(stderr, "short input\n");
        return 2;
    }
    pfem2gpu::ParticleHandler<dim> handler(prm, (int)hd[1]);
    std::vector<double> Vout(dim * nD);
    handler.set_mesh(m);
    handler.set_solution_vectors(V.data(), Vold.data(), Vout.data());
    handler.seed_particles();
    handler.initialize_maps();
    for (int64_t s = 0; s < steps; ++s) {
        handler.correct_particle_velocity();
        handler.move_particles();
        handler.project_particle_fields();
        wr(out, Vout.data(), Vout.size());
    }
    const auto P = handler.particles();
    const int64_t n = (int64_t)P.size();
    wr(out, &n, 1);
    for (const auto& p : P) wr(out, &p.id, 1);
    for (const auto& p : P) wr(out, &p.cell, 1);
    for (const auto& p : P) wr(out, p.location.data(), dim);
    for (const auto& p : P) wr(out, p.reference_location.data(), dim);
    for (const auto& p : P) wr(out, p.velocity.data(), dim);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s input output\n", argv[0]);
        return 2;
    }
    FILE* in = fopen(argv[1], "rb");
    FILE* out = fopen(argv[2], "wb");
    if (!in || !out) return 2;
    std::vector<int64_t> hd;
    double dt = 0;
    if (!rd(in, hd, 11) || fread(&dt, 8, 1, in) != 1) return 2;
    int rc = 2;
    try {
        rc = hd[0] == 2 ? run<2>(hd, dt, in, out) : run<3>(hd, dt, in, out);
    } catch (const pfem2gpu::Error& e) {
        fprintf(stderr, "%s\n", e.what());
        rc = 10 + e.code;
    }
    fclose(in);
    fclose(out);
    return rc;
}
