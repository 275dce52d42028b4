// Drives P cell-partitioned pfem2gpu::ParticleHandler<dim> handles in one
// process the way P MPI ranks would (each phase on every partition before the
// next, the exchange done in memory in place of MPI_Alltoallv / MPI_Exscan),
// next to one unpartitioned handle, through the solver's data flow (seed,
// then per step correct from the last projection, move, project), and checks
// that the partitions' particles (in cell order) and their assembled
// projection equal the single handle's bit for bit.
//
// Input: the format of handler_driver.cpp (its Vold is not used).  argv[3] =
// number of partitions.  Prints the particles sent between partitions; exit
// status 0 = identical, 1 = a difference (printed), 10 + code on a pfem2gpu
// error.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pfem2gpu_handler.hpp"

template <typename T>
static bool rd(FILE* f, std::vector<T>& v, size_t n)
{
    v.resize(n);
    return fread(v.data(), sizeof(T), n, f) == n;
}

template <int dim>
using Handler = pfem2gpu::ParticleHandler<dim>;

template <int dim>
static void append(typename Handler<dim>::Exchange& to, const typename Handler<dim>::Exchange& from, size_t i)
{
    to.id.push_back(from.id[i]);
    to.cell.push_back(from.cell[i]);
    for (int d = 0; d < dim; ++d) {
        to.x.push_back(from.x[i * dim + d]);
        to.xi.push_back(from.xi[i * dim + d]);
        to.v.push_back(from.v[i * dim + d]);
    }
}

// Owner of a cell among contiguous ranges bounds[r] .. bounds[r + 1].
static int owner(const std::vector<int64_t>& bounds, int64_t c)
{
    return (int)(std::upper_bound(bounds.begin(), bounds.end(), c) - bounds.begin()) - 1;
}

static bool same(const double* a, const double* b, size_t n)
{
    return std::memcmp(a, b, n * sizeof(double)) == 0;
}

template <int dim>
static int run(const std::vector<int64_t>& hd, double dt, FILE* in, int P)
{
    constexpr int NV = 1 << dim, PW = 4 << dim;
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
        !rd(in, V, dim * nD) || !rd(in, Vold, dim * nD))
        return 2;
    const int prec = (int)hd[1];
    std::vector<int64_t> bounds(P + 1);
    for (int r = 0; r <= P; ++r) bounds[r] = r * nC / P;
    // halos (cells outside a range sharing a DoF with it) and DoF owners (lowest rank)
    std::vector<std::vector<int32_t>> halo(P);
    std::vector<int> dof_owner(nD, P);
    for (int64_t c = 0; c < nC; ++c)
        for (int k = 0; k < NV; ++k) {
            int& o = dof_owner[m.cell_dofs[c * NV + k]];
            o = std::min(o, owner(bounds, c));
        }
    for (int r = 0; r < P; ++r) {
        std::vector<char> mark(nD, 0);
        for (int64_t c = bounds[r]; c < bounds[r + 1]; ++c)
            for (int k = 0; k < NV; ++k) mark[m.cell_dofs[c * NV + k]] = 1;
        for (int64_t c = 0; c < nC; ++c) {
            if (c >= bounds[r] && c < bounds[r + 1]) continue;
            bool t = false;
            for (int k = 0; k < NV; ++k) t = t || mark[m.cell_dofs[c * NV + k]];
            if (t) halo[r].push_back((int32_t)c);
        }
    }
    Handler<dim> one(prm, prec);
    one.set_mesh(m);
    std::vector<Handler<dim>*> part;
    for (int r = 0; r < P; ++r) {
        part.push_back(new Handler<dim>(prm, prec));
        part[r]->set_mesh(m);
        part[r]->set_partition(bounds[r], bounds[r + 1]);
    }
    std::vector<double> U1(dim * nD), U(dim * nD);
    std::vector<std::vector<double>> Ur(P, std::vector<double>(dim * nD));
    one.seed_particles(V.data());
    for (int r = 0; r < P; ++r) part[r]->seed_particles(V.data());
    uint32_t next_id = part[0]->stats().next_id;
    int64_t sent = 0;
    int rc = 0;
    for (int64_t s = 0; s <= steps && rc == 0; ++s) {
        if (s > 0) {
            one.correct_particle_velocity_from_projection(V.data());
            one.move_particles(nullptr);
            // phase 1 on every partition, then the exchange
            std::vector<typename Handler<dim>::Exchange> inbox(P);
            for (int r = 0; r < P; ++r) {
                part[r]->correct_particle_velocity_from_projection(V.data());
                const auto out = part[r]->move_exchange_begin(nullptr);
                sent += (int64_t)out.size();
                for (size_t i = 0; i < out.size(); ++i) append<dim>(inbox[owner(bounds, out.cell[i])], out, i);
            }
            std::vector<int64_t> seeds(P);
            for (int r = 0; r < P; ++r) seeds[r] = part[r]->move_inbox(inbox[r]);
            int64_t below = 0, all = 0;
            for (int r = 0; r < P; ++r) all += seeds[r];
            for (int r = 0; r < P; ++r) {
                part[r]->move_exchange_end((uint32_t)(next_id + below), (uint32_t)(next_id + all));
                below += seeds[r];
            }
            next_id += (uint32_t)all;
        }
        // halo partial sums from their owners, then every partition's projection
        std::vector<std::vector<double>> hv(P);
        for (int r = 0; r < P; ++r) {
            hv[r].resize(halo[r].size() * PW);
            for (size_t j = 0; j < halo[r].size(); ++j) {
                const int o = owner(bounds, halo[r][j]);
                const auto p = part[o]->get_partials({halo[r][j]});
                std::copy(p.begin(), p.end(), hv[r].begin() + j * PW);
            }
        }
        for (int r = 0; r < P; ++r) {
            part[r]->set_partials(halo[r], hv[r]);
            part[r]->project_particle_fields(Ur[r].data());
        }
        one.project_particle_fields(U1.data());
        for (int d = 0; d < dim; ++d)
            for (int64_t k = 0; k < nD; ++k) U[d * nD + k] = Ur[dof_owner[k]][d * nD + k];
        if (!same(U.data(), U1.data(), U.size())) {
            fprintf(stderr, "projection differs at step %lld\n", (long long)s);
            rc = 1;
        }
        std::vector<pfem2gpu::Particle<dim>> all;
        for (int r = 0; r < P; ++r) {
            const auto pr = part[r]->particles();
            all.insert(all.end(), pr.begin(), pr.end());
        }
        const auto p1 = one.particles();
        bool ok = all.size() == p1.size();
        for (size_t i = 0; ok && i < all.size(); ++i) {
            ok = all[i].id == p1[i].id && all[i].cell == p1[i].cell &&
                 same(all[i].location.data(), p1[i].location.data(), dim) &&
                 same(all[i].reference_location.data(), p1[i].reference_location.data(), dim) &&
                 same(all[i].velocity.data(), p1[i].velocity.data(), dim);
        }
        if (!ok) {
            fprintf(stderr, "particles differ at step %lld (%zu vs %zu)\n", (long long)s, all.size(), p1.size());
            rc = 1;
        }
    }
    if (rc == 0 && part[0]->stats().next_id != one.stats().next_id) {
        fprintf(stderr, "next ids differ\n");
        rc = 1;
    }
    printf("%lld\n", (long long)sent);
    for (auto* h : part) delete h;
    return rc;
}

int main(int argc, char** argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s input partitions\n", argv[0]);
        return 2;
    }
    FILE* in = fopen(argv[1], "rb");
    if (!in) return 2;
    const int P = atoi(argv[2]);
    std::vector<int64_t> hd;
    double dt = 0;
    if (P < 1 || !rd(in, hd, 11) || fread(&dt, 8, 1, in) != 1) return 2;
    int rc = 2;
    try {
        rc = hd[0] == 2 ? run<2>(hd, dt, in, P) : run<3>(hd, dt, in, P);
    } catch (const pfem2gpu::Error& e) {
        fprintf(stderr, "%s\n", e.what());
        rc = 10 + e.code;
    }
    fclose(in);
    return rc;
}
