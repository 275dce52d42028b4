// pfem2gpu_handler.hpp -- C++ mirror of pfem2ParticleHandler<dim> over the C ABI.
//
// Same public method names and call sequence as the reference class
// (src/pfem2particlehandler.h:17-71): the solver-side inputs that the
// reference fetches through its pfem2Solver pointer (mesh, parameters, the
// FEM velocity vectors getSolutionV/getOldSolutionV/setSolutionV,
// src/pfem2fem.cpp:622-644) are bound once instead, so that
//
//     handler.seed_particles();
//     handler.initialize_maps();
//     for (...) {
//         handler.correct_particle_velocity();
//         handler.move_particles();
//         handler.project_particle_fields();
//         ...
//     }
//
// reads as src/pfem2solver.cpp:155-164 does.  Errors throw pfem2gpu::Error
// (the reference throws deal.II exceptions); no CUDA type appears here.
// Header-only; link with libpfem2gpu.so.
#ifndef PFEM2GPU_HANDLER_HPP
#define PFEM2GPU_HANDLER_HPP

#include <array>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "pfem2gpu.h"

namespace pfem2gpu {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), code(code) {}
    int code;
};

inline void check(int rc, pfem2gpu_handle* h = nullptr)
{
    if (rc == PFEM2GPU_OK) return;
    std::string msg = std::string("pfem2gpu: ") + pfem2gpu_error_string(rc);
    if (h) {
        char buf[512] = {0};
        if (pfem2gpu_last_error(h, buf, sizeof buf) == PFEM2GPU_OK && buf[0]) msg += std::string(": ") + buf;
    }
    throw Error(rc, msg);
}

// Q1 mesh in deal.II numbering: vertices (n_verts x dim), and per cell the
// 2^dim vertex indices (cell->vertex_index(i)) and vertex DoFs
// (cell->vertex_dof_index(i, 0)) in lexicographic vertex order.
struct Mesh {
    int64_t n_cells = 0, n_verts = 0, n_dofs = 0;
    std::vector<double> vertices;
    std::vector<int32_t> cell_vertices, cell_dofs;
};

// GridIn::read_unv (src/pfem2solver.cpp:116-119) through pfem2gpu_read_unv:
// the mesh of a UNV file, each vertex its own DoF (vertex_dof_index = vertex
// index, deal.II's Q1 numbering before any renumbering).
inline Mesh read_unv(const std::string& path, int dim)
{
    Mesh m;
    int32_t d = 0;
    if (pfem2gpu_read_unv(path.c_str(), dim, &d, &m.n_verts, &m.n_cells, nullptr, nullptr, 0, 0) != PFEM2GPU_OK)
        throw Error(PFEM2GPU_ERR_ARG, std::string("pfem2gpu: ") + pfem2gpu_read_unv_error());
    m.vertices.resize((size_t)m.n_verts * d);
    m.cell_vertices.resize((size_t)m.n_cells << d);
    check(pfem2gpu_read_unv(path.c_str(), d, nullptr, &m.n_verts, &m.n_cells, m.vertices.data(),
                            m.cell_vertices.data(), m.n_verts, m.n_cells));
    m.cell_dofs = m.cell_vertices;
    m.n_dofs = m.n_verts;
    return m;
}

// The particle record of the reference (src/pfem2particle.h:63-72), without
// the per-particle DoF copy (the cell's DoFs are a per-cell table here).
template <int dim>
struct Particle {
    uint32_t id = 0;
    int32_t cell = 0;
    std::array<double, dim> location{}, reference_location{}, velocity{};
};

template <int dim>
class ParticleHandler {
public:
    static_assert(dim == 2 || dim == 3, "dim must be 2 or 3");

    // pfem2ParticleHandler(fe) + setPfem2Solver (src/pfem2particlehandler.cpp:10-15,30-40):
    // the particle keys of the .prm file and the form (PFEM2GPU_FP64 / PFEM2GPU_FP32).
    explicit ParticleHandler(const pfem2gpu_params& params, int precision = PFEM2GPU_FP64)
    {
        check(pfem2gpu_create(dim, precision, &params, &h_));
    }
    ~ParticleHandler()
    {
        if (h_) pfem2gpu_destroy(h_);
    }
    ParticleHandler(const ParticleHandler&) = delete;
    ParticleHandler& operator=(const ParticleHandler&) = delete;

    // The mesh the reference borrows from its solver.
    void set_mesh(const Mesh& m)
    {
        mesh_ = m;
        maps_ = false;
    }
    // The FEM vectors, component-major V[d * n_dofs + dof] (the reference's
    // std::array<TrilinosWrappers::MPI::Vector, dim> copied component by
    // component); out receives the projection.  They must outlive the calls.
    void set_solution_vectors(const double* V, const double* Vold, double* V_out)
    {
        V_ = V;
        Vold_ = Vold;
        Vout_ = V_out;
    }

    // initialize_maps (src/pfem2particlehandler.cpp:320-324): uploads the mesh;
    // the library builds vertex_to_cells and the centre directions.
    void initialize_maps()
    {
        if (maps_) return;
        check(pfem2gpu_set_mesh(h_, mesh_.n_cells, mesh_.n_verts, mesh_.n_dofs, mesh_.vertices.data(),
                                mesh_.cell_vertices.data(), mesh_.cell_dofs.data(), nullptr, nullptr, nullptr),
              h_);
        maps_ = true;
    }

    // seed_particles (:43-109).  The reference seeds before initialize_maps;
    // the mesh is uploaded here when that has not happened yet.
    void seed_particles()
    {
        initialize_maps();
        check(pfem2gpu_seed(h_, need(V_)), h_);
    }
    // correct_particle_velocity (:112-139).
    void correct_particle_velocity() { check(pfem2gpu_correct(h_, need(V_), need(Vold_)), h_); }
    // move_particles (:142-171), with the velocity of the last seed/correct.
    void move_particles() { check(pfem2gpu_move(h_, nullptr), h_); }
    // project_particle_fields (:174-215) into the bound output vector.
    void project_particle_fields() { check(pfem2gpu_project(h_, need(Vout_)), h_); }

    // Explicit-vector forms of the same calls.
    void seed_particles(const double* V)
    {
        initialize_maps();
        check(pfem2gpu_seed(h_, V), h_);
    }
    void correct_particle_velocity(const double* V, const double* Vold) { check(pfem2gpu_correct(h_, V, Vold), h_); }
    void move_particles(const double* V) { check(pfem2gpu_move(h_, V), h_); }
    void project_particle_fields(double* V_out) { check(pfem2gpu_project(h_, V_out), h_); }
    // correct_particle_velocity with Vold = the last projection, kept on the
    // device (fem_step copies the projection into the old solution,
    // src/pfem2fem.cpp:523-524): only V crosses the boundary.
    void correct_particle_velocity_from_projection(const double* V)
    {
        check(pfem2gpu_correct_from_projection(h_, V), h_);
    }

    // Cell-range partitions: this handle owns the particles of cells
    // [cell_begin, cell_end) of the mesh (the reference's distribution of the
    // cells over MPI ranks); a move runs in three phases around the caller's
    // exchange, the reference's send_recv_particles
    // (src/pfem2particlehandler.cpp:480-502,507-618), and the projection
    // needs the partial sums of the cells that share a DoF with this handle's
    // cells (:202-205).  See include/pfem2gpu.h for the ids to pass.
    struct Exchange {
        std::vector<uint32_t> id;
        std::vector<int32_t> cell;
        std::vector<double> x, xi, v;  // n x dim, row-major
        size_t size() const { return id.size(); }
        void resize(size_t n)
        {
            id.resize(n);
            cell.resize(n);
            x.resize(n * dim);
            xi.resize(n * dim);
            v.resize(n * dim);
        }
    };
    void set_partition(int64_t cell_begin, int64_t cell_end)
    {
        initialize_maps();
        check(pfem2gpu_set_partition(h_, cell_begin, cell_end), h_);
    }
    // Phases 1 and 2a: correction, sub-steps and relocation; returns the
    // particles that ended in other partitions' cells (they leave this
    // handle).  V null: the staged velocity.
    Exchange move_exchange_begin(const double* V)
    {
        int64_t n = 0, got = 0;
        check(pfem2gpu_move_exchange_begin(h_, V, &n), h_);
        Exchange out;
        out.resize((size_t)n);
        check(pfem2gpu_move_outbox(h_, out.id.data(), out.cell.data(), out.x.data(), out.xi.data(), out.v.data(), n,
                                   &got),
              h_);
        return out;
    }
    // Phase 2b: the particles other partitions sent to this handle's cells;
    // returns the number of particles count correction will add here.
    int64_t move_inbox(const Exchange& in)
    {
        int64_t seeds = 0;
        check(pfem2gpu_move_inbox(h_, (int64_t)in.size(), in.id.data(), in.cell.data(), in.x.data(), in.xi.data(),
                                  in.v.data(), &seeds),
              h_);
        return seeds;
    }
    // Phase 3: count correction and the new layout; new particles get ids
    // first_id + 1, ..., the handle's next id becomes next_id.
    void move_exchange_end(uint32_t first_id, uint32_t next_id)
    {
        check(pfem2gpu_move_exchange_end(h_, first_id, next_id), h_);
    }
    // Projection partial sums of cells, (4 << dim) doubles per cell.
    std::vector<double> get_partials(const std::vector<int32_t>& cells)
    {
        std::vector<double> out(cells.size() * (4u << dim));
        check(pfem2gpu_get_partials(h_, (int64_t)cells.size(), cells.data(), out.data()), h_);
        return out;
    }
    void set_partials(const std::vector<int32_t>& cells, const std::vector<double>& values)
    {
        if (values.size() != cells.size() * (4u << dim))
            throw Error(PFEM2GPU_ERR_ARG, "pfem2gpu: set_partials needs (4 << dim) values per cell");
        check(pfem2gpu_set_partials(h_, (int64_t)cells.size(), cells.data(), values.data()), h_);
    }

    // output_particle_solution (:218-317) for one rank: particles-NN.000.vtu + particles-NN.pvtu.
    void output_particle_solution(int timestep_number, const std::string& directory = ".")
    {
        char base[64];
        std::snprintf(base, sizeof base, "particles-%02d", timestep_number);
        const std::string dir = directory.empty() ? std::string(".") : directory;
        check(pfem2gpu_write_vtu(h_, (dir + "/" + base + ".000.vtu").c_str()), h_);
        std::ofstream f(dir + "/" + base + ".pvtu");
        f << "<?xml version=\"1.0\" ?> \n<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" "
             "byte_order=\"LittleEndian\">\n  <PUnstructuredGrid GhostLevel=\"0\">\n"
             "    <PPointData Scalars=\"scalars\">\n"
             "      <PDataArray type=\"Float32\" Name=\"velocity\" NumberOfComponents=\"3\" format=\"ascii\"/>\n"
             "      <PDataArray type=\"Float32\" Name=\"subdomain\" format=\"ascii\"/>\n"
             "    </PPointData>\n    <PPoints>\n"
             "      <PDataArray type=\"Float32\" NumberOfComponents=\"3\"/>\n    </PPoints>\n"
          << "    <Piece Source=\"" << base << ".000.vtu\"/>  </PUnstructuredGrid>\n</VTKFile>\n";
        if (!f) throw Error(PFEM2GPU_ERR_ARG, "pfem2gpu: cannot write " + dir + "/" + base + ".pvtu");
    }

    // begin()/end(): a host copy of the particles, in the device order
    // (cells ascending).
    std::vector<Particle<dim>> particles()
    {
        int64_t n = 0;  // count query: ERR_ARG (arrays too small) still sets n
        const int rc = pfem2gpu_get_particles(h_, nullptr, nullptr, nullptr, nullptr, nullptr, 0, &n);
        if (rc != PFEM2GPU_ERR_ARG) check(rc, h_);
        std::vector<uint32_t> id(n);
        std::vector<int32_t> cell(n);
        std::vector<double> x(n * dim), xi(n * dim), v(n * dim);
        check(pfem2gpu_get_particles(h_, id.data(), cell.data(), x.data(), xi.data(), v.data(), n, &n), h_);
        std::vector<Particle<dim>> out(n);
        for (int64_t p = 0; p < n; ++p) {
            out[p].id = id[p];
            out[p].cell = cell[p];
            for (int d = 0; d < dim; ++d) {
                out[p].location[d] = x[p * dim + d];
                out[p].reference_location[d] = xi[p * dim + d];
                out[p].velocity[d] = v[p * dim + d];
            }
        }
        return out;
    }

    // clear_particles / insert_particle (:327-344): collected on the host and
    // uploaded by the next call of commit_particles().
    void clear_particles() { pending_.clear(); }
    void insert_particle(const Particle<dim>& p) { pending_.push_back(p); }
    void commit_particles(uint32_t next_id)
    {
        initialize_maps();
        const size_t n = pending_.size();
        std::vector<uint32_t> id(n);
        std::vector<int32_t> cell(n);
        std::vector<double> x(n * dim), xi(n * dim), v(n * dim);
        for (size_t p = 0; p < n; ++p) {
            id[p] = pending_[p].id;
            cell[p] = pending_[p].cell;
            for (int d = 0; d < dim; ++d) {
                x[p * dim + d] = pending_[p].location[d];
                xi[p * dim + d] = pending_[p].reference_location[d];
                v[p * dim + d] = pending_[p].velocity[d];
            }
        }
        check(pfem2gpu_set_particles(h_, (int64_t)n, id.data(), cell.data(), x.data(), xi.data(), v.data(), next_id),
              h_);
        pending_.clear();
    }

    pfem2gpu_stats stats()
    {
        pfem2gpu_stats s{};
        check(pfem2gpu_get_stats(h_, &s), h_);
        return s;
    }
    void synchronize() { check(pfem2gpu_synchronize(h_), h_); }

    // Differentiated window (no counterpart in the reference): `steps` steps
    // of correct + move without count correction from the current particles,
    // then the projection U; and the gradients of J (dJ/dU = gU) with respect
    // to the starting particle velocities (n x dim, particles() order), V
    // and Vold.  Vold or v0 may be null (no correction / the particles' own
    // velocities); outputs may be null.  The particles are not changed.
    void adjoint(int steps, int checkpoint_every, const double* V, const double* Vold, const double* v0,
                 const double* gU, double* U, double* g_v0, double* g_V, double* g_Vold)
    {
        check(pfem2gpu_adjoint(h_, steps, checkpoint_every, V, Vold, v0, gU, U, g_v0, g_V, g_Vold), h_);
    }
    pfem2gpu_handle* handle() const { return h_; }

    const Mesh& mesh() const { return mesh_; }
    // The handle, with the mesh uploaded (for FemSystems and direct C calls).
    pfem2gpu_handle* handle()
    {
        initialize_maps();
        return h_;
    }

private:
    template <typename T>
    static T* need(T* p)
    {
        if (!p) throw Error(PFEM2GPU_ERR_STATE, "pfem2gpu: solution vectors not bound (set_solution_vectors)");
        return p;
    }

    pfem2gpu_handle* h_ = nullptr;
    Mesh mesh_;
    bool maps_ = false;
    const double* V_ = nullptr;
    const double* Vold_ = nullptr;
    double* Vout_ = nullptr;
    std::vector<Particle<dim>> pending_;
};

// pfem2Fem's assembly methods (src/pfem2fem.cpp:247-510) on the mesh of a
// ParticleHandler: setup_system's sparsity pattern once, then per step the
// three systems (volume and boundary-face terms) into caller arrays, as
// matrices x nnz values on that pattern and right-hand sides x n_dofs.  The
// constraints and the solves stay with the caller.
template <int dim>
class FemSystems {
public:
    FemSystems(ParticleHandler<dim>& particles, double rho, double mu)
        : h_(particles.handle()), rho_(rho), mu_(mu), n_dofs_(particles.mesh().n_dofs)
    {
    }

    // DoFTools::make_sparsity_pattern for Q1 (setup_system, :78-94).
    void setup_system(std::vector<int32_t>& row_ptr, std::vector<int32_t>& cols)
    {
        int64_t nnz = 0;
        check(pfem2gpu_fem_pattern(h_, nullptr, nullptr, 0, &nnz), h_);
        cols.resize((size_t)nnz);
        row_ptr.resize((size_t)n_dofs_ + 1);
        check(pfem2gpu_fem_pattern(h_, row_ptr.data(), cols.data(), nnz, &nnz), h_);
        nnz_ = nnz;
    }
    // Boundary id of every cell face (-1 interior) and the Dirichlet id sets
    // (getVelocityDirichletBCpatchIDs, getPressureDirichletBCpatchIDs).
    void set_boundary(const std::vector<int32_t>& face_ids, const std::vector<int32_t>& velocity_dirichlet,
                      const std::vector<int32_t>& pressure_dirichlet)
    {
        check(pfem2gpu_fem_set_boundary(h_, face_ids.data(), (int32_t)velocity_dirichlet.size(),
                                        velocity_dirichlet.data(), (int32_t)pressure_dirichlet.size(),
                                        pressure_dirichlet.data()),
              h_);
    }
    // assemble_velocity_prediction (:247-383): dim matrices, dim right-hand sides.
    void assemble_velocity_prediction(double time_step, const double* V, const double* Vold, double* A, double* rhs)
    {
        check(pfem2gpu_fem_assemble(h_, PFEM2GPU_FEM_PREDICTION, rho_, mu_, time_step, V, Vold, nullptr, A, rhs), h_);
    }
    // assemble_pressure_equation (:393-449): one matrix, one right-hand side.
    void assemble_pressure_equation(double time_step, const double* predictionV, double* A, double* rhs)
    {
        check(pfem2gpu_fem_assemble(h_, PFEM2GPU_FEM_PRESSURE, rho_, mu_, time_step, predictionV, nullptr, nullptr, A,
                                    rhs),
              h_);
    }
    // assemble_velocity_correction (:461-510): one matrix, dim right-hand sides.
    void assemble_velocity_correction(double time_step, const double* predictionV, const double* P, double* A,
                                      double* rhs)
    {
        check(pfem2gpu_fem_assemble(h_, PFEM2GPU_FEM_CORRECTION, rho_, mu_, time_step, predictionV, nullptr, P, A,
                                    rhs),
              h_);
    }
    // velocity_prediction_bc (:150-245): the prediction's Dirichlet rows and
    // their values (values[d * rows.size() + k]) from the pressure P, for the
    // Dirichlet velocities of the listed boundary ids.
    void velocity_prediction_bc(double time_step, const double* P, const std::vector<int32_t>& ids,
                                const std::vector<double>& id_velocities, std::vector<int32_t>& rows,
                                std::vector<double>& values)
    {
        int64_t n = 0;
        check(pfem2gpu_fem_velocity_bc(h_, rho_, time_step, P, (int32_t)ids.size(), ids.data(), id_velocities.data(),
                                       nullptr, nullptr, 0, &n),
              h_);
        rows.resize((size_t)n);
        values.resize((size_t)n * dim);
        check(pfem2gpu_fem_velocity_bc(h_, rho_, time_step, P, (int32_t)ids.size(), ids.data(), id_velocities.data(),
                                       rows.data(), values.data(), n, &n),
              h_);
    }
    // The constraints' effect on an assembled system (Dirichlet rows).
    void apply_dirichlet(int system, const std::vector<int32_t>& rows, const std::vector<double>& values, double* A,
                         double* rhs)
    {
        check(pfem2gpu_fem_constrain(h_, system, (int32_t)rows.size(), rows.data(), values.data(), A, rhs), h_);
    }
    int64_t nnz() const { return nnz_; }

private:
    pfem2gpu_handle* h_;
    double rho_, mu_;
    int64_t n_dofs_, nnz_ = 0;
};

}  // namespace pfem2gpu

#endif
