// pfem2particlehandler_b200.cpp -- the reference's pfem2ParticleHandler<dim>
// (src/pfem2particlehandler.h, used unchanged) implemented over the C ABI of
// libpfem2gpu.so (include/pfem2gpu.h).
//
// A build of the reference compiles this file instead of
// src/pfem2particlehandler.cpp (pfem2gpu.cmake: option PFEM2_WITH_B200), so
// pfem2Solver, pfem2Fem and the case drivers compile and run unchanged: the
// loop of src/pfem2solver.cpp:154-164 calls seed_particles, initialize_maps,
// correct_particle_velocity, move_particles and project_particle_fields on
// the same class, and these run on one GPU.
//
// The reference header leaves no member for the device state, so each
// handler object's state lives in a table keyed by the object's address,
// created on first use and released by the destructor.  The particles stay
// on the device; begin()/end() serve a host copy of them (refreshed whenever
// the device particles changed), and insert_particle/remove_particle/
// clear_particles edit that copy, which is sent back to the device before
// the next particle operation.  Changes made to particles through the
// iterators themselves are not sent back.
//
// Mesh: the locally owned active cells of the DoFHandler in iteration order,
// their vertices (cell->vertex(i), cell->vertex_index(i)) and vertex DoFs
// (cell->vertex_dof_index(i, 0), the reference's set_cell_dofs,
// src/pfem2particle.cpp:83-87); the vertex maps of initialize_maps are built
// on the device.  One MPI rank: the reference's particle migration
// (send_recv_particles) has no counterpart here, so a run on more ranks
// throws.
//
// Nodal velocities cross the boundary once per call as component-major
// arrays read from (getSolutionV, getOldSolutionV) and written to
// (setSolutionV) the FEM solver, as the reference reads and writes them
// (src/pfem2fem.cpp:622-644).  Old solution: fem_step copies the projected
// velocity into it (src/pfem2fem.cpp:523-524) before solving, so after the
// first projection correct_particle_velocity uses the handler's own last
// projection, kept on the device (pfem2gpu_correct_from_projection), and
// uploads V only.  Define PFEM2_B200_UPLOAD_OLD_SOLUTION to upload the old
// solution every step instead.
//
// Form: the FP64 form (the reference's arithmetic) unless PFEM2_B200_FP32
// is defined.  Sub-steps: Euler (the reference's) unless PFEM2_B200_RK2 is
// defined (the midpoint rule, which the reference does not have).  Errors of the C ABI throw std::runtime_error with the
// library's message; the reference throws deal.II exceptions.
#include "pfem2particlehandler.h"

#include <cstdint>
#include <fstream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "pfem2fem.h"
#include "pfem2gpu.h"
#include "pfem2parameterhandler.h"
#include "pfem2solver.h"

namespace {

#ifdef PFEM2_B200_FP32
constexpr int kPrecision = PFEM2GPU_FP32;
#else
constexpr int kPrecision = PFEM2GPU_FP64;
#endif

void check(int rc, pfem2gpu_handle* h, const char* what)
{
    if (rc == PFEM2GPU_OK) return;
    std::string msg = std::string("pfem2ParticleHandler (B200): ") + what + ": " + pfem2gpu_error_string(rc);
    if (h) {
        char buf[512] = {0};
        if (pfem2gpu_last_error(h, buf, sizeof buf) == PFEM2GPU_OK && buf[0]) msg += std::string(" (") + buf + ")";
    }
    throw std::runtime_error(msg);
}

template <int dim>
struct DeviceState {
    pfem2gpu_handle* h = nullptr;
    bool has_mesh = false;
    bool has_projection = false;
    bool host_copy_valid = false;  // `particles` equals the device particles
    bool host_copy_edited = false; // `particles` was edited: send it before the next device operation
    int64_t n_cells = 0, n_dofs = 0;
    std::vector<int32_t> cell_dofs;   // n_cells x 2^dim
    std::vector<int32_t> cell_index;  // device cell -> cell->index() (tria_position)
    std::map<int, int32_t> index_to_cell;
    std::vector<double> V, Vold, Vout;  // component-major, dim x n_dofs

    ~DeviceState()
    {
        if (h) pfem2gpu_destroy(h);
    }
};

template <int dim>
std::map<const void*, std::unique_ptr<DeviceState<dim>>>& states()
{
    static std::map<const void*, std::unique_ptr<DeviceState<dim>>> table;
    return table;
}

template <int dim>
DeviceState<dim>& state_of(const void* handler)
{
    auto& t = states<dim>();
    auto it = t.find(handler);
    if (it == t.end()) it = t.emplace(handler, std::make_unique<DeviceState<dim>>()).first;
    return *it->second;
}

template <int dim>
void read_vectors(const std::array<TrilinosWrappers::MPI::Vector, dim>& src, int64_t n_dofs, std::vector<double>& dst)
{
    dst.resize((size_t)dim * n_dofs);
    for (int d = 0; d < dim; ++d)
        for (int64_t k = 0; k < n_dofs; ++k) dst[(size_t)d * n_dofs + k] = src[d]((types::global_dof_index)k);
}

}  // namespace

template <int dim>
pfem2ParticleHandler<dim>::pfem2ParticleHandler(const FE_Q<dim>* finite_element)
    : particles()
    , quantities()
    , particleCount(0)
    , mainSolver(nullptr)
    , feq(finite_element)
{
}

template <int dim>
pfem2ParticleHandler<dim>::~pfem2ParticleHandler()
{
    clear_particles();
    states<dim>().erase(this);
}

template <int dim>
const pfem2Solver<dim>* pfem2ParticleHandler<dim>::getPfem2Solver() const
{
    return mainSolver;
}

// setPfem2Solver (src/pfem2particlehandler.cpp:30-40): the sub-step count,
// the sub-step length and the per-part maximum; the device handle is made
// by the first call that needs it, when the per-cell counts are known too.
template <int dim>
void pfem2ParticleHandler<dim>::setPfem2Solver(pfem2Solver<dim>* mainSolver)
{
    this->mainSolver = mainSolver;
    particle_integration_steps = mainSolver->getParameterHandler().getParticleIntegrationSteps();
    if (particle_integration_steps == 0) particle_integration_steps = 1;
    this->particle_transport_timestep =
        mainSolver->getParameterHandler().getTimeStep() / (double)particle_integration_steps;
    this->maxParticlesPerCellPart = mainSolver->getParameterHandler().getMaxParticlesPerCellPart();
}

namespace {

// The device handle and the mesh of the handler's solver, made once.
template <int dim>
DeviceState<dim>& device_for(pfem2ParticleHandler<dim>* self, pfem2Solver<dim>* solver,
                             const std::array<unsigned int, dim>& quantities, unsigned int max_per_part,
                             unsigned int steps)
{
    DeviceState<dim>& s = state_of<dim>(self);
    if (!solver) throw std::runtime_error("pfem2ParticleHandler (B200): setPfem2Solver was not called");
    if (Utilities::MPI::n_mpi_processes(solver->getCommunicator()) != 1)
        throw std::runtime_error("pfem2ParticleHandler (B200): runs on one MPI rank");
    if (!s.h) {
        pfem2gpu_params p{};
        for (int d = 0; d < 3; ++d) p.particles_per_cell[d] = d < dim ? (int32_t)quantities[d] : 1;
        p.max_particles_per_cell_part = (int32_t)max_per_part;
        p.particle_integration_steps = (int32_t)steps;
        p.time_step = solver->getParameterHandler().getTimeStep();
#ifdef PFEM2_B200_RK2
        p.integrator = PFEM2GPU_RK2;
#endif
        check(pfem2gpu_create(dim, kPrecision, &p, &s.h), nullptr, "create");
    }
    if (!s.has_mesh) {
        constexpr int NV = GeometryInfo<dim>::vertices_per_cell;
        const auto& dof_handler = solver->getFemSolver().getDoFhandler();
        std::vector<double> vertices;
        std::vector<int32_t> cell_vertices;
        std::map<unsigned int, int32_t> vertex_id;  // triangulation vertex -> device vertex
        s.cell_dofs.clear();
        s.cell_index.clear();
        s.index_to_cell.clear();
        for (const auto& cell : dof_handler.active_cell_iterators()) {
            if (!cell->is_locally_owned()) continue;
            s.index_to_cell[cell->index()] = (int32_t)s.cell_index.size();
            s.cell_index.push_back(cell->index());
            for (int i = 0; i < NV; ++i) {
                const unsigned int vi = cell->vertex_index(i);
                auto it = vertex_id.find(vi);
                if (it == vertex_id.end()) {
                    it = vertex_id.emplace(vi, (int32_t)(vertices.size() / dim)).first;
                    const Point<dim> x = cell->vertex(i);
                    for (int d = 0; d < dim; ++d) vertices.push_back(x[d]);
                }
                cell_vertices.push_back(it->second);
                s.cell_dofs.push_back((int32_t)cell->vertex_dof_index(i, 0));
            }
        }
        s.n_cells = (int64_t)s.cell_index.size();
        s.n_dofs = (int64_t)dof_handler.n_dofs();
        check(pfem2gpu_set_mesh(s.h, s.n_cells, (int64_t)(vertices.size() / dim), s.n_dofs, vertices.data(),
                                cell_vertices.data(), s.cell_dofs.data(), nullptr, nullptr, nullptr),
              s.h, "set_mesh");
        s.has_mesh = true;
    }
    return s;
}

// Send the edited host copy of the particles back to the device.
template <int dim>
void send_host_copy(DeviceState<dim>& s, const std::vector<pfem2Particle<dim>>& particles, int particle_count)
{
    if (!s.host_copy_edited) return;
    const size_t n = particles.size();
    std::vector<uint32_t> id(n);
    std::vector<int32_t> cell(n);
    std::vector<double> x(n * dim), xi(n * dim), v(n * dim);
    for (size_t k = 0; k < n; ++k) {
        const auto& p = particles[k];
        auto it = s.index_to_cell.find(p.get_tria_position());
        if (it == s.index_to_cell.end())
            throw std::runtime_error("pfem2ParticleHandler (B200): particle in a cell this rank does not own");
        id[k] = p.get_id();
        cell[k] = it->second;
        for (int d = 0; d < dim; ++d) {
            x[k * dim + d] = p.get_location()[d];
            xi[k * dim + d] = p.get_reference_location()[d];
            v[k * dim + d] = p.get_velocity_component(d);
        }
    }
    check(pfem2gpu_set_particles(s.h, (int64_t)n, id.data(), cell.data(), x.data(), xi.data(), v.data(),
                                 (uint32_t)particle_count),
          s.h, "set_particles");
    s.host_copy_edited = false;
    s.host_copy_valid = true;
}

}  // namespace

// seed_particles (src/pfem2particlehandler.cpp:43-109): every part of every
// locally owned cell gets a particle at its centre with the interpolated
// FEM velocity; ids continue particleCount.
template <int dim>
void pfem2ParticleHandler<dim>::seed_particles()
{
    TimerOutput::Scope timer_section(mainSolver->getTimer(), "Particle seeding");
    quantities = mainSolver->getParameterHandler().getParticlesPerCell();
    DeviceState<dim>& s = device_for<dim>(this, mainSolver, quantities, maxParticlesPerCellPart,
                                          particle_integration_steps);
    read_vectors<dim>(mainSolver->getFemSolver().getSolutionV(), s.n_dofs, s.V);
    check(pfem2gpu_seed(s.h, s.V.data()), s.h, "seed");
    pfem2gpu_stats st{};
    check(pfem2gpu_get_stats(s.h, &st), s.h, "get_stats");
    particleCount = (int)st.next_id;
    s.host_copy_valid = false;
    std::cout << "Created and placed " << particleCount << " particles on process "
              << Utilities::MPI::this_mpi_process(mainSolver->getCommunicator()) << std::endl;
}

// initialize_maps (:320-324): the vertex maps are built on the device when
// the mesh is set; this only makes sure that has happened.
template <int dim>
void pfem2ParticleHandler<dim>::initialize_maps()
{
    if (quantities[0] == 0) quantities = mainSolver->getParameterHandler().getParticlesPerCell();
    device_for<dim>(this, mainSolver, quantities, maxParticlesPerCellPart, particle_integration_steps);
}

// correct_particle_velocity (:112-139): v += sum_i N_i (V - Vold)_i.
template <int dim>
void pfem2ParticleHandler<dim>::correct_particle_velocity()
{
    TimerOutput::Scope timer_section(mainSolver->getTimer(), "Particle velocity correction");
    DeviceState<dim>& s = state_of<dim>(this);
    send_host_copy<dim>(s, particles, particleCount);
    read_vectors<dim>(mainSolver->getFemSolver().getSolutionV(), s.n_dofs, s.V);
#ifndef PFEM2_B200_UPLOAD_OLD_SOLUTION
    if (s.has_projection) {
        check(pfem2gpu_correct_from_projection(s.h, s.V.data()), s.h, "correct_from_projection");
        s.host_copy_valid = false;
        return;
    }
#endif
    read_vectors<dim>(mainSolver->getFemSolver().getOldSolutionV(), s.n_dofs, s.Vold);
    check(pfem2gpu_correct(s.h, s.V.data(), s.Vold.data()), s.h, "correct");
    s.host_copy_valid = false;
}

// move_particles (:142-171): the sub-steps with relocation, then
// check_particle_distribution, in the solution velocity staged by the
// correction (or uploaded here when no correction preceded).
template <int dim>
void pfem2ParticleHandler<dim>::move_particles()
{
    TimerOutput::Scope timer_section(mainSolver->getTimer(), "Particle transport");
    DeviceState<dim>& s = state_of<dim>(this);
    send_host_copy<dim>(s, particles, particleCount);
    read_vectors<dim>(mainSolver->getFemSolver().getSolutionV(), s.n_dofs, s.V);
    check(pfem2gpu_move(s.h, s.V.data()), s.h, "move");
    s.host_copy_valid = false;
}

// project_particle_fields (:174-215): V = sum N v / sum N per DoF, handed to
// the FEM solver with setSolutionV component by component.
template <int dim>
void pfem2ParticleHandler<dim>::project_particle_fields()
{
    TimerOutput::Scope timer_section(mainSolver->getTimer(), "Particle fields projection");
    DeviceState<dim>& s = state_of<dim>(this);
    send_host_copy<dim>(s, particles, particleCount);
    s.Vout.resize((size_t)dim * s.n_dofs);
    check(pfem2gpu_project(s.h, s.Vout.data()), s.h, "project");
    s.has_projection = true;
    pfem2gpu_stats st{};
    check(pfem2gpu_get_stats(s.h, &st), s.h, "get_stats");
    particleCount = (int)st.next_id;
    for (int d = 0; d < dim; ++d) {
        TrilinosWrappers::MPI::Vector nodeVelocity;
        nodeVelocity.reinit(mainSolver->getFemSolver().getLocallyOwnedDofs(), mainSolver->getCommunicator());
        const auto range = nodeVelocity.local_range();
        for (auto k = range.first; k < range.second; ++k) nodeVelocity[k] = s.Vout[(size_t)d * s.n_dofs + k];
        nodeVelocity.compress(VectorOperation::insert);
        mainSolver->getFemSolver().setSolutionV(nodeVelocity, d);
    }
}

// output_particle_solution (:218-317): the VTU file of this rank (from the
// particles packed on the device) and the .pvtu of rank 0.
template <int dim>
void pfem2ParticleHandler<dim>::output_particle_solution(int timestep_number)
{
    DeviceState<dim>& s = state_of<dim>(this);
    send_host_copy<dim>(s, particles, particleCount);
    const std::string base = "particles-" + Utilities::int_to_string(timestep_number, 2);
    const std::string vtu = base + "." + Utilities::int_to_string(Utilities::MPI::this_mpi_process(mainSolver->getCommunicator()), 3) + ".vtu";
    check(pfem2gpu_write_vtu(s.h, vtu.c_str()), s.h, "write_vtu");
    std::ofstream master((base + ".pvtu").c_str());
    master << "<?xml version=\"1.0\" ?> \n<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" "
              "byte_order=\"LittleEndian\">\n  <PUnstructuredGrid GhostLevel=\"0\">\n"
              "    <PPointData Scalars=\"scalars\">\n"
              "      <PDataArray type=\"Float32\" Name=\"velocity\" NumberOfComponents=\"3\" format=\"ascii\"/>\n"
              "      <PDataArray type=\"Float32\" Name=\"subdomain\" format=\"ascii\"/>\n    </PPointData>\n"
              "    <PPoints>\n      <PDataArray type=\"Float32\" NumberOfComponents=\"3\"/>\n    </PPoints>\n"
           << "    <Piece Source=\"" << vtu << "\"/>  </PUnstructuredGrid>\n</VTKFile>\n";
}

template <int dim>
void pfem2ParticleHandler<dim>::clear_particles()
{
    particles.clear();
    auto& t = states<dim>();
    auto it = t.find(this);
    if (it != t.end() && it->second->h) {
        it->second->host_copy_valid = true;
        it->second->host_copy_edited = true;
    }
}

template <int dim>
pfem2ParticleIterator<dim> pfem2ParticleHandler<dim>::remove_particle(pfem2ParticleIterator<dim> particleIndex)
{
    DeviceState<dim>& s = state_of<dim>(this);
    const auto off = particleIndex - particles.begin();
    begin();  // the host copy is current before it is edited
    s.host_copy_edited = true;
    return particles.erase(particles.begin() + off);
}

template <int dim>
void pfem2ParticleHandler<dim>::insert_particle(pfem2Particle<dim>& particle,
                                                const typename DoFHandler<dim>::active_cell_iterator& cell)
{
    DeviceState<dim>& s = state_of<dim>(this);
    if (s.h && s.has_mesh) {
        begin();
        s.host_copy_edited = true;
    }
    particle.set_tria_position(cell->index());
    particle.set_cell_dofs(cell);
    particles.push_back(particle);
}

// begin()/end(): the host copy of the device particles (pfem2gpu_get_particles).
template <int dim>
pfem2ParticleIterator<dim> pfem2ParticleHandler<dim>::begin()
{
    DeviceState<dim>& s = state_of<dim>(this);
    if (s.h && s.has_mesh && !s.host_copy_valid && !s.host_copy_edited) {
        constexpr int NV = GeometryInfo<dim>::vertices_per_cell;
        int64_t n = 0;
        check(pfem2gpu_get_particles(s.h, nullptr, nullptr, nullptr, nullptr, nullptr, 0, &n), s.h, "get_particles");
        std::vector<uint32_t> id(n);
        std::vector<int32_t> cell(n);
        std::vector<double> x(n * dim), xi(n * dim), v(n * dim);
        check(pfem2gpu_get_particles(s.h, id.data(), cell.data(), x.data(), xi.data(), v.data(), n, &n), s.h,
              "get_particles");
        particles.clear();
        particles.reserve(n);
        for (int64_t k = 0; k < n; ++k) {
            Point<dim> loc, ref;
            Tensor<1, dim> vel;
            for (int d = 0; d < dim; ++d) {
                loc[d] = x[k * dim + d];
                ref[d] = xi[k * dim + d];
                vel[d] = v[k * dim + d];
            }
            pfem2Particle<dim> p(loc, ref, id[k]);
            p.set_velocity(vel);
            p.set_tria_position(s.cell_index[cell[k]]);
            for (int i = 0; i < NV; ++i) p.cell_dofs[i] = s.cell_dofs[(size_t)cell[k] * NV + i];
            particles.push_back(p);
        }
        s.host_copy_valid = true;
    }
    return particles.begin();
}

template <int dim>
pfem2ParticleIterator<dim> pfem2ParticleHandler<dim>::end()
{
    return particles.end();
}

// The explicit instantiations for dim 2 and 3 are those at the end of
// src/pfem2particlehandler.h.
