/*
 * pfem2gpu.h -- C ABI of the B200 PFEM-2 particle path.
 *
 * Drop-in for the particle cycle of pfem2ParticleHandler<dim>
 * (src/pfem2particlehandler.h:17-71 of the reference): seeding, velocity
 * correction, sub-stepped transport with relocation and count correction,
 * and the particle-to-mesh velocity projection.  The FEM step stays with the
 * caller; nodal velocities cross this boundary once per call as plain
 * component-major double arrays, V[d * n_dofs + dof], the layout of the
 * reference's std::array<TrilinosWrappers::MPI::Vector, dim>.
 *
 * Conventions: every function returns PFEM2GPU_OK (0) or an error code; no
 * C++ exception crosses the ABI.  One handle is used from one host thread.
 * All device work of a handle runs in order on the handle's CUDA stream, on
 * the device that was current at pfem2gpu_create.  Host input arrays are
 * read before the call returns unless they were registered with
 * pfem2gpu_host_register, in which case they must stay unchanged until the
 * next call that returns host data (project, get_particles, get_stats,
 * synchronize).
 */
#ifndef PFEM2GPU_H
#define PFEM2GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFEM2GPU_OK 0
#define PFEM2GPU_ERR_ARG 1        /* invalid argument or size */
#define PFEM2GPU_ERR_CUDA 2       /* CUDA runtime error (details: pfem2gpu_last_error) */
#define PFEM2GPU_ERR_STATE 3      /* call out of order (no mesh, no particles, ...) */
#define PFEM2GPU_ERR_CAPACITY 4   /* particle arrays full; raise params.capacity */
#define PFEM2GPU_ERR_NOMEM 5      /* device allocation failed */
#define PFEM2GPU_ERR_NODEVICE 6   /* no CUDA device */
#define PFEM2GPU_ERR_DEVICE 7     /* a kernel reported bad input (see stats.error_flags) */
#define PFEM2GPU_ERR_SCRATCH 8    /* pfem2gpu_project_noalloc: mesh larger than its static scratch */

#define PFEM2GPU_FP64 0           /* plain form: the reference's arithmetic, FP64 state */
#define PFEM2GPU_FP32 1           /* FP32 state and interpolation, FP64 for face crossings */

/* Particle parameters; the names follow the reference's .prm keys
 * (src/pfem2parameterhandler.cpp:64-74, 40). */
typedef struct pfem2gpu_params {
    int32_t particles_per_cell[3];        /* "Number of particles in the x/y/z direction" */
    int32_t max_particles_per_cell_part;  /* "Maximum number of particles per cell part" */
    int32_t particle_integration_steps;   /* "Particle integration steps" (0 -> 1) */
    double time_step;                     /* "Time step" (sub-step = time_step / steps) */
    uint32_t removal_seed;                /* over-full parts keep the smallest key(id); 0: key = id */
    int32_t empty_dof_policy;             /* 0: reference (0/0 = NaN at DoFs no particle reaches); 1: keep input V */
    int64_t capacity;                     /* particle capacity (0: 2 x cells x parts) */
    int32_t integrator;                   /* PFEM2GPU_EULER (the reference's sub-steps) or PFEM2GPU_RK2 */
} pfem2gpu_params;

/* Sub-step integrators.  Euler is the reference's move_particles
 * (src/pfem2particlehandler.cpp:151-163): x += h u(xi).  RK2 has no
 * counterpart in the reference: the midpoint rule in the particle's own cell,
 * x += h u(xi_mid) with xi_mid = xi + (h/2) J(xi)^-1 u(xi) and u the cell's Q1
 * field (extrapolated where xi_mid lies outside the unit cell; a
 * non-positive Jacobian determinant falls back to u(xi)); second order.  The
 * differentiated window supports Euler only (PFEM2GPU_ERR_ARG with RK2). */
#define PFEM2GPU_EULER 0
#define PFEM2GPU_RK2 1

typedef struct pfem2gpu_stats {
    int64_t n_particles;
    int64_t lost;          /* deleted by relocation (left the mesh) */
    int64_t removed;       /* deleted by count correction */
    int64_t seeded;        /* inserted by count correction */
    int64_t map_failures;  /* inverse-map failures (ExcTransformationFailed) */
    int64_t near_face;     /* relocations ending within 1e-12 of a face */
    int64_t searched;      /* relocations that needed the vertex-patch search */
    int64_t nan_dofs;      /* DoFs without particle weight in the last projection */
    int64_t fallback64;    /* FP32 form: sub-steps relocated in FP64 */
    int64_t particle_steps;/* particles advanced, summed over all moves */
    uint32_t next_id;      /* last particle id handed out (particleCount) */
    uint32_t error_flags;  /* 1 capacity, 2 vertex with > 64 cells, 4 bad cell index */
} pfem2gpu_stats;

typedef struct pfem2gpu_handle pfem2gpu_handle;

/* Constructor + setPfem2Solver (src/pfem2particlehandler.cpp:10-15,30-40). */
int pfem2gpu_create(int dim, int precision, const pfem2gpu_params* params, pfem2gpu_handle** out);
int pfem2gpu_destroy(pfem2gpu_handle* h);

/* Mesh and initialize_maps (src/pfem2particlehandler.cpp:320-324).
 * vertices: n_verts x dim; cell_vertices, cell_dofs: n_cells x 2^dim in deal.II
 * lexicographic vertex order (the DoF of vertex i is cell->vertex_dof_index(i,0),
 * src/pfem2particle.cpp:83-87).  The vertex maps (GridTools::vertex_to_cell_map,
 * vertex_to_cell_centers_directions) may be passed (offsets n_verts+1, cells
 * ascending, unit directions dim per entry) or NULL to have them built on the
 * device (counting sort by vertex, cells ascending, FP64 directions centre -
 * vertex normalised by the square root of the sum of squares). */
int pfem2gpu_set_mesh(pfem2gpu_handle* h, int64_t n_cells, int64_t n_verts, int64_t n_dofs,
                      const double* vertices, const int32_t* cell_vertices, const int32_t* cell_dofs,
                      const int32_t* v2c_offsets, const int32_t* v2c_cells, const double* v2c_dirs);

/* The vertex maps in use (given or built), copied to host arrays: offsets
 * n_verts+1, cells and dirs (dim per entry) of >= capacity entries; *n = the
 * number of entries.  With cells and dirs NULL only offsets and *n are
 * read (the query for the capacity). */
int pfem2gpu_get_vertex_maps(pfem2gpu_handle* h, int32_t* offsets, int32_t* cells, double* dirs, int64_t capacity,
                             int64_t* n);

/* GridIn::read_unv as the reference's solver calls it
 * (src/pfem2solver.cpp:116-119), host only (no device needed): datasets 2411
 * (nodes) and 2412 (elements) of an I-DEAS universal file; quads (44, 94) in
 * 2D, hexes (115) in 3D become cells in deal.II's lexicographic vertex order,
 * left-handed cells get their first two directions swapped, nodes no cell
 * uses are dropped and vertices are numbered by ascending node label.  dim 0
 * takes it from the elements (*dim_out: the mesh's).  With vertices and
 * cell_vertices NULL only the counts are returned; then arrays of
 * n_verts x dim and n_cells x 2^dim.
 * The reason of a failure: pfem2gpu_read_unv_error(). */
int pfem2gpu_read_unv(const char* path, int dim, int32_t* dim_out, int64_t* n_verts, int64_t* n_cells,
                      double* vertices, int32_t* cell_vertices, int64_t verts_capacity, int64_t cells_capacity);
const char* pfem2gpu_read_unv_error(void);

/* ---------------------------------------------------------------------------
 * The solver step's Q1 systems (src/pfem2fem.cpp): the volume integrals of
 * assemble_velocity_prediction (:247-319, SCHEMEB off),
 * assemble_pressure_equation (:393-435) and assemble_velocity_correction
 * (:461-510), computed per cell on the device in FP64 (QGauss(2), the Q1
 * map's Jacobian at each point) and summed into CSR matrices and right-hand
 * sides in ascending cell order, as a cell loop adds local systems.  With
 * boundary ids set (pfem2gpu_fem_set_boundary), the boundary-face terms of
 * the prediction (:320-383) and of the pressure equation (:436-449) are
 * added on the faces outside the Dirichlet sets.  The constraints
 * (AffineConstraints::distribute_local_to_global) stay with the caller.
 * ------------------------------------------------------------------------- */
#define PFEM2GPU_FEM_PREDICTION 0 /* U = solution V, U2 = old solution V: dim matrices, dim right-hand sides */
#define PFEM2GPU_FEM_PRESSURE 1   /* U = predicted V: one matrix, one right-hand side */
#define PFEM2GPU_FEM_CORRECTION 2 /* U = predicted V, P = pressure: one matrix, dim right-hand sides */

/* CSR pattern of the matrices (DoFTools::make_sparsity_pattern for Q1: per
 * DoF the DoFs sharing a cell with it, ascending), built on the device once
 * per mesh; row_ptr n_dofs+1, cols >= capacity entries (NULL: *nnz only). */
int pfem2gpu_fem_pattern(pfem2gpu_handle* h, int32_t* row_ptr, int32_t* cols, int64_t capacity, int64_t* nnz);
/* Boundary ids per cell and face (n_cells x 2 dim, deal.II face numbering:
 * face 2d lies at xi_d = 0, face 2d+1 at xi_d = 1; -1 for an interior face)
 * and the Dirichlet sets (getVelocityDirichletBCpatchIDs,
 * getPressureDirichletBCpatchIDs): the prediction gets face terms on
 * boundary faces outside the velocity set, the pressure equation on those
 * outside the pressure set.  face_ids NULL: no face terms. */
int pfem2gpu_fem_set_boundary(pfem2gpu_handle* h, const int32_t* face_ids, int32_t n_velocity_dirichlet,
                              const int32_t* velocity_dirichlet, int32_t n_pressure_dirichlet,
                              const int32_t* pressure_dirichlet);
/* One system on device vectors (component-major U, U2 of dim x n_dofs; P of
 * n_dofs): A receives matrices x nnz values on the pattern, rhs right-hand
 * sides x n_dofs.  Enqueued on the handle's stream, not synchronized.  rho,
 * mu and dt as the reference's fluid density, viscosity and time step. */
int pfem2gpu_fem_assemble_device(pfem2gpu_handle* h, int system, double rho, double mu, double dt, const double* dU,
                                 const double* dU2, const double* dP, double* dA, double* drhs);
/* The same on host arrays (copies in and out, synchronized). */
int pfem2gpu_fem_assemble(pfem2gpu_handle* h, int system, double rho, double mu, double dt, const double* U,
                          const double* U2, const double* P, double* A, double* rhs);
/* Dirichlet rows on an assembled system: the effect, summed over the cells,
 * of AffineConstraints::distribute_local_to_global for constraints
 * x_r = g_r without coupling (interpolate_boundary_values, and the
 * inhomogeneities of velocity_prediction_bc, src/pfem2fem.cpp:150-245).  A
 * constrained row keeps its diagonal A_rr alone and its right-hand side
 * becomes A_rr g_r; every other row moves A_rc g_c of each constrained
 * column c (ascending) to its right-hand side and zeroes A_rc.  rows: n
 * distinct DoFs; values: one set of n values per right-hand side of the
 * system (right-hand side q uses matrix min(q, matrices - 1)).  The _device
 * form works on device A and rhs (rows and values are host arrays). */
/* velocity_prediction_bc (src/pfem2fem.cpp:150-245): the values of the
 * prediction's Dirichlet rows, on the DoFs of the boundary faces in the
 * velocity Dirichlet set of pfem2gpu_fem_set_boundary: the face integral of
 * the pressure gradient, times dt / rho, divided by the face integral of the
 * shape function, plus the Dirichlet velocity of the boundary id (ids[k] ->
 * velocities[k * dim ..]; of the last such face in cell and face order, as
 * the reference's map keeps; an id not listed counts as zero).  P: pressure
 * at the DoFs.  Out: rows (ascending) and values[d * n + k]; NULL arrays
 * return *n only.  Feed them to pfem2gpu_fem_constrain. */
int pfem2gpu_fem_velocity_bc(pfem2gpu_handle* h, double rho, double dt, const double* P, int32_t n_ids,
                             const int32_t* ids, const double* velocities, int32_t* rows, double* values,
                             int64_t capacity, int64_t* n);
int pfem2gpu_fem_constrain(pfem2gpu_handle* h, int system, int32_t n, const int32_t* rows, const double* values,
                           double* A, double* rhs);
int pfem2gpu_fem_constrain_device(pfem2gpu_handle* h, int system, int32_t n, const int32_t* rows,
                                  const double* values, double* dA, double* drhs);

/* seed_particles (src/pfem2particlehandler.cpp:43-109). */
int pfem2gpu_seed(pfem2gpu_handle* h, const double* V);
/* correct_particle_velocity (:112-139): v += sum N_i (V - Vold)_i; applied
 * fused with the next move, or before any call that reads particles. */
int pfem2gpu_correct(pfem2gpu_handle* h, const double* V, const double* Vold);
/* correct_particle_velocity with Vold = the handle's last projection
 * (pfem2gpu_project / pfem2gpu_step_device), which stays on the device: the
 * reference's data flow, where fem_step copies the projected velocity into
 * the old solution (src/pfem2fem.cpp:523-524) before it solves for the new
 * one (src/pfem2solver.cpp:162-165), so only V crosses the boundary.
 * PFEM2GPU_ERR_STATE before the first projection. */
int pfem2gpu_correct_from_projection(pfem2gpu_handle* h, const double* V);
/* move_particles (:142-171): sub-steps + relocation + count correction.
 * V == NULL reuses the velocity of the preceding seed/correct/move call. */
int pfem2gpu_move(pfem2gpu_handle* h, const double* V);
/* project_particle_fields (:174-215): V_out = sum N v / sum N per DoF. */
int pfem2gpu_project(pfem2gpu_handle* h, double* V_out);

/* Same with device-resident vectors (same layout); project does not synchronize. */
int pfem2gpu_seed_device(pfem2gpu_handle* h, const double* dV);
int pfem2gpu_correct_device(pfem2gpu_handle* h, const double* dV, const double* dVold);
int pfem2gpu_move_device(pfem2gpu_handle* h, const double* dV);
int pfem2gpu_project_device(pfem2gpu_handle* h, double* dV_out);
int pfem2gpu_correct_from_projection_device(pfem2gpu_handle* h, const double* dV);
/* One whole time step (correct + move + project) on device vectors, replayed
 * as one CUDA graph after the first calls with the same pointers.  dVold NULL:
 * Vold = the handle's last projection, as pfem2gpu_correct_from_projection
 * (PFEM2GPU_ERR_STATE before the first projection); the step's projection
 * becomes the handle's last projection either way. */
int pfem2gpu_step_device(pfem2gpu_handle* h, const double* dV, const double* dVold, double* dV_out);

/* Particle access for output_particle_solution (:218-317) and begin()/end():
 * arrays sized >= capacity (n x dim for x, xi, v); any may be NULL.  *n gets
 * the particle count; PFEM2GPU_ERR_ARG if capacity is too small. */
int pfem2gpu_get_particles(pfem2gpu_handle* h, uint32_t* id, int32_t* cell, double* x, double* xi, double* v,
                           int64_t capacity, int64_t* n);
/* Replace the particle set (insert_particle/clear_particles, :327-344).
 * x is used by the FP64 form, ignored by the FP32 form. */
int pfem2gpu_set_particles(pfem2gpu_handle* h, int64_t n, const uint32_t* id, const int32_t* cell, const double* x,
                           const double* xi, const double* v, uint32_t next_id);
/* Particle VTU file as output_particle_solution writes it (rank 0 of 1);
 * the data come from pfem2gpu_pack_output_device in one copy. */
int pfem2gpu_write_vtu(pfem2gpu_handle* h, const char* path);
/* The data of output_particle_solution (:218-317) packed on the device as the
 * Float32 values its file holds: d_out[3k .. 3k+2] = position of the k-th
 * particle (pfem2gpu_get_particles order), d_out[3n + 3k .. 3n + 3k+2] = its
 * velocity (2D: third components 0).  d_out: device array of >= 6 x capacity
 * floats; *n gets the particle count (PFEM2GPU_ERR_ARG if capacity is
 * smaller).  Asynchronous on the handle's stream: synchronise before reading
 * d_out from another stream or the host. */
int pfem2gpu_pack_output_device(pfem2gpu_handle* h, float* d_out, int64_t capacity, int64_t* n);

/* ---------------------------------------------------------------------------
 * Cell-range partitions: one handle per GPU, each holding the whole mesh and
 * the whole nodal velocity and owning the particles of cells
 * [cell_begin, cell_end).  The reference distributes cells over MPI ranks and
 * sends the particles found in another rank's cells after each relocation
 * (send_recv_particles, src/pfem2particlehandler.cpp:480-502,507-618), and
 * sums the projection over the ghost cells of each DoF
 * (project_particle_fields, :202-205 compress(add)).  A partitioned move is
 * host-driven in three phases; the caller routes the outboxes to the owners
 * of their cells and scans the seed counts over the partitions in cell order:
 *
 *   begin(h, V, &n_out)            correct + sub-steps + relocation
 *   outbox(h, ..., &n)             particles that ended in foreign cells
 *   inbox(h, m, ..., &n_seeds)     particles that ended in this handle's cells
 *   end(h, first_id, next_id)      count correction, new layout, partials
 *
 * first_id = the ids handed out before this move + the seeds of all lower
 * partitions; next_id = the ids handed out before + every partition's seeds.
 * With those, every cell's particles, their order and their ids are those of
 * one unpartitioned handle, so the FP64 form is bit-identical to it.  The
 * projection then needs the partial sums of the cells that share a DoF with
 * this handle's cells (get/set_partials) before pfem2gpu_project; DoFs none of
 * whose cells are this handle's or were set are NaN (no particles).
 * pfem2gpu_move, pfem2gpu_move_device and pfem2gpu_step_device return
 * PFEM2GPU_ERR_STATE on a partitioned handle.
 * ------------------------------------------------------------------------- */
/* Own cells [cell_begin, cell_end) of the mesh; after set_mesh, before seed or
 * set_particles.  seed then seeds the own cells only, with the ids of an
 * unpartitioned seed (next_id afterwards = n_cells x particles per cell). */
int pfem2gpu_set_partition(pfem2gpu_handle* h, int64_t cell_begin, int64_t cell_end);
/* Phase 1: velocity correction (if pending), sub-steps and relocation; *n_out
 * gets the number of particles that ended in other partitions' cells.
 * V == NULL reuses the staged velocity. */
int pfem2gpu_move_exchange_begin(pfem2gpu_handle* h, const double* V, int64_t* n_out);
/* Phase 2a: those particles (arrays of >= capacity entries; x, xi, v row-major
 * n x dim; x may be NULL in the FP32 form); they leave this handle. */
int pfem2gpu_move_outbox(pfem2gpu_handle* h, uint32_t* id, int32_t* cell, double* x, double* xi, double* v,
                         int64_t capacity, int64_t* n);
/* Phase 2b: the particles other partitions sent to this handle's cells (all
 * of them, in any order); *n_seeds gets the number of particles the count
 * correction will add in this handle's cells.  PFEM2GPU_ERR_ARG if a cell is
 * foreign, PFEM2GPU_ERR_CAPACITY beyond the particle capacity. */
int pfem2gpu_move_inbox(pfem2gpu_handle* h, int64_t n, const uint32_t* id, const int32_t* cell, const double* x,
                        const double* xi, const double* v, int64_t* n_seeds);
/* Phase 3: count correction, sorted layout and projection partials; the new
 * particles get ids first_id + 1 ...; the handle's next id becomes next_id. */
int pfem2gpu_move_exchange_end(pfem2gpu_handle* h, uint32_t first_id, uint32_t next_id);
/* Projection partial sums of n cells (out/in: n x 32 doubles in 3D, n x 16 in
 * 2D, the per-vertex sum N v and sum N of the cell); valid after a move. */
int pfem2gpu_get_partials(pfem2gpu_handle* h, int64_t n, const int32_t* cells, double* out);
int pfem2gpu_set_partials(pfem2gpu_handle* h, int64_t n, const int32_t* cells, const double* in);

int pfem2gpu_get_stats(pfem2gpu_handle* h, pfem2gpu_stats* out);
int pfem2gpu_reset_stats(pfem2gpu_handle* h);
int pfem2gpu_synchronize(pfem2gpu_handle* h);
int pfem2gpu_get_stream(pfem2gpu_handle* h, void** stream);
int pfem2gpu_host_register(void* ptr, size_t bytes);
int pfem2gpu_host_unregister(void* ptr);

/* Timing hooks (the reference's TimerOutput sections, :114,144,176): with
 * profiling on, every launch is bracketed by CUDA events on the handle's
 * stream; the report is a JSON object {"kernel": [total_ms, launches], ...}. */
int pfem2gpu_profile(pfem2gpu_handle* h, int enable);
int pfem2gpu_profile_report(pfem2gpu_handle* h, char* buf, int64_t len);
int pfem2gpu_launch_count(pfem2gpu_handle* h, uint64_t* count);

/* ---------------------------------------------------------------------------
 * Differentiated window and its adjoint.
 *
 * No counterpart in the reference (it has no adjoint).  The window is
 * `steps` time steps of correct_particle_velocity (when Vold is given, with
 * the same V - Vold every step) and move_particles' sub-steps with relocation
 * (src/pfem2particlehandler.cpp:112-167, 413-503) from the handle's current
 * particles, with check_particle_distribution (:356-410) left out, followed by
 * project_particle_fields (:174-215): U = P(v0, V, Vold), dim x n_dofs
 * component-major (empty_dof_policy applies to DoFs no particle reaches).
 * The trajectories are the form's own (FP64 or FP32); particle velocities,
 * their corrections and the projection sums of the window are FP64 in both
 * forms, and the sums are deterministic.  The handle's
 * particles are not changed; the handle's staged velocity becomes V.
 *
 * The adjoint returns, for a given gU = dJ/dU of a scalar objective J, the
 * gradients dJ/dv0 (n x dim, one row per particle in the order of
 * pfem2gpu_get_particles at the window start, n = stats.n_particles),
 * dJ/dV and dJ/dVold (dim x n_dofs).  Every particle's cell sequence is held
 * fixed (cell assignment is discrete and not differentiated); particles
 * deleted inside the window get zero gradient.  The forward keeps the
 * particle state at the start of every `checkpoint_every` steps; the
 * backward recomputes one such segment at a time from its checkpoint, so
 * memory grows with steps / checkpoint_every, not with steps.
 * checkpoint_every x particle_integration_steps is limited by the backward
 * kernel's shared memory (about 200 states in 3D FP64): PFEM2GPU_ERR_ARG
 * beyond.  dJ/dV and dJ/dVold are summed with FP64 atomics per cell vertex:
 * their last bits can differ between runs; U and dJ/dv0 are deterministic.
 *
 * window_forward_device: device arrays (v0 may be NULL: the particles' own
 * velocities; Vold may be NULL: no correction).  window_backward_device
 * differentiates the most recent forward (it may be called again with another
 * gU); outputs may be NULL.  pfem2gpu_adjoint: forward + backward on host
 * arrays.  PFEM2GPU_ERR_DEVICE if a recomputed segment does not end where the
 * forward pass ended it (never expected).
 */
int pfem2gpu_window_forward_device(pfem2gpu_handle* h, int32_t steps, int32_t checkpoint_every, const double* dV,
                                   const double* dVold, const double* dv0, double* dU_out);
int pfem2gpu_window_backward_device(pfem2gpu_handle* h, const double* dgU, double* dg_v0, double* dg_V,
                                    double* dg_Vold);
int pfem2gpu_adjoint(pfem2gpu_handle* h, int32_t steps, int32_t checkpoint_every, const double* V, const double* Vold,
                     const double* v0, const double* gU, double* U, double* g_v0, double* g_V, double* g_Vold);
/* Particles of the most recent window forward (-1: none). */
int pfem2gpu_window_size(pfem2gpu_handle* h, int64_t* n);
/* Their states at the end of that window (cell -1: deleted inside it), host
 * arrays of >= capacity rows in the window's particle order. */
int pfem2gpu_window_particles(pfem2gpu_handle* h, int32_t* cell, double* xi, double* v, int64_t capacity, int64_t* n);

/* ---------------------------------------------------------------------------
 * pfem2gpu_project_noalloc -- projection that allocates no device memory.
 *
 * No counterpart in the reference: it has no GPU path.  This is
 * project_particle_fields (src/pfem2particlehandler.cpp:174-215) as one
 * stateless call, for callers that may not allocate device memory at the
 * point where they need the projection: a solver whose device memory is all
 * reserved by its own pool or caching allocator, a time loop that must not
 * hit cudaMalloc/cudaFree (cudaFree synchronises the whole device), or code
 * that cannot keep a pfem2gpu handle.  It needs no handle and takes mesh
 * and particles from caller-owned device arrays.
 *
 * The work memory is one static device array of
 * PFEM2GPU_NOALLOC_SCRATCH_BYTES (64 MiB) per device, part of this library's
 * image.  With CUDA's lazy module loading (the default since CUDA 12.2) it is
 * reserved on a device when the call first runs there; with
 * CUDA_MODULE_LOADING=EAGER every context that loads the library reserves it
 * at once.  It stays reserved until the process exits.  The call needs
 *   256 + 4*n_dofs + 4*(n_dofs+1) + 4*ceil(n_dofs/2048)
 *       + 4*n_cells*2^dim + 32*n_cells*2^dim          bytes
 * (each term rounded up to 256), about 290 B per cell in 3D and 115 B per
 * cell in 2D: up to roughly 230,000 hexes or 580,000 quads.  A larger mesh
 * is refused with PFEM2GPU_ERR_SCRATCH before any device work.
 *
 * Inputs, all on the current device: cell_dofs n_cells x 2^dim (deal.II
 * lexicographic vertex order); the particles' cells (ascending: each cell's
 * particles contiguous, as the particle handler stores them), reference
 * coordinates xi and velocities v, both component-major (xi[d*n + p]).
 * Output V_out: dim x n_dofs component-major; DoFs that no particle reaches
 * get NaN (empty_dof_policy 0, the reference's 0/0) or keep their value on
 * entry (policy 1).  Nothing else needs any value on entry: the call zeroes
 * the counters it uses itself.  *n_empty_dofs (if not NULL) gets the count of
 * such DoFs.  Unsorted or out-of-range cells or DoFs: PFEM2GPU_ERR_ARG,
 * with V_out left as it was on entry.
 *
 * The call runs on `stream` (a cudaStream_t; NULL = the default stream) and
 * returns after its work there has finished.  Calls on one device share the
 * one scratch array, so two calls in flight at once would race on it; the
 * library prevents that with a per-device lock held until the call's work
 * has finished, so concurrent callers wait for each other.  A stream that is
 * being captured into a CUDA graph is refused (PFEM2GPU_ERR_STATE).  Every
 * call looks up the scratch array's address (cudaGetSymbolAddress) with its
 * device current, so it follows the context that is current.
 * The sums are those of the FP64 form: V_out equals pfem2gpu_project of an
 * FP64 handle that holds the same particles in the same order, bit for bit.
 */
#define PFEM2GPU_NOALLOC_SCRATCH_BYTES (64ull << 20)
int pfem2gpu_project_noalloc(int dim, int32_t n_cells, int32_t n_dofs, const int32_t* d_cell_dofs,
                             int64_t n_particles, const int32_t* d_cell, const double* d_xi, const double* d_v,
                             int empty_dof_policy, double* d_V_out, int64_t* n_empty_dofs, void* stream);

const char* pfem2gpu_error_string(int code);
int pfem2gpu_last_error(pfem2gpu_handle* h, char* buf, int64_t len);

#ifdef __cplusplus
}
#endif
#endif
