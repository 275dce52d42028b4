/*
 * pfem2_oracle.h -- FP64 CPU restatement of the PFEM-2 particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product (libpfem2gpu) and the timed CPU baseline of bench.py.  Nothing in
 * the product links it or falls back to it.
 *
 * PARITY UNPINNED: the reference (andreyypopov/pfem2dealii) has no tests and
 * no golden vectors, and it cannot be compiled in this environment (it needs
 * deal.II >= 9.4 with p4est, Trilinos and MPI).  The arithmetic the reference
 * delegates to deal.II (FE_Q<dim>(1)::shape_value, MappingQ1 forward and
 * inverse maps, GeometryInfo::is_inside_unit_cell, GridTools vertex maps) is
 * restated here from the published algorithms; analytic known-answer tests in
 * tests/ pin what mathematics can pin.
 *
 * Every function cites the reference file:line it follows (paths relative to
 * the reference project root).
 */
#ifndef PFEM2_ORACLE_H
#define PFEM2_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Removal order inside an over-full cell part (check_particle_distribution). */
enum {
    ORC_ORDER_ID = 0,     /* examine particles by ascending key(id): deterministic, GPU-comparable */
    ORC_ORDER_VECTOR = 1  /* the reference's swap-with-back std::vector order */
};

typedef struct orc_params {
    int32_t q[3];                 /* particles per cell per direction (prm "Number of particles in the x/y/z direction") */
    int32_t max_per_part;         /* prm "Maximum number of particles per cell part" */
    int32_t substeps;             /* prm "Particle integration steps" (0 -> 1) */
    double dt;                    /* prm "Time step" (full FEM step) */
    int32_t removal_order;        /* ORC_ORDER_* */
    uint32_t removal_seed;        /* key(id) = seed ? mix32(id ^ seed) : id */
    int32_t n_threads;            /* >1: parallel particle loops (baseline timing) */
    int32_t integrator;           /* ORC_EULER (the reference) or ORC_RK2 (opt-in, see orc_move) */
} orc_params;

enum {
    ORC_EULER = 0, /* x += h u(xi): move_particles, src/pfem2particlehandler.cpp:151-163 */
    ORC_RK2 = 1    /* midpoint rule in the particle's own cell; no reference counterpart */
};

typedef struct orc_stats {
    int64_t n_particles;
    int64_t lost;           /* deleted by relocation (no cell found) */
    int64_t removed;        /* deleted by count correction */
    int64_t seeded;         /* inserted by count correction */
    int64_t map_failures;   /* inverse-map failures (ExcTransformationFailed equivalents) */
    int64_t near_face;      /* particles with xi_d within 1e-12 of 0 or 1 after relocation */
    int64_t searched;       /* particles that left their cell and went through the vertex-patch search */
    int64_t nan_dofs;       /* DoFs with zero projection weight (0/0 in project) */
    uint32_t next_id;       /* last id handed out (particleCount) */
} orc_stats;

typedef struct orc_handle orc_handle;

orc_handle* orc_create(int dim, const orc_params* prm);
void orc_destroy(orc_handle* h);

/* Mesh: vertex coordinates (n_verts x dim), cell vertices and cell DoFs
 * (n_cells x 2^dim, deal.II lexicographic vertex order). */
int orc_set_mesh(orc_handle* h, int64_t n_cells, int64_t n_verts, int64_t n_dofs,
                 const double* vertices, const int32_t* cell_vertices,
                 const int32_t* cell_dofs);

/* Vertex -> cell map (CSR, cells ascending) and unit vertex->cell-centre
 * directions built by orc_set_mesh; offsets has n_verts+1 entries. */
int64_t orc_vertex_map_size(const orc_handle* h);
void orc_get_vertex_maps(const orc_handle* h, int32_t* offsets, int32_t* cells, double* dirs);

/* V arrays are component-major: V[d * n_dofs + dof] (one Trilinos vector per component). */
int orc_seed(orc_handle* h, const double* V);
int orc_correct(orc_handle* h, const double* V, const double* Vold);
int orc_move(orc_handle* h, const double* V);
int orc_project(orc_handle* h, double* V_out);

/* Particle state, in the oracle's current vector order. */
int64_t orc_n_particles(const orc_handle* h);
void orc_get_particles(const orc_handle* h, uint32_t* id, int32_t* cell, double* x,
                       double* xi, double* v);
int orc_set_particles(orc_handle* h, int64_t n, const uint32_t* id, const int32_t* cell,
                      const double* x, const double* xi, const double* v, uint32_t next_id);
void orc_get_stats(const orc_handle* h, orc_stats* s);
void orc_reset_stats(orc_handle* h);

/* Differentiated window (no counterpart in the reference, which has no
 * adjoint): K steps of correct (if Vold != NULL) + sub-steps with relocation
 * from the current particles, count correction left out, then the projection
 * U (dim x n_dofs; empty_policy 0: NaN where no particle weighs, 1: V there).
 * The particle set is unchanged.  v0: n x dim starting velocities or NULL.
 * The adjoint holds every particle's cell sequence fixed and returns, for
 * dJ/dU = gU, the gradients with respect to the starting particle velocities
 * (g_v0, n x dim), V and Vold (dim x n_dofs).  Outputs may be NULL. */
int orc_window_forward(orc_handle* h, int K, const double* V, const double* Vold, const double* v0,
                       int empty_policy, double* U);
int orc_window_particles(orc_handle* h, int K, const double* V, const double* Vold, const double* v0, int32_t* cell,
                         double* x, double* xi, double* v);
int orc_window_adjoint(orc_handle* h, int K, const double* V, const double* Vold, const double* v0,
                       int empty_policy, const double* gU, double* U, double* g_v0, double* g_V, double* g_Vold);

/* Geometry primitives, exposed for known-answer tests. */
void orc_shape_values(int dim, const double* xi, double* N);
void orc_forward_map(int dim, const double* X, const double* xi, double* x);
int orc_inverse_map(int dim, const double* X, const double* p, double* xi);
uint32_t orc_key(uint32_t id, uint32_t seed);

#ifdef __cplusplus
}
#endif
#endif
