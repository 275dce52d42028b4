/* FP64 CPU restatement of the Q1 FEM systems' volume terms
 * (src/pfem2fem.cpp:247-510) -- test infrastructure only. */
#ifndef FEM_ORACLE_H
#define FEM_ORACLE_H
#include <stdint.h>

#define ORC_FEM_PREDICTION 0 /* U = solution V, U2 = old solution V: dim matrices, dim right-hand sides */
#define ORC_FEM_PRESSURE 1   /* U = predicted V: one matrix, one right-hand side */
#define ORC_FEM_CORRECTION 2 /* U = predicted V, P = pressure: one matrix, dim right-hand sides */

#ifdef __cplusplus
extern "C" {
#endif
/* CSR pattern of the Q1 DoF adjacency, columns ascending; returns nnz (row_ptr/cols may be NULL). */
int64_t orc_fem_pattern(int dim, int64_t n_cells, int64_t n_dofs, const int32_t* cell_dofs, int32_t* row_ptr,
                        int32_t* cols);
/* A: (matrices x nnz), rhs: (right-hand sides x n_dofs); cellX: n_cells x 2^dim x dim. */
/* fmask (may be NULL): per cell, bit f = boundary face f with prediction
 * face terms, bit 8 + f = with pressure face terms. */
int orc_fem_assemble(int dim, int system, int64_t n_cells, int64_t n_dofs, const double* cellX,
                     const int32_t* cell_dofs, const int32_t* row_ptr, const int32_t* cols, double rho, double mu,
                     double dt, const double* U, const double* U2, const double* P, const uint16_t* fmask, double* A,
                     double* rhs);
/* velocity_prediction_bc: flags (n_dofs) and values (dim x n_dofs) of the prediction's Dirichlet rows. */
void orc_fem_velocity_bc(int dim, int64_t n_cells, int64_t n_dofs, const double* cellX, const int32_t* cell_dofs,
                         const int32_t* face_ids, int n_vd, const int32_t* vd, int n_ids, const int32_t* ids,
                         const double* velocities, double rho, double dt, const double* P, int32_t* flags,
                         double* values);
#ifdef __cplusplus
}
#endif
#endif
