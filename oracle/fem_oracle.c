/* FP64 CPU restatement of the Q1 FEM systems' volume terms -- TEST
 * INFRASTRUCTURE ONLY: the checker of the library's device assembly, never
 * called by the product.
 *
 * Follows src/pfem2fem.cpp: assemble_velocity_prediction (:247-319, the
 * volume integral; SCHEMEB off), assemble_pressure_equation (:393-435) and
 * assemble_velocity_correction (:461-510), as a sequential cell loop that
 * adds each cell's local matrix and right-hand side into the global ones
 * (distribute_local_to_global without constraints).  Boundary-face terms and
 * the constraints stay with the caller.  FE values are the Q1 /
 * QGauss(2) / MappingQ1 quantities of deal.II (not vendored here, so parity
 * with it is unpinned): quadrature points (1 -+ 1/sqrt 3)/2 per direction, x
 * fastest, weight 1/2 per direction; J[d][e] = sum_i X_i[d] dN_i/dxi_e; the
 * physical gradient J^-T grad N; JxW = det J * weight.
 *
 * Pattern: for every DoF, the DoFs sharing a cell with it, ascending
 * (DoFTools::make_sparsity_pattern for Q1).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fem_oracle.h"

static const double QP[2] = {0.21132486540518711775, 0.78867513459481288225};

static void fe_point(int dim, const double* X, int q, double* N, double* g, double* jxw)
{
    const int nv = 1 << dim;
    double xi[3], gr[8][3], J[3][3], Ji[3][3], det;
    for (int d = 0; d < dim; ++d) xi[d] = QP[(q >> d) & 1];
    for (int i = 0; i < nv; ++i) {
        double n = 1.0;
        for (int d = 0; d < dim; ++d) n = n * (((i >> d) & 1) ? xi[d] : 1.0 - xi[d]);
        N[i] = n;
        for (int e = 0; e < dim; ++e) {
            double t = ((i >> e) & 1) ? 1.0 : -1.0;
            for (int d = 0; d < dim; ++d)
                if (d != e) t = t * (((i >> d) & 1) ? xi[d] : 1.0 - xi[d]);
            gr[i][e] = t;
        }
    }
    for (int d = 0; d < dim; ++d)
        for (int e = 0; e < dim; ++e) {
            double s = 0.0;
            for (int i = 0; i < nv; ++i) s = s + X[i * dim + d] * gr[i][e];
            J[d][e] = s;
        }
    if (dim == 2) {
        det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        Ji[0][0] = J[1][1] / det;
        Ji[0][1] = -J[0][1] / det;
        Ji[1][0] = -J[1][0] / det;
        Ji[1][1] = J[0][0] / det;
    } else {
        const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
        Ji[0][0] = c00 / det;
        Ji[1][0] = c01 / det;
        Ji[2][0] = c02 / det;
        Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
        Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
        Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
        Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
        Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
        Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    }
    for (int i = 0; i < nv; ++i)
        for (int d = 0; d < dim; ++d) {
            double s = 0.0;
            for (int e = 0; e < dim; ++e) s = s + Ji[e][d] * gr[i][e];
            g[i * 3 + d] = s;
        }
    *jxw = det * (dim == 2 ? 0.25 : 0.125);
}

/* Face f (xi_{f/2} = f%2), face point qf: the other directions ascending,
 * the first fastest, weight 1/2 each; outward normal J^-T nhat normalised,
 * surface element det J |J^-T nhat| w (deal.II FEFaceValues, MappingQ1). */
static void fe_face_point(int dim, const double* X, int f, int qf, double* N, double* g, double* n, double* jxw)
{
    const int nv = 1 << dim, fd = f >> 1, side = f & 1;
    double xi[3], gr[8][3], J[3][3], Ji[3][3], det;
    int k = 0;
    for (int d = 0; d < dim; ++d) {
        if (d == fd) xi[d] = side ? 1.0 : 0.0;
        else xi[d] = QP[(qf >> k++) & 1];
    }
    for (int i = 0; i < nv; ++i) {
        double nn = 1.0;
        for (int d = 0; d < dim; ++d) nn = nn * (((i >> d) & 1) ? xi[d] : 1.0 - xi[d]);
        N[i] = nn;
        for (int e = 0; e < dim; ++e) {
            double t = ((i >> e) & 1) ? 1.0 : -1.0;
            for (int d = 0; d < dim; ++d)
                if (d != e) t = t * (((i >> d) & 1) ? xi[d] : 1.0 - xi[d]);
            gr[i][e] = t;
        }
    }
    for (int d = 0; d < dim; ++d)
        for (int e = 0; e < dim; ++e) {
            double sum = 0.0;
            for (int i = 0; i < nv; ++i) sum = sum + X[i * dim + d] * gr[i][e];
            J[d][e] = sum;
        }
    if (dim == 2) {
        det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        Ji[0][0] = J[1][1] / det;
        Ji[0][1] = -J[0][1] / det;
        Ji[1][0] = -J[1][0] / det;
        Ji[1][1] = J[0][0] / det;
    } else {
        const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
        Ji[0][0] = c00 / det;
        Ji[1][0] = c01 / det;
        Ji[2][0] = c02 / det;
        Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
        Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
        Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
        Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
        Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
        Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    }
    for (int i = 0; i < nv; ++i)
        for (int d = 0; d < dim; ++d) {
            double sum = 0.0;
            for (int e = 0; e < dim; ++e) sum = sum + Ji[e][d] * gr[i][e];
            g[i * 3 + d] = sum;
        }
    double v[3], nrm = 0.0;
    for (int a = 0; a < dim; ++a) {
        v[a] = side ? Ji[fd][a] : -Ji[fd][a];
        nrm = nrm + v[a] * v[a];
    }
    nrm = sqrt(nrm);
    for (int a = 0; a < dim; ++a) n[a] = v[a] / nrm;
    *jxw = det * nrm * (dim == 2 ? 0.5 : 0.25);
}

static int cmp_int(const void* a, const void* b)
{
    const int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

int64_t orc_fem_pattern(int dim, int64_t n_cells, int64_t n_dofs, const int32_t* cell_dofs, int32_t* row_ptr,
                        int32_t* cols)
{
    const int nv = 1 << dim;
    /* candidate (row, col) pairs grouped by row, then sorted and made unique */
    int64_t* cnt = calloc((size_t)n_dofs + 1, sizeof(int64_t));
    for (int64_t c = 0; c < n_cells; ++c)
        for (int i = 0; i < nv; ++i) cnt[cell_dofs[c * nv + i] + 1] += nv;
    for (int64_t d = 0; d < n_dofs; ++d) cnt[d + 1] += cnt[d];
    int* cand = malloc((size_t)cnt[n_dofs] * sizeof(int) + 1);
    int64_t* fill = malloc((size_t)n_dofs * sizeof(int64_t) + 1);
    for (int64_t d = 0; d < n_dofs; ++d) fill[d] = cnt[d];
    for (int64_t c = 0; c < n_cells; ++c)
        for (int i = 0; i < nv; ++i)
            for (int j = 0; j < nv; ++j) cand[fill[cell_dofs[c * nv + i]]++] = cell_dofs[c * nv + j];
    int64_t nnz = 0;
    for (int64_t d = 0; d < n_dofs; ++d) {
        int* p = cand + cnt[d];
        const int64_t m = cnt[d + 1] - cnt[d];
        qsort(p, (size_t)m, sizeof(int), cmp_int);
        if (row_ptr) row_ptr[d] = (int32_t)nnz;
        for (int64_t k = 0; k < m; ++k)
            if (k == 0 || p[k] != p[k - 1]) {
                if (cols) cols[nnz] = p[k];
                ++nnz;
            }
    }
    if (row_ptr) row_ptr[n_dofs] = (int32_t)nnz;
    free(cand);
    free(fill);
    free(cnt);
    return nnz;
}

static int64_t find_col(const int32_t* row_ptr, const int32_t* cols, int row, int col)
{
    int64_t lo = row_ptr[row], hi = row_ptr[row + 1] - 1;
    while (lo <= hi) {
        const int64_t mid = (lo + hi) / 2;
        if (cols[mid] == col) return mid;
        if (cols[mid] < col) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

int orc_fem_assemble(int dim, int system, int64_t n_cells, int64_t n_dofs, const double* cellX,
                     const int32_t* cell_dofs, const int32_t* row_ptr, const int32_t* cols, double rho, double mu,
                     double dt, const double* U, const double* U2, const double* P, const uint16_t* fmask, double* A,
                     double* rhs)
{
    const int nv = 1 << dim, nq = 1 << dim;
    const int nm = system == ORC_FEM_PREDICTION ? dim : 1;
    const int ns = system == ORC_FEM_PRESSURE ? 1 : dim;
    const int64_t nnz = row_ptr[n_dofs];
    memset(A, 0, (size_t)nm * (size_t)nnz * sizeof(double));
    memset(rhs, 0, (size_t)ns * (size_t)n_dofs * sizeof(double));
    double M[3][8][8], r[3][8], N[8], g[8 * 3], w;
    for (int64_t c = 0; c < n_cells; ++c) {
        const double* X = cellX + c * nv * dim;
        const int32_t* dof = cell_dofs + c * nv;
        memset(M, 0, sizeof M);
        memset(r, 0, sizeof r);
        for (int q = 0; q < nq; ++q) {
            fe_point(dim, X, q, N, g, &w);
            for (int i = 0; i < nv; ++i) {
                const double Ni = N[i];
                const double* gi = g + i * 3;
                if (system == ORC_FEM_PREDICTION) {
                    for (int j = 0; j < nv; ++j) {
                        const double* gj = g + j * 3;
                        double aux = rho * Ni * N[j] * w;
                        for (int k = 0; k < dim; ++k) {
                            M[k][i][j] = M[k][i][j] + aux;
                            r[k][i] = r[k][i] + aux * U2[k * n_dofs + dof[j]];
                        }
                        aux = mu * dt * w;
                        if (dim == 2) {
                            M[0][i][j] = M[0][i][j] + aux * (gi[1] * gj[1] + 4.0 / 3.0 * gi[0] * gj[0]);
                            M[1][i][j] = M[1][i][j] + aux * (gi[0] * gj[0] + 4.0 / 3.0 * gi[1] * gj[1]);
                            r[0][i] = r[0][i] - aux * (gi[1] * gj[0] - 2.0 / 3.0 * gi[0] * gj[1]) * U[1 * n_dofs + dof[j]];
                            r[1][i] = r[1][i] - aux * (gi[0] * gj[1] - 2.0 / 3.0 * gi[1] * gj[0]) * U[0 * n_dofs + dof[j]];
                        } else {
                            const double u0 = U[dof[j]], u1 = U[n_dofs + dof[j]], u2 = U[2 * n_dofs + dof[j]];
                            M[0][i][j] = M[0][i][j] + aux * (4.0 / 3.0 * gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2]);
                            M[1][i][j] = M[1][i][j] + aux * (gj[0] * gi[0] + 4.0 / 3.0 * gi[1] * gj[1] + gi[2] * gj[2]);
                            M[2][i][j] = M[2][i][j] + aux * (gj[0] * gi[0] + gj[1] * gi[1] + 4.0 / 3.0 * gi[2] * gj[2]);
                            r[0][i] = r[0][i] - aux * ((gi[1] * gj[0] - 2.0 / 3.0 * gi[0] * gj[1]) * u1 +
                                                       (gi[2] * gj[0] - 2.0 / 3.0 * gi[0] * gj[2]) * u2);
                            r[1][i] = r[1][i] - aux * ((gi[0] * gj[1] - 2.0 / 3.0 * gi[1] * gj[0]) * u0 +
                                                       (gi[2] * gj[1] - 2.0 / 3.0 * gi[1] * gj[2]) * u2);
                            r[2][i] = r[2][i] - aux * ((gi[0] * gj[2] - 2.0 / 3.0 * gi[2] * gj[0]) * u0 +
                                                       (gi[1] * gj[2] - 2.0 / 3.0 * gi[2] * gj[1]) * u1);
                        }
                    }
                } else if (system == ORC_FEM_PRESSURE) {
                    const double coeff = rho / dt;
                    for (int j = 0; j < nv; ++j) {
                        const double* gj = g + j * 3;
                        double dot = gi[0] * gj[0];
                        for (int d = 1; d < dim; ++d) dot = dot + gi[d] * gj[d];
                        M[0][i][j] = M[0][i][j] + dot * w;
                        double aux = 0.0;
                        for (int k = 0; k < dim; ++k) aux = aux + U[k * n_dofs + dof[j]] * gi[k];
                        r[0][i] = r[0][i] + coeff * aux * N[j] * w;
                    }
                } else {
                    const double aux2 = dt * Ni * w;
                    for (int j = 0; j < nv; ++j) {
                        const double* gj = g + j * 3;
                        const double aux = rho * Ni * N[j] * w;
                        const double p = P[dof[j]];
                        for (int k = 0; k < dim; ++k) {
                            if (k == 0) M[0][i][j] = M[0][i][j] + aux;
                            r[k][i] = r[k][i] + aux * U[k * n_dofs + dof[j]];
                            r[k][i] = r[k][i] - aux2 * gj[k] * p;
                        }
                    }
                }
            }
        }
        /* boundary faces outside the Dirichlet set: :320-383 (prediction), :436-449 (pressure) */
        const unsigned faces = !fmask ? 0u
                               : system == ORC_FEM_PREDICTION ? (fmask[c] & 0xffu)
                               : system == ORC_FEM_PRESSURE   ? ((unsigned)fmask[c] >> 8)
                                                              : 0u;
        for (int f = 0; f < 2 * dim; ++f) {
            if (!((faces >> f) & 1u)) continue;
            for (int qf = 0; qf < (1 << (dim - 1)); ++qf) {
                double nrm[3];
                fe_face_point(dim, X, f, qf, N, g, nrm, &w);
                if (system == ORC_FEM_PREDICTION && dim == 2) {
                    for (int i = 0; i < nv; ++i)
                        for (int j = 0; j < nv; ++j) {
                            const double* gj = g + j * 3;
                            const double u0 = U[dof[j]], u1 = U[n_dofs + dof[j]];
                            M[0][i][j] = M[0][i][j] - mu * dt * N[i] * 4.0 / 3.0 * gj[0] * nrm[0] * w;
                            r[0][i] = r[0][i] + mu * dt * N[i] * (-2.0 / 3.0) * gj[1] * u1 * nrm[0] * w;
                            M[1][i][j] = M[1][i][j] - mu * dt * N[i] * gj[0] * nrm[0] * w;
                            r[1][i] = r[1][i] + mu * dt * N[i] * gj[1] * u0 * nrm[0] * w;
                        }
                } else if (system == ORC_FEM_PREDICTION) {
                    double tX[3] = {0, 0, 0}, tY[3] = {0, 0, 0}, tZ[3] = {0, 0, 0};
                    for (int ii = 0; ii < nv; ++ii) {
                        const double* gg = g + ii * 3;
                        const double v0 = 0.0, v1 = U[n_dofs + dof[ii]], v2 = U[2 * n_dofs + dof[ii]];
                        tX[0] = tX[0] + ((4.0 / 3.0) * gg[0] * v0 - (2.0 / 3.0) * gg[1] * v1 - (2.0 / 3.0) * gg[2] * v2);
                        tX[1] = tX[1] + (gg[1] * v0 + gg[0] * v1);
                        tX[2] = tX[2] + (gg[2] * v0 + gg[0] * v2);
                        tY[0] = tY[0] + (gg[1] * v0 + gg[0] * v1);
                        tY[1] = tY[1] + ((-2.0 / 3.0) * gg[0] * v0 + (4.0 / 3.0) * gg[1] * v1 - (2.0 / 3.0) * gg[2] * v2);
                        tY[2] = tY[2] + (gg[2] * v1 + gg[1] * v2);
                        tZ[0] = tZ[0] + (gg[2] * v0 + gg[0] * v2);
                        tZ[1] = tZ[1] + (gg[2] * v1 + gg[1] * v2);
                        tZ[2] = tZ[2] + ((-2.0 / 3.0) * gg[0] * v0 - (2.0 / 3.0) * gg[1] * v1 + (4.0 / 3.0) * gg[2] * v2);
                    }
                    const double* T[3] = {tX, tY, tZ};
                    for (int i = 0; i < nv; ++i) {
                        const double aux = mu * dt * N[i] * w;
                        for (int k = 0; k < 3; ++k) {
                            double dot = (aux * T[k][0]) * nrm[0];
                            for (int d = 1; d < 3; ++d) dot = dot + (aux * T[k][d]) * nrm[d];
                            r[k][i] = r[k][i] + dot;
                        }
                    }
                } else {
                    const double coeff = rho / dt;
                    double Vq[3] = {0, 0, 0};
                    for (int ii = 0; ii < nv; ++ii)
                        for (int k = 0; k < dim; ++k) Vq[k] = Vq[k] + N[ii] * U[k * n_dofs + dof[ii]];
                    for (int i = 0; i < nv; ++i) {
                        double dot = (coeff * N[i] * Vq[0]) * nrm[0];
                        for (int d = 1; d < dim; ++d) dot = dot + (coeff * N[i] * Vq[d]) * nrm[d];
                        r[0][i] = r[0][i] - dot * w;
                    }
                }
            }
        }
        for (int i = 0; i < nv; ++i) {
            for (int j = 0; j < nv; ++j) {
                const int64_t pos = find_col(row_ptr, cols, dof[i], dof[j]);
                if (pos < 0) return 1;
                for (int m = 0; m < nm; ++m) A[m * nnz + pos] = A[m * nnz + pos] + M[m][i][j];
            }
            for (int k = 0; k < ns; ++k) rhs[k * n_dofs + dof[i]] = rhs[k * n_dofs + dof[i]] + r[k][i];
        }
    }
    return 0;
}

/* velocity_prediction_bc (src/pfem2fem.cpp:150-245) and
 * fill_velocity_boundary_dofs_list (:128-148): per cell (ascending) and
 * boundary face in the velocity Dirichlet set (ascending), at each face
 * point, the pressure gradient sum_j grad N_j p_j times N_i and N_i added to
 * vertex i; summed into the DoFs in cell order; on DoFs of such faces
 * value_d = grad_d * (dt / rho) / weight + the velocity of the last such
 * face's id.  flags[r] = 1 on those DoFs. */
void orc_fem_velocity_bc(int dim, int64_t n_cells, int64_t n_dofs, const double* cellX, const int32_t* cell_dofs,
                         const int32_t* face_ids, int n_vd, const int32_t* vd, int n_ids, const int32_t* ids,
                         const double* velocities, double rho, double dt, const double* P, int32_t* flags,
                         double* values)
{
    const int nv = 1 << dim, nf = 2 * dim;
    double* pg = calloc((size_t)n_dofs * (dim + 1), sizeof(double));
    int32_t* last = malloc((size_t)n_dofs * sizeof(int32_t));
    for (int64_t r = 0; r < n_dofs; ++r) last[r] = -1;
    double N[8], g[8 * 3], nrm[3], w;
    for (int64_t c = 0; c < n_cells; ++c) {
        const double* X = cellX + c * nv * dim;
        const int32_t* dof = cell_dofs + c * nv;
        double loc[8][4];
        int lid[8];
        memset(loc, 0, sizeof loc);
        for (int i = 0; i < nv; ++i) lid[i] = -1;
        for (int f = 0; f < nf; ++f) {
            const int32_t id = face_ids[c * nf + f];
            if (id < 0) continue;
            int isd = 0;
            for (int k = 0; k < n_vd; ++k) isd |= vd[k] == id;
            if (!isd) continue;
            for (int i = 0; i < nv; ++i)
                if (((i >> (f >> 1)) & 1) == (f & 1)) lid[i] = id;
            for (int qf = 0; qf < (1 << (dim - 1)); ++qf) {
                fe_face_point(dim, X, f, qf, N, g, nrm, &w);
                double gp[3] = {0, 0, 0};
                for (int j = 0; j < nv; ++j)
                    for (int d = 0; d < dim; ++d) gp[d] = gp[d] + g[j * 3 + d] * P[dof[j]];
                for (int i = 0; i < nv; ++i) {
                    for (int d = 0; d < dim; ++d) loc[i][d] = loc[i][d] + N[i] * gp[d];
                    loc[i][dim] = loc[i][dim] + N[i];
                }
            }
        }
        for (int i = 0; i < nv; ++i) {
            for (int q = 0; q <= dim; ++q) pg[dof[i] * (dim + 1) + q] = pg[dof[i] * (dim + 1) + q] + loc[i][q];
            if (lid[i] >= 0) last[dof[i]] = lid[i];
        }
    }
    const double coeff = dt / rho;
    for (int64_t r = 0; r < n_dofs; ++r) {
        flags[r] = last[r] >= 0;
        int slot = -1;
        for (int k = 0; k < n_ids; ++k)
            if (ids[k] == last[r]) slot = k;
        for (int d = 0; d < dim; ++d)
            values[d * n_dofs + r] = last[r] >= 0 ? pg[r * (dim + 1) + d] * coeff / pg[r * (dim + 1) + dim] +
                                                         (slot >= 0 ? velocities[slot * dim + d] : 0.0)
                                                   : 0.0;
    }
    free(pg);
    free(last);
}
