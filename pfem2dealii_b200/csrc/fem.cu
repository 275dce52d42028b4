// Q1 FEM systems of the solver step on the device (src/pfem2fem.cpp:247-509):
// the volume integrals of the velocity prediction, the pressure equation and
// the velocity correction, summed into CSR matrices and right-hand sides.
// Compiled with --fmad=false: every product and sum is rounded separately.
//
// Element values, per cell and quadrature point (QGauss(2), x fastest,
// weights 1/2 per direction): J[d][e] = sum_i X_i[d] dN_i/dxi_e (i
// ascending), its inverse by cofactors, physical gradients
// g_i[d] = sum_e Jinv[e][d] dN_i/dxi_e, JxW = det J * w.  The local matrix
// and right-hand side terms are added in the reference's order (q outer, i,
// then j; within one (q, i, j) the terms in the order of the source lines),
// and a global entry is the sum of its cells' local values in ascending cell
// order, as a sequential cell loop adds them.
#include <cstdint>

#include "common.cuh"
#include "launch.h"

namespace pfem2 {
namespace {

constexpr double QG0 = 0.21132486540518711775, QG1 = 0.78867513459481288225;  // (1 -+ 1/sqrt 3) / 2

template <int DIM>
struct Quad {
    double N[1 << DIM];           // shape values
    double g[1 << DIM][DIM];      // physical gradients
    double jxw;
};

// Shape values, reference gradients, then the physical quantities at q.
template <int DIM>
__device__ void quad_point(const double* __restrict__ X, int q, Quad<DIM>& out)
{
    constexpr int NV = 1 << DIM;
    double xi[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi[d] = ((q >> d) & 1) ? QG1 : QG0;
    double gr[NV][DIM];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double n = 1.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) n = n * (((i >> d) & 1) ? xi[d] : 1.0 - xi[d]);
        out.N[i] = n;
#pragma unroll
        for (int e = 0; e < DIM; ++e) {
            double t = ((i >> e) & 1) ? 1.0 : -1.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d)
                if (d != e) t = t * (((i >> d) & 1) ? xi[d] : 1.0 - xi[d]);
            gr[i][e] = t;
        }
    }
    double J[DIM][DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
        for (int e = 0; e < DIM; ++e) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < NV; ++i) s = s + X[i * DIM + d] * gr[i][e];
            J[d][e] = s;
        }
    double det, Ji[DIM][DIM];
    if constexpr (DIM == 2) {
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
#pragma unroll
    for (int i = 0; i < NV; ++i)
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            double s = 0.0;
#pragma unroll
            for (int e = 0; e < DIM; ++e) s = s + Ji[e][d] * gr[i][e];
            out.g[i][d] = s;
        }
    out.jxw = det * (DIM == 2 ? 0.25 : 0.125);
}

// Face f (deal.II numbering: xi_{f/2} = f%2), face point qf of QGauss(2) in
// the face's other directions (ascending, the first fastest; weight 1/2
// each): shape values and gradients as in the cell, the outward unit normal
// n = J^-T nhat / |J^-T nhat| and the surface element det J |J^-T nhat| w.
template <int DIM>
struct FaceQuad {
    double N[1 << DIM];
    double g[1 << DIM][DIM];
    double n[DIM];
    double jxw;
};

template <int DIM>
__device__ void face_point(const double* __restrict__ X, int f, int qf, FaceQuad<DIM>& out)
{
    constexpr int NV = 1 << DIM;
    const int fd = f >> 1, side = f & 1;
    double xi[DIM];
    int k = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        if (d == fd) {
            xi[d] = side ? 1.0 : 0.0;
        } else {
            xi[d] = ((qf >> k) & 1) ? QG1 : QG0;
            ++k;
        }
    }
    double gr[NV][DIM];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double nn = 1.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) nn = nn * (((i >> d) & 1) ? xi[d] : 1.0 - xi[d]);
        out.N[i] = nn;
#pragma unroll
        for (int e = 0; e < DIM; ++e) {
            double t = ((i >> e) & 1) ? 1.0 : -1.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d)
                if (d != e) t = t * (((i >> d) & 1) ? xi[d] : 1.0 - xi[d]);
            gr[i][e] = t;
        }
    }
    double J[DIM][DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
        for (int e = 0; e < DIM; ++e) {
            double sum = 0.0;
#pragma unroll
            for (int i = 0; i < NV; ++i) sum = sum + X[i * DIM + d] * gr[i][e];
            J[d][e] = sum;
        }
    double det, Ji[DIM][DIM];
    if constexpr (DIM == 2) {
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
#pragma unroll
    for (int i = 0; i < NV; ++i)
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            double sum = 0.0;
#pragma unroll
            for (int e = 0; e < DIM; ++e) sum = sum + Ji[e][d] * gr[i][e];
            out.g[i][d] = sum;
        }
    double v[DIM], nrm = 0.0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        v[a] = side ? Ji[fd][a] : -Ji[fd][a];
        nrm = nrm + v[a] * v[a];
    }
    nrm = sqrt(nrm);
#pragma unroll
    for (int a = 0; a < DIM; ++a) out.n[a] = v[a] / nrm;
    out.jxw = det * nrm * (DIM == 2 ? 0.5 : 0.25);
}

// Boundary-face terms of row i (the faces set in the cell's mask for this
// system, ascending; their points in order), after the volume terms:
// assemble_velocity_prediction :320-383, assemble_pressure_equation
// :436-449.  The 3D prediction term takes velocity components 1..dim-1 of
// the cell's DoFs, component 0 as zero, as the reference's loop does.
template <int DIM, int SYS, int NM, int NS>
__device__ void face_terms(const FemArgs& f, long long c, int i, const int* dof, double (*M)[1 << DIM], double* r)
{
    constexpr int NV = 1 << DIM;
    const unsigned mk = f.fmask[c];
    const unsigned faces = SYS == FEM_PREDICTION ? (mk & 0xffu) : (mk >> 8);
    if (!faces) return;
    double X[NV * DIM];
#pragma unroll
    for (int k = 0; k < NV * DIM; ++k) X[k] = f.cellX[(size_t)c * NV * DIM + k];
    for (int fc = 0; fc < 2 * DIM; ++fc) {
        if (!((faces >> fc) & 1u)) continue;
        for (int qf = 0; qf < (1 << (DIM - 1)); ++qf) {
            FaceQuad<DIM> F;
            face_point<DIM>(X, fc, qf, F);
            const double Ni = F.N[i];
            if constexpr (SYS == FEM_PREDICTION) {
                if constexpr (DIM == 2) {
                    for (int j = 0; j < NV; ++j) {
                        const double u0 = f.U[dof[j]], u1 = f.U[(size_t)f.nD + dof[j]];
                        M[0][j] = M[0][j] - f.mu * f.dt * Ni * 4.0 / 3.0 * F.g[j][0] * F.n[0] * F.jxw;
                        r[0] = r[0] + f.mu * f.dt * Ni * (-2.0 / 3.0) * F.g[j][1] * u1 * F.n[0] * F.jxw;
                        M[1][j] = M[1][j] - f.mu * f.dt * Ni * F.g[j][0] * F.n[0] * F.jxw;
                        r[1] = r[1] + f.mu * f.dt * Ni * F.g[j][1] * u0 * F.n[0] * F.jxw;
                    }
                } else {
                    double tX[3] = {0.0, 0.0, 0.0}, tY[3] = {0.0, 0.0, 0.0}, tZ[3] = {0.0, 0.0, 0.0};
                    for (int ii = 0; ii < NV; ++ii) {
                        const double* g = F.g[ii];
                        const double v0 = 0.0, v1 = f.U[(size_t)f.nD + dof[ii]], v2 = f.U[(size_t)2 * f.nD + dof[ii]];
                        tX[0] = tX[0] + ((4.0 / 3.0) * g[0] * v0 - (2.0 / 3.0) * g[1] * v1 - (2.0 / 3.0) * g[2] * v2);
                        tX[1] = tX[1] + (g[1] * v0 + g[0] * v1);
                        tX[2] = tX[2] + (g[2] * v0 + g[0] * v2);
                        tY[0] = tY[0] + (g[1] * v0 + g[0] * v1);
                        tY[1] = tY[1] + ((-2.0 / 3.0) * g[0] * v0 + (4.0 / 3.0) * g[1] * v1 - (2.0 / 3.0) * g[2] * v2);
                        tY[2] = tY[2] + (g[2] * v1 + g[1] * v2);
                        tZ[0] = tZ[0] + (g[2] * v0 + g[0] * v2);
                        tZ[1] = tZ[1] + (g[2] * v1 + g[1] * v2);
                        tZ[2] = tZ[2] + ((-2.0 / 3.0) * g[0] * v0 - (2.0 / 3.0) * g[1] * v1 + (4.0 / 3.0) * g[2] * v2);
                    }
                    const double aux = f.mu * f.dt * Ni * F.jxw;
                    const double* T[3] = {tX, tY, tZ};
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        double dot = (aux * T[k][0]) * F.n[0];
#pragma unroll
                        for (int d = 1; d < 3; ++d) dot = dot + (aux * T[k][d]) * F.n[d];
                        r[k] = r[k] + dot;
                    }
                }
            } else if constexpr (SYS == FEM_PRESSURE) {
                const double coeff = f.rho / f.dt;
                double Vq[DIM];
#pragma unroll
                for (int k = 0; k < DIM; ++k) Vq[k] = 0.0;
                for (int ii = 0; ii < NV; ++ii)
#pragma unroll
                    for (int k = 0; k < DIM; ++k) Vq[k] = Vq[k] + F.N[ii] * f.U[(size_t)k * f.nD + dof[ii]];
                double dot = (coeff * Ni * Vq[0]) * F.n[0];
#pragma unroll
                for (int d = 1; d < DIM; ++d) dot = dot + (coeff * Ni * Vq[d]) * F.n[d];
                r[0] = r[0] - dot * F.jxw;
            }
        }
    }
}

// One lane per (cell, local row i), 32 / 2^dim cells per warp.  The cell's
// 2^dim quadrature points are computed once, lane i taking point i, into
// shared memory; then lane i accumulates row i of the cell's local matrices
// (NM of them, NV entries each) and its right-hand-side entries, reading the
// points in order.
constexpr int FEM_WARPS = 4;

template <int DIM, int SYS>
__global__ void __launch_bounds__(FEM_WARPS * 32) k_fem_local(FemArgs f)
{
    constexpr int NV = 1 << DIM, NQ = 1 << DIM, CPW = 32 / NV;
    constexpr int NS = SYS == FEM_PRESSURE ? 1 : DIM;   // right-hand sides
    constexpr int NM = SYS == FEM_PREDICTION ? DIM : 1;  // matrices
    __shared__ Quad<DIM> qd[FEM_WARPS][CPW][NQ];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int jc = lane / NV, i = lane % NV;
    const long long nwarps = (long long)gridDim.x * FEM_WARPS;
    for (long long gw = (long long)blockIdx.x * FEM_WARPS + warp; gw * CPW < f.nC; gw += nwarps) {
        const long long c = gw * CPW + jc;
        const bool valid = c < f.nC;
        if (valid) {
            double X[NV * DIM];
#pragma unroll
            for (int k = 0; k < NV * DIM; ++k) X[k] = f.cellX[(size_t)c * NV * DIM + k];
            quad_point<DIM>(X, i, qd[warp][jc][i]);
        }
        __syncwarp();
        if (valid) {
            int dof[NV];
#pragma unroll
            for (int j = 0; j < NV; ++j) dof[j] = f.cd[(size_t)c * NV + j];
            double M[NM][NV], r[NS];
#pragma unroll
            for (int m = 0; m < NM; ++m)
#pragma unroll
                for (int j = 0; j < NV; ++j) M[m][j] = 0.0;
#pragma unroll
            for (int k = 0; k < NS; ++k) r[k] = 0.0;
            for (int q = 0; q < NQ; ++q) {
                const Quad<DIM>& Q = qd[warp][jc][q];
                const double w = Q.jxw;
                const double Ni = Q.N[i];
                double gi[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) gi[d] = Q.g[i][d];
                if constexpr (SYS == FEM_PREDICTION) {
#pragma unroll
                    for (int j = 0; j < NV; ++j) {
                        const double* gj = Q.g[j];
                        double aux = f.rho * Ni * Q.N[j] * w;
#pragma unroll
                        for (int k = 0; k < DIM; ++k) {
                            M[k][j] = M[k][j] + aux;
                            r[k] = r[k] + aux * f.U2[(size_t)k * f.nD + dof[j]];
                        }
                        aux = f.mu * f.dt * w;
                        double u[DIM];
#pragma unroll
                        for (int k = 0; k < DIM; ++k) u[k] = f.U[(size_t)k * f.nD + dof[j]];
                        if constexpr (DIM == 2) {
                            M[0][j] = M[0][j] + aux * (gi[1] * gj[1] + 4.0 / 3.0 * gi[0] * gj[0]);
                            M[1][j] = M[1][j] + aux * (gi[0] * gj[0] + 4.0 / 3.0 * gi[1] * gj[1]);
                            r[0] = r[0] - aux * (gi[1] * gj[0] - 2.0 / 3.0 * gi[0] * gj[1]) * u[1];
                            r[1] = r[1] - aux * (gi[0] * gj[1] - 2.0 / 3.0 * gi[1] * gj[0]) * u[0];
                        } else {
                            M[0][j] = M[0][j] + aux * (4.0 / 3.0 * gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2]);
                            M[1][j] = M[1][j] + aux * (gj[0] * gi[0] + 4.0 / 3.0 * gi[1] * gj[1] + gi[2] * gj[2]);
                            M[2][j] = M[2][j] + aux * (gj[0] * gi[0] + gj[1] * gi[1] + 4.0 / 3.0 * gi[2] * gj[2]);
                            r[0] = r[0] - aux * ((gi[1] * gj[0] - 2.0 / 3.0 * gi[0] * gj[1]) * u[1] +
                                                 (gi[2] * gj[0] - 2.0 / 3.0 * gi[0] * gj[2]) * u[2]);
                            r[1] = r[1] - aux * ((gi[0] * gj[1] - 2.0 / 3.0 * gi[1] * gj[0]) * u[0] +
                                                 (gi[2] * gj[1] - 2.0 / 3.0 * gi[1] * gj[2]) * u[2]);
                            r[2] = r[2] - aux * ((gi[0] * gj[2] - 2.0 / 3.0 * gi[2] * gj[0]) * u[0] +
                                                 (gi[1] * gj[2] - 2.0 / 3.0 * gi[2] * gj[1]) * u[1]);
                        }
                    }
                } else if constexpr (SYS == FEM_PRESSURE) {
                    const double coeff = f.rho / f.dt;
#pragma unroll
                    for (int j = 0; j < NV; ++j) {
                        const double* gj = Q.g[j];
                        double dot = gi[0] * gj[0];
#pragma unroll
                        for (int d = 1; d < DIM; ++d) dot = dot + gi[d] * gj[d];
                        M[0][j] = M[0][j] + dot * w;
                        double aux = 0.0;
#pragma unroll
                        for (int k = 0; k < DIM; ++k) aux = aux + f.U[(size_t)k * f.nD + dof[j]] * gi[k];
                        r[0] = r[0] + coeff * aux * Q.N[j] * w;
                    }
                } else {
                    const double aux2 = f.dt * Ni * w;
#pragma unroll
                    for (int j = 0; j < NV; ++j) {
                        const double* gj = Q.g[j];
                        const double aux = f.rho * Ni * Q.N[j] * w;
                        const double p = f.P[dof[j]];
#pragma unroll
                        for (int k = 0; k < DIM; ++k) {
                            if (k == 0) M[0][j] = M[0][j] + aux;  // the same matrix for every component
                            r[k] = r[k] + aux * f.U[(size_t)k * f.nD + dof[j]];
                            r[k] = r[k] - aux2 * gj[k] * p;
                        }
                    }
                }
            }
            const size_t t = (size_t)c * NV + i;
            double* L = f.local + t * NM * NV;
#pragma unroll
            for (int m = 0; m < NM; ++m)
#pragma unroll
                for (int j = 0; j < NV; ++j) L[m * NV + j] = M[m][j];
#pragma unroll
            for (int k = 0; k < NS; ++k) f.local_rhs[t * NS + k] = r[k];
        }
        __syncwarp();
    }
}

// Boundary-face terms, added to the finished volume values of row i of each
// cell with such faces (the same additions, in the same order, as adding
// them to the accumulators after the volume loop).
template <int DIM, int SYS>
__global__ void __launch_bounds__(128) k_fem_faces(FemArgs f)
{
    constexpr int NV = 1 << DIM;
    constexpr int NS = SYS == FEM_PRESSURE ? 1 : DIM;
    constexpr int NM = SYS == FEM_PREDICTION ? DIM : 1;
    const long long total = (long long)f.nC * NV;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long c = t / NV;
        const int i = (int)(t % NV);
        const unsigned mk = f.fmask[c];
        if (!(SYS == FEM_PREDICTION ? (mk & 0xffu) : (mk >> 8))) continue;
        int dof[NV];
#pragma unroll
        for (int j = 0; j < NV; ++j) dof[j] = f.cd[(size_t)c * NV + j];
        double M[NM][NV], r[NS];
        double* L = f.local + (size_t)t * NM * NV;
#pragma unroll
        for (int m = 0; m < NM; ++m)
#pragma unroll
            for (int j = 0; j < NV; ++j) M[m][j] = L[m * NV + j];
#pragma unroll
        for (int k = 0; k < NS; ++k) r[k] = f.local_rhs[(size_t)t * NS + k];
        face_terms<DIM, SYS, NM, NS>(f, c, i, dof, M, r);
#pragma unroll
        for (int m = 0; m < NM; ++m)
#pragma unroll
            for (int j = 0; j < NV; ++j) L[m * NV + j] = M[m][j];
#pragma unroll
        for (int k = 0; k < NS; ++k) f.local_rhs[(size_t)t * NS + k] = r[k];
    }
}

// Contribution lists, built once per mesh: for every matrix entry the local
// values (cell, local row, local column) that add into it, in ascending cell
// order -- the order in which a cell loop adds them.  One warp per row, a
// lane per entry; pass 1 (fill == false) counts, pass 2 writes from con_off.
template <int DIM>
__global__ void __launch_bounds__(256) k_fem_contrib(FemArgs f, bool fill, uint32_t* __restrict__ count)
{
    constexpr int NV = 1 << DIM;
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; row < f.nD; row += nwarps) {
        const int b = f.d2c_off[row], e = f.d2c_off[row + 1];
        const int cb = f.row_ptr[row], ce = f.row_ptr[row + 1];
        for (int c0 = cb; c0 < ce; c0 += 32) {
            const int pos = c0 + lane;
            const int col = pos < ce ? f.cols[pos] : -1;
            int n = 0, base = (fill && pos < ce) ? f.con_off[pos] : 0;
            for (int k = b; k < e; ++k) {
                const int ent = f.d2c_ent[k];  // cell * NV + local row
                const int c = ent / NV;
#pragma unroll
                for (int j = 0; j < NV; ++j)
                    if (f.cd[(size_t)c * NV + j] == col) {
                        if (fill) f.con[base + n] = ent * NV + j;
                        ++n;
                    }
            }
            if (!fill && pos < ce) count[pos] = (uint32_t)n;
        }
    }
}

// Matrix values: one thread per entry, the sum of its local values in list
// order.  Right-hand sides: one thread per DoF, its cells in ascending order.
template <int DIM, int SYS>
__global__ void __launch_bounds__(256) k_fem_gather(FemArgs f)
{
    constexpr int NV = 1 << DIM;
    constexpr int NS = SYS == FEM_PRESSURE ? 1 : DIM;
    constexpr int NM = SYS == FEM_PREDICTION ? DIM : 1;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < f.nnz; e += stride) {
        double acc[NM];
#pragma unroll
        for (int m = 0; m < NM; ++m) acc[m] = 0.0;
        const int kb = f.con_off[e], ke = f.con_off[e + 1];
        for (int k = kb; k < ke; ++k) {
            const int tj = f.con[k];
            const size_t t = (size_t)(tj / NV);
            const int j = tj % NV;
#pragma unroll
            for (int m = 0; m < NM; ++m) acc[m] = acc[m] + f.local[(t * NM + m) * NV + j];
        }
#pragma unroll
        for (int m = 0; m < NM; ++m) f.A[(size_t)m * f.nnz + e] = acc[m];
    }
    for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < f.nD; row += stride) {
        const int b = f.d2c_off[row], e = f.d2c_off[row + 1];
        double s[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) s[k] = 0.0;
        for (int k = b; k < e; ++k) {
            const size_t t = (size_t)f.d2c_ent[k];
#pragma unroll
            for (int q = 0; q < NS; ++q) s[q] = s[q] + f.local_rhs[t * NS + q];
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) f.rhs[(size_t)q * f.nD + row] = s[q];
    }
}

// CSR pattern: the DoFs sharing a cell with each row DoF, ascending.  Pass 1
// (fill == false) counts, pass 2 writes from row_ptr.  A row longer than
// FEM_ROWMAX sets err.
template <int DIM>
__global__ void k_fem_pattern(FemArgs f, bool fill, uint32_t* __restrict__ count, unsigned* __restrict__ err)
{
    constexpr int NV = 1 << DIM;
    for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < f.nD;
         row += (long long)gridDim.x * blockDim.x) {
        int list[FEM_ROWMAX];
        int n = 0;
        bool over = false;
        for (int k = f.d2c_off[row]; k < f.d2c_off[row + 1]; ++k) {
            const int c = f.d2c_ent[k] / NV;
            for (int j = 0; j < NV; ++j) {
                const int d = f.cd[(size_t)c * NV + j];
                int p = n;  // insertion point, keeping the list ascending and unique
                while (p > 0 && list[p - 1] > d) --p;
                if (p > 0 && list[p - 1] == d) continue;
                if (n == FEM_ROWMAX) {
                    over = true;
                    continue;
                }
                for (int s = n; s > p; --s) list[s] = list[s - 1];
                list[p] = d;
                ++n;
            }
        }
        if (over) atomicOr(err, 1u);
        if (!fill) {
            count[row] = (uint32_t)n;
        } else {
            const int b = f.row_ptr[row];
            for (int s = 0; s < n; ++s) f.cols[b + s] = list[s];
        }
    }
}

// Dirichlet rows (the effect of AffineConstraints::distribute_local_to_global
// for constraints without coupling, summed over the cells): one thread per
// row.  A constrained row keeps its diagonal A_rr and nothing else, its
// right-hand side becomes A_rr g_r; in every other row each constrained
// column c, ascending, moves A_rc g_c to the right-hand side and is zeroed.
// con_val[r] = index of r among the constrained rows or -1; g holds ns
// value sets (one per right-hand side) of n_con values; right-hand side q
// uses matrix min(q, nm - 1).
__global__ void __launch_bounds__(256) k_fem_constrain(int nD, long long nnz, int nm, int ns, const int32_t* row_ptr,
                                                       const int32_t* cols, const int32_t* con_idx, int n_con,
                                                       const double* g, double* A, double* rhs)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nD; r += (long long)gridDim.x * blockDim.x) {
        const int b = row_ptr[r], e = row_ptr[r + 1];
        const int ir = con_idx[r];
        if (ir >= 0) {
            for (int q = 0; q < ns; ++q) {
                const int m = q < nm ? q : nm - 1;
                double diag = 0.0;
                for (int k = b; k < e; ++k)
                    if (cols[k] == (int)r) diag = A[(size_t)m * nnz + k];
                rhs[(size_t)q * nD + r] = diag * g[(size_t)q * n_con + ir];
            }
            for (int m = 0; m < nm; ++m)
                for (int k = b; k < e; ++k)
                    if (cols[k] != (int)r) A[(size_t)m * nnz + k] = 0.0;
            continue;
        }
        for (int q = 0; q < ns; ++q) {
            const int m = q < nm ? q : nm - 1;
            double s = rhs[(size_t)q * nD + r];
            for (int k = b; k < e; ++k) {
                const int ic = con_idx[cols[k]];
                if (ic >= 0) s = s - A[(size_t)m * nnz + k] * g[(size_t)q * n_con + ic];
            }
            rhs[(size_t)q * nD + r] = s;
        }
        for (int m = 0; m < nm; ++m)
            for (int k = b; k < e; ++k)
                if (con_idx[cols[k]] >= 0) A[(size_t)m * nnz + k] = 0.0;
    }
}

// velocity_prediction_bc (src/pfem2fem.cpp:150-245), per (cell, vertex i):
// over the cell's velocity-Dirichlet boundary faces (ascending) and their
// points, the pressure gradient at the point, sum_j grad N_j p_j (j
// ascending), times N_i, and N_i itself (the weight); and the boundary id of
// the last such face containing vertex i (-1: none), for the Dirichlet
// velocity the reference's map keeps.
template <int DIM>
__global__ void __launch_bounds__(128) k_fem_bc_local(FemArgs f, const uint8_t* __restrict__ dmask,
                                                      const int32_t* __restrict__ face_id, const double* __restrict__ P,
                                                      double* __restrict__ out, int32_t* __restrict__ last_id)
{
    constexpr int NV = 1 << DIM;
    const long long total = (long long)f.nC * NV;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long c = t / NV;
        const int i = (int)(t % NV);
        const unsigned faces = dmask[c];
        double acc[DIM + 1];
#pragma unroll
        for (int k = 0; k <= DIM; ++k) acc[k] = 0.0;
        int lid = -1;
        if (faces) {
            double X[NV * DIM];
#pragma unroll
            for (int k = 0; k < NV * DIM; ++k) X[k] = f.cellX[(size_t)c * NV * DIM + k];
            double p[NV];
#pragma unroll
            for (int j = 0; j < NV; ++j) p[j] = P[f.cd[(size_t)c * NV + j]];
            for (int fc = 0; fc < 2 * DIM; ++fc) {
                if (!((faces >> fc) & 1u)) continue;
                if ((((i >> (fc >> 1)) & 1) == (fc & 1))) lid = face_id[(size_t)c * 2 * DIM + fc];
                for (int qf = 0; qf < (1 << (DIM - 1)); ++qf) {
                    FaceQuad<DIM> F;
                    face_point<DIM>(X, fc, qf, F);
                    double g[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) g[d] = 0.0;
#pragma unroll
                    for (int j = 0; j < NV; ++j)
#pragma unroll
                        for (int d = 0; d < DIM; ++d) g[d] = g[d] + F.g[j][d] * p[j];
                    const double sv = F.N[i];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) acc[d] = acc[d] + sv * g[d];
                    acc[DIM] = acc[DIM] + sv;
                }
            }
        }
#pragma unroll
        for (int k = 0; k <= DIM; ++k) out[(size_t)t * (DIM + 1) + k] = acc[k];
        last_id[t] = lid;
    }
}

// Per DoF: the cells' values summed in ascending cell order, then, on a DoF
// of a Dirichlet face, value_k = grad_k * (dt / rho) / weight + the Dirichlet
// velocity of the last face's id (flag 1), else flag 0.
template <int DIM>
__global__ void __launch_bounds__(256) k_fem_bc_dof(FemArgs f, const double* __restrict__ in,
                                                    const int32_t* __restrict__ last_id, int n_ids,
                                                    const int32_t* __restrict__ ids, const double* __restrict__ id_vel,
                                                    double coeff, double* __restrict__ value, int32_t* __restrict__ flag)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < f.nD; r += (long long)gridDim.x * blockDim.x) {
        double acc[DIM + 1];
#pragma unroll
        for (int k = 0; k <= DIM; ++k) acc[k] = 0.0;
        int lid = -1;
        for (int k = f.d2c_off[r]; k < f.d2c_off[r + 1]; ++k) {
            const size_t t = (size_t)f.d2c_ent[k];
#pragma unroll
            for (int q = 0; q <= DIM; ++q) acc[q] = acc[q] + in[t * (DIM + 1) + q];
            if (last_id[t] >= 0) lid = last_id[t];
        }
        int slot = -1;
        for (int k = 0; k < n_ids; ++k)
            if (ids[k] == lid) slot = k;
        flag[r] = lid >= 0 ? 1 : 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d)
            value[(size_t)d * f.nD + r] =
                lid >= 0 ? acc[d] * coeff / acc[DIM] + (slot >= 0 ? id_vel[(size_t)slot * DIM + d] : 0.0) : 0.0;
    }
}

int fem_grid(const void* k, int threads) { return occupancy_grid(k, threads); }

}  // namespace

int launch_fem_constrain(int nD, long long nnz, int nm, int ns, const int32_t* row_ptr, const int32_t* cols,
                         const int32_t* con_idx, int n_con, const double* g, double* A, double* rhs, cudaStream_t s)
{
    k_fem_constrain<<<fem_grid((const void*)k_fem_constrain, 256), 256, 0, s>>>(nD, nnz, nm, ns, row_ptr, cols, con_idx,
                                                                                  n_con, g, A, rhs);
    return 1;
}

int launch_fem_velocity_bc(int dim, const FemArgs& f, const uint8_t* dmask, const int32_t* face_id, const double* P,
                           double* local, int32_t* last_id, int n_ids, const int32_t* ids, const double* id_vel,
                           double coeff, double* value, int32_t* flag, cudaStream_t s)
{
    if (dim == 2) {
        k_fem_bc_local<2><<<fem_grid((const void*)k_fem_bc_local<2>, 128), 128, 0, s>>>(f, dmask, face_id, P, local,
                                                                                       last_id);
        k_fem_bc_dof<2><<<fem_grid((const void*)k_fem_bc_dof<2>, 256), 256, 0, s>>>(f, local, last_id, n_ids, ids,
                                                                                   id_vel, coeff, value, flag);
    } else {
        k_fem_bc_local<3><<<fem_grid((const void*)k_fem_bc_local<3>, 128), 128, 0, s>>>(f, dmask, face_id, P, local,
                                                                                       last_id);
        k_fem_bc_dof<3><<<fem_grid((const void*)k_fem_bc_dof<3>, 256), 256, 0, s>>>(f, local, last_id, n_ids, ids,
                                                                                   id_vel, coeff, value, flag);
    }
    return 2;
}

int launch_fem_contrib(int dim, const FemArgs& f, bool fill, uint32_t* count, cudaStream_t s)
{
    if (dim == 2) k_fem_contrib<2><<<fem_grid((const void*)k_fem_contrib<2>, 256), 256, 0, s>>>(f, fill, count);
    else k_fem_contrib<3><<<fem_grid((const void*)k_fem_contrib<3>, 256), 256, 0, s>>>(f, fill, count);
    return 1;
}

int launch_fem_pattern(int dim, const FemArgs& f, bool fill, uint32_t* count, unsigned* err, cudaStream_t s)
{
    if (dim == 2) k_fem_pattern<2><<<fem_grid((const void*)k_fem_pattern<2>, 128), 128, 0, s>>>(f, fill, count, err);
    else k_fem_pattern<3><<<fem_grid((const void*)k_fem_pattern<3>, 128), 128, 0, s>>>(f, fill, count, err);
    return 1;
}

template <int DIM, int SYS>
static int fem_t(const FemArgs& f, cudaStream_t s)
{
    k_fem_local<DIM, SYS><<<fem_grid((const void*)k_fem_local<DIM, SYS>, FEM_WARPS * 32), FEM_WARPS * 32, 0, s>>>(f);
    int n = 2;
    if constexpr (SYS != FEM_CORRECTION) {
        if (f.fmask) {
            k_fem_faces<DIM, SYS><<<fem_grid((const void*)k_fem_faces<DIM, SYS>, 128), 128, 0, s>>>(f);
            n = 3;
        }
    }
    k_fem_gather<DIM, SYS><<<fem_grid((const void*)k_fem_gather<DIM, SYS>, 256), 256, 0, s>>>(f);
    return n;
}

int launch_fem_assemble(int dim, int sys, const FemArgs& f, cudaStream_t s)
{
    if (dim == 2) {
        if (sys == FEM_PREDICTION) return fem_t<2, FEM_PREDICTION>(f, s);
        if (sys == FEM_PRESSURE) return fem_t<2, FEM_PRESSURE>(f, s);
        return fem_t<2, FEM_CORRECTION>(f, s);
    }
    if (sys == FEM_PREDICTION) return fem_t<3, FEM_PREDICTION>(f, s);
    if (sys == FEM_PRESSURE) return fem_t<3, FEM_PRESSURE>(f, s);
    return fem_t<3, FEM_CORRECTION>(f, s);
}

}  // namespace pfem2
