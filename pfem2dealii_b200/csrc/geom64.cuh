// FP64 Q1 geometry: shape functions, the multilinear map, its Jacobian and
// inverse (deal.II FE_Q<dim>(1) and MappingQ1, used by the reference at
// src/pfem2particlehandler.cpp:91,97,131,155,193,394,400,425,463 and
// src/pfem2particle.cpp:190).
//
// The FP64 form compiles this header with --fmad=false: every product and sum
// is rounded separately in the written order, the same arithmetic as an
// FMA-free CPU build, so the FP64 particle path reproduces its CPU
// restatement bit for bit.  The FP32 form reuses it (with contraction) only
// for particles that cross a cell face.
#pragma once

#include "common.cuh"

namespace pfem2 {

__device__ __forceinline__ double lag64(int b, double t) { return b ? t : 1.0 - t; }

// N_i = prod_d (b_d ? xi_d : 1 - xi_d), vertex bits b_d = (i >> d) & 1.
template <int DIM>
__device__ __forceinline__ void shape64(const double* xi, double* N)
{
#pragma unroll
    for (int i = 0; i < (1 << DIM); ++i) {
        double n = lag64(i & 1, xi[0]);
        if (DIM > 1) n = n * lag64((i >> 1) & 1, xi[1]);
        if (DIM > 2) n = n * lag64((i >> 2) & 1, xi[2]);
        N[i] = n;
    }
}

// dN_i/dxi_k = (b_k ? 1 : -1) prod_{m != k} (b_m ? xi_m : 1 - xi_m), product in m order.
template <int DIM>
__device__ __forceinline__ void shape_grad64(const double* xi, double (*G)[DIM])
{
#pragma unroll
    for (int i = 0; i < (1 << DIM); ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            double g = ((i >> k) & 1) ? 1.0 : -1.0;
#pragma unroll
            for (int m = 0; m < DIM; ++m)
                if (m != k) g = g * lag64((i >> m) & 1, xi[m]);
            G[i][k] = g;
        }
}

template <int DIM>
__device__ __forceinline__ void fwd64(const double (*X)[DIM], const double* xi, double* x)
{
    double N[1 << DIM];
    shape64<DIM>(xi, N);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < (1 << DIM); ++i) acc = acc + N[i] * X[i][d];
        x[d] = acc;
    }
}

template <int DIM>
__device__ __forceinline__ void jac64(const double (*X)[DIM], const double* xi, double (*J)[DIM])
{
    double G[1 << DIM][DIM];
#pragma unroll
    for (int i = 0; i < (1 << DIM); ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            double g = ((i >> k) & 1) ? 1.0 : -1.0;
#pragma unroll
            for (int m = 0; m < DIM; ++m)
                if (m != k) g = g * lag64((i >> m) & 1, xi[m]);
            G[i][k] = g;
        }
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            double acc = 0.0;
#pragma unroll
            for (int i = 0; i < (1 << DIM); ++i) acc = acc + G[i][k] * X[i][d];
            J[d][k] = acc;
        }
}

// Adjugate times reciprocal determinant; returns the determinant.
template <int DIM>
__device__ __forceinline__ double invert64(const double (*A)[DIM], double (*Ai)[DIM])
{
    if constexpr (DIM == 2) {
        const double det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
        const double r = 1.0 / det;
        Ai[0][0] = A[1][1] * r;
        Ai[0][1] = -A[0][1] * r;
        Ai[1][0] = -A[1][0] * r;
        Ai[1][1] = A[0][0] * r;
        return det;
    } else {
        const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
        const double c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
        const double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
        const double det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
        const double r = 1.0 / det;
        Ai[0][0] = c00 * r;
        Ai[1][0] = c01 * r;
        Ai[2][0] = c02 * r;
        Ai[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * r;
        Ai[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * r;
        Ai[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * r;
        Ai[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * r;
        Ai[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * r;
        Ai[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * r;
        return det;
    }
}

template <int DIM>
__device__ __forceinline__ void matvec64(const double (*A)[DIM], const double* x, double* y)
{
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc = acc + A[k][d] * x[d];
        y[k] = acc;
    }
}

template <int DIM>
__device__ __forceinline__ double norm2_64(const double* a)
{
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) s = s + a[d] * a[d];
    return s;
}

// GeometryInfo<dim>::is_inside_unit_cell(p), no tolerance; NaN is outside.
template <int DIM, typename R>
__device__ __forceinline__ bool inside_unit(const R* xi)
{
    bool in = true;
#pragma unroll
    for (int d = 0; d < DIM; ++d) in = in && (xi[d] >= R(0) && xi[d] <= R(1));
    return in;
}

template <int DIM>
__device__ __forceinline__ bool inside_unit_eps(const double* xi, double eps)
{
    bool in = true;
#pragma unroll
    for (int d = 0; d < DIM; ++d) in = in && (xi[d] >= -eps && xi[d] <= 1.0 + eps);
    return in;
}

template <int DIM>
__device__ __forceinline__ bool near_face64(const double* xi)
{
    bool nf = false;
#pragma unroll
    for (int d = 0; d < DIM; ++d) nf = nf || fabs(xi[d]) < 1e-12 || fabs(1.0 - xi[d]) < 1e-12;
    return nf;
}

// 2D closed-form bilinear inverse: r = xi e + eta f + xi eta g with
// e = X1-X0, f = X2-X0, g = X3-X1-X2+X0, r = p-X0; eliminating xi leaves
// cross(f,g) eta^2 + (cross(f,e) - cross(r,g)) eta - cross(r,e) = 0, solved
// without cancellation, root nearest 1/2, xi by projection.  0 = success.
__device__ __forceinline__ int bilinear_exact64(const double (*X)[2], const double* p, double* xi)
{
    const double ex = X[1][0] - X[0][0], ey = X[1][1] - X[0][1];
    const double fx = X[2][0] - X[0][0], fy = X[2][1] - X[0][1];
    const double gx = ((X[3][0] - X[1][0]) - X[2][0]) + X[0][0];
    const double gy = ((X[3][1] - X[1][1]) - X[2][1]) + X[0][1];
    const double rx = p[0] - X[0][0], ry = p[1] - X[0][1];
    const double qa = fx * gy - fy * gx;
    const double qb = (fx * ey - fy * ex) - (rx * gy - ry * gx);
    const double qc = -(rx * ey - ry * ex);
    double eta;
    if (qa == 0.0) {
        if (qb == 0.0) return 1;
        eta = -qc / qb;
    } else {
        const double disc = qb * qb - 4.0 * qa * qc;
        if (!(disc >= 0.0)) return 1;
        const double sq = sqrt(disc);
        const double q = -0.5 * (qb + (qb >= 0.0 ? sq : -sq));
        if (q == 0.0) {
            eta = 0.0;
        } else {
            const double e1 = q / qa;
            const double e2 = qc / q;
            eta = (fabs(e1 - 0.5) < fabs(e2 - 0.5)) ? e1 : e2;
        }
    }
    const double wx = ex + eta * gx, wy = ey + eta * gy;
    const double tx = rx - eta * fx, ty = ry - eta * fy;
    const double ww = wx * wx + wy * wy;
    if (!(ww > 0.0)) return 1;
    xi[0] = (tx * wx + ty * wy) / ww;
    xi[1] = eta;
    return 0;
}

// Inverse of the least-squares affine approximation of one cell's map:
// column k of A is the mean edge vector in direction k, b = centroid - A/2.
// Written as aff = [A^-1 row-major | b]; NaN marks a singular cell.
template <int DIM>
__device__ __forceinline__ void affine_setup64(const double (*X)[DIM], double* aff)
{
    constexpr int NV = 1 << DIM;
    const double half = (double)(NV / 2);
    double A[DIM][DIM], Ai[DIM][DIM], b[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        double mean = 0.0;
#pragma unroll
        for (int i = 0; i < NV; ++i) mean = mean + X[i][d];
        mean = mean / (double)NV;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            double sp = 0.0, sm = 0.0;
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                if ((i >> k) & 1) sp = sp + X[i][d];
                else sm = sm + X[i][d];
            }
            A[d][k] = (sp - sm) / half;
        }
        double ac = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) ac = ac + A[d][k] * 0.5;
        b[d] = mean - ac;
    }
    const double det = invert64<DIM>(A, Ai);
    const bool bad = !(det != 0.0) || !isfinite(det);
#pragma unroll
    for (int k = 0; k < DIM; ++k)
#pragma unroll
        for (int d = 0; d < DIM; ++d) aff[k * DIM + d] = bad ? __longlong_as_double(0x7ff8000000000000ll) : Ai[k][d];
#pragma unroll
    for (int d = 0; d < DIM; ++d) aff[DIM * DIM + d] = b[d];
}

// MappingQ1::transform_real_to_unit_cell restated (deal.II's published
// strategy): 2D closed form accepted inside the unit cell within 1e-12;
// otherwise Newton from the affine guess clamped to the unit cell, residual
// weighted by J^-1, converged below 1e-11, step halved down to 0.05 while the
// weighted residual does not drop, one restart from the clamped iterate, fail
// on det <= 0 or after 20 iterations.  0 = success.
template <int DIM>
__device__ __forceinline__ int inverse_map64(const double (*X)[DIM], const double* __restrict__ aff,
                                             const double* p, double* xi_out)
{
    double xi[DIM], f[DIM], x[DIM], r[DIM];
    if constexpr (DIM == 2) {
        double e[2];
        if (bilinear_exact64(X, p, e) == 0 && inside_unit_eps<2>(e, 1e-12)) {
            xi_out[0] = e[0];
            xi_out[1] = e[1];
            return 0;
        }
    }
    {
        double Ai[DIM][DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k)
#pragma unroll
            for (int d = 0; d < DIM; ++d) Ai[k][d] = aff[k * DIM + d];
        if (Ai[0][0] != Ai[0][0]) return 1;
#pragma unroll
        for (int d = 0; d < DIM; ++d) r[d] = p[d] - aff[DIM * DIM + d];
        matvec64<DIM>(Ai, r, xi);
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi[d] = xi[d] < 0.0 ? 0.0 : (xi[d] > 1.0 ? 1.0 : xi[d]);
    fwd64<DIM>(X, xi, x);
#pragma unroll
    for (int d = 0; d < DIM; ++d) f[d] = x[d] - p[d];
    bool restarted = false;
    for (int it = 0; it < 20; ++it) {
        double J[DIM][DIM], Ji[DIM][DIM], delta[DIM], trial[DIM], ft[DIM], dt[DIM];
        jac64<DIM>(X, xi, J);
        const double det = invert64<DIM>(J, Ji);
        if (!(det > 0.0)) return 1;
        matvec64<DIM>(Ji, f, delta);
        const double dn = norm2_64<DIM>(delta);
        if (dn <= 1e-22) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi_out[d] = xi[d];
            return 0;
        }
        double step = 1.0, tn = 0.0;
        bool accepted = false;
        for (int ls = 0; ls < 8; ++ls) {  // 1, 1/2, ..., 1/32 then stop
#pragma unroll
            for (int d = 0; d < DIM; ++d) trial[d] = xi[d] - step * delta[d];
            fwd64<DIM>(X, trial, x);
#pragma unroll
            for (int d = 0; d < DIM; ++d) ft[d] = x[d] - p[d];
            matvec64<DIM>(Ji, ft, dt);
            tn = norm2_64<DIM>(dt);
            if (tn < dn) {
                accepted = true;
                break;
            }
            if (step > 0.05) step = step * 0.5;
            else break;
        }
        if (!accepted) {
            if (restarted) return 1;
            restarted = true;
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = xi[d] < 0.0 ? 0.0 : (xi[d] > 1.0 ? 1.0 : xi[d]);
            fwd64<DIM>(X, xi, x);
#pragma unroll
            for (int d = 0; d < DIM; ++d) f[d] = x[d] - p[d];
            continue;
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xi[d] = trial[d];
            f[d] = ft[d];
        }
        if (tn <= 1e-22) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi_out[d] = xi[d];
            return 0;
        }
    }
    return 1;
}

// Inverse of an affine cell's map from its stored inverse (aff = [A^-1 | b],
// x = A xi + b exactly for a parallelepiped).  0 = success (1: singular cell).
template <int DIM>
__device__ __forceinline__ int inverse_affine64(const double* __restrict__ aff, const double* p, double* xi)
{
    const double a00 = __ldg(aff);
    if (a00 != a00) return 1;
    double r[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) r[d] = p[d] - __ldg(aff + DIM * DIM + d);
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) acc = acc + __ldg(aff + k * DIM + d) * r[d];
        xi[k] = acc;
    }
    return 0;
}

template <int DIM>
__device__ __forceinline__ void load_cell64(const double* __restrict__ cellX, uint32_t c, double (*X)[DIM])
{
    const double* p = cellX + (size_t)c * ((1 << DIM) * DIM);
#pragma unroll
    for (int i = 0; i < (1 << DIM); ++i)
#pragma unroll
        for (int d = 0; d < DIM; ++d) X[i][d] = __ldg(p + i * DIM + d);
}

// u = sum_i N_i(xi) V[d][dof_i] from the staged component-major nodal
// vectors (V_d[dof] at Vd + d*nD), accumulated from zero in vertex order:
// the reference's interpolation (src/pfem2particlehandler.cpp:96-101).
template <int DIM>
__device__ __forceinline__ void velocity_from_dofs(const int32_t* __restrict__ cd, const double* __restrict__ Vd,
                                                   int nD, uint32_t c, const double* xi, double* u)
{
    constexpr int NV = 1 << DIM;
    double N[NV];
    shape64<DIM>(xi, N);
#pragma unroll
    for (int d = 0; d < DIM; ++d) u[d] = 0.0;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
        const int32_t dof = __ldg(cd + (size_t)c * NV + iv);
#pragma unroll
        for (int d = 0; d < DIM; ++d) u[d] = u[d] + N[iv] * __ldg(Vd + (size_t)d * nD + dof);
    }
}

}  // namespace pfem2
