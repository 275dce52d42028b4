// FP32 form geometry.  Each cell stores the coefficients of its multilinear
// map relative to vertex 0,  x(xi) - X0 = sum_{k=1}^{NV-1} a_k prod_{d in k} xi_d,
// as nested forward differences of the vertex coordinates (a_k = Delta^k X),
// which are exactly zero for the bilinear/trilinear terms of a parallelepiped
// cell.  A particle is advanced in reference coordinates: the displacement
// u dt is converted to an increment of xi by solving x(xi + d) - x(xi) = u dt,
// with the left side expanded in d so nothing cancels; accuracy therefore
// does not depend on where the cell sits in the domain.
#pragma once

#include "common.cuh"

namespace pfem2 {

template <int DIM>
struct Geo32 {
    float a[(1 << DIM) - 1][DIM];
    bool affine;
};

template <int DIM>
__device__ __forceinline__ void load_geo32(const float* __restrict__ geo, uint32_t c, Geo32<DIM>& g)
{
    constexpr int GS = Dims<DIM>::GEO;
    const float4* p = reinterpret_cast<const float4*>(geo + (size_t)c * GS);
    float buf[GS];
#pragma unroll
    for (int k = 0; k < GS / 4; ++k) {
        const float4 t = __ldg(p + k);
        buf[4 * k + 0] = t.x;
        buf[4 * k + 1] = t.y;
        buf[4 * k + 2] = t.z;
        buf[4 * k + 3] = t.w;
    }
#pragma unroll
    for (int k = 0; k < (1 << DIM) - 1; ++k)
#pragma unroll
        for (int d = 0; d < DIM; ++d) g.a[k][d] = buf[k * DIM + d];
    g.affine = buf[GS - 1] != 0.0f;
}

// Jacobian of the map at y.
template <int DIM>
__device__ __forceinline__ void jac32(const Geo32<DIM>& g, const float* y, float (*J)[DIM])
{
    if constexpr (DIM == 2) {
#pragma unroll
        for (int d = 0; d < 2; ++d) {
            J[d][0] = g.a[0][d] + g.a[2][d] * y[1];
            J[d][1] = g.a[1][d] + g.a[2][d] * y[0];
        }
    } else {
        // a[0]=a_{x} a[1]=a_{y} a[2]=a_{xy} a[3]=a_{z} a[4]=a_{xz} a[5]=a_{yz} a[6]=a_{xyz}
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            J[d][0] = g.a[0][d] + g.a[2][d] * y[1] + g.a[4][d] * y[2] + g.a[6][d] * (y[1] * y[2]);
            J[d][1] = g.a[1][d] + g.a[2][d] * y[0] + g.a[5][d] * y[2] + g.a[6][d] * (y[0] * y[2]);
            J[d][2] = g.a[3][d] + g.a[4][d] * y[0] + g.a[5][d] * y[1] + g.a[6][d] * (y[0] * y[1]);
        }
    }
}

// x(xi + d) - x(xi), expanded in d.
template <int DIM>
__device__ __forceinline__ void delta32(const Geo32<DIM>& g, const float* xi, const float* dl, float* out)
{
    if constexpr (DIM == 2) {
        const float y1 = xi[1] + dl[1];
        const float b = dl[0] * y1 + xi[0] * dl[1];
#pragma unroll
        for (int d = 0; d < 2; ++d) out[d] = g.a[0][d] * dl[0] + g.a[1][d] * dl[1] + g.a[2][d] * b;
    } else {
        const float y1 = xi[1] + dl[1], y2 = xi[2] + dl[2];
        const float bxy = dl[0] * y1 + xi[0] * dl[1];
        const float bxz = dl[0] * y2 + xi[0] * dl[2];
        const float byz = dl[1] * y2 + xi[1] * dl[2];
        const float bxyz = dl[0] * (y1 * y2) + xi[0] * byz;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            out[d] = g.a[0][d] * dl[0] + g.a[1][d] * dl[1] + g.a[3][d] * dl[2] + g.a[2][d] * bxy +
                     g.a[4][d] * bxz + g.a[5][d] * byz + g.a[6][d] * bxyz;
    }
}

template <int DIM>
__device__ __forceinline__ float invert32(const float (*A)[DIM], float (*Ai)[DIM])
{
    if constexpr (DIM == 2) {
        const float det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
        const float r = 1.0f / det;
        Ai[0][0] = A[1][1] * r;
        Ai[0][1] = -A[0][1] * r;
        Ai[1][0] = -A[1][0] * r;
        Ai[1][1] = A[0][0] * r;
        return det;
    } else {
        const float c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
        const float c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
        const float c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
        const float det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
        const float r = 1.0f / det;
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
__device__ __forceinline__ void shape32(const float* xi, float* N)
{
#pragma unroll
    for (int i = 0; i < (1 << DIM); ++i) {
        float n = (i & 1) ? xi[0] : 1.0f - xi[0];
        if (DIM > 1) n *= ((i >> 1) & 1) ? xi[1] : 1.0f - xi[1];
        if (DIM > 2) n *= ((i >> 2) & 1) ? xi[2] : 1.0f - xi[2];
        N[i] = n;
    }
}

// Reference-coordinate increment d with x(xi + d) - x(xi) = dx, from
// d0 = J(xi)^-1 dx (exact for affine cells), then the chord iteration
// d -= J(xi)^-1 (x(xi + d) - x(xi) - dx) with the start point's inverse
// Jacobian: on the mildly non-affine cells a sub-step crosses, the error
// falls by the cell's twist times |d| per iteration (a few hundredths), as
// fast as Newton needs in FP32, without a Jacobian and an inverse per
// iteration.  Returns false when the iteration does not settle within 8
// corrections (the caller then relocates in FP64).
template <int DIM>
__device__ __forceinline__ bool advance32(const Geo32<DIM>& g, const float* xi, const float* dx, float* dl)
{
    float J[DIM][DIM], Ji[DIM][DIM];
    jac32<DIM>(g, xi, J);
    const float det = invert32<DIM>(J, Ji);
    if (!(det > 0.0f)) return false;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        float s = 0.0f;
#pragma unroll
        for (int d = 0; d < DIM; ++d) s += Ji[k][d] * dx[d];
        dl[k] = s;
    }
    if (g.affine) return true;
    for (int it = 0; it < 8; ++it) {
        float r[DIM];
        delta32<DIM>(g, xi, dl, r);
#pragma unroll
        for (int d = 0; d < DIM; ++d) r[d] -= dx[d];
        float mx = 0.0f;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            float s = 0.0f;
#pragma unroll
            for (int d = 0; d < DIM; ++d) s += Ji[k][d] * r[d];
            dl[k] -= s;
            mx = fmaxf(mx, fabsf(s));
        }
        if (mx <= 2e-7f) return true;
    }
    return false;
}

}  // namespace pfem2
