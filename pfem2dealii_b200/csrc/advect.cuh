// Fused particle pass: velocity correction + S sub-steps of (interpolate,
// Euler advance, relocate), one thread per particle.
//
// Follows, per particle, correct_particle_velocity
// (src/pfem2particlehandler.cpp:112-139), move_particles (:142-167) and
// sort_particles_into_subdomains_and_cells (:413-503).  The reference runs
// each stage over the whole particle vector; the stages touch nothing but the
// particle itself and read-only mesh data, so running them back to back per
// particle gives the same values while reading and writing each particle once
// per time step.  Particles arrive sorted by cell, so the cell geometry and
// DoF velocities a warp needs are mostly the same few cache lines.
#pragma once

#include "common.cuh"
#include "geom64.cuh"
#include "geom32.cuh"

namespace pfem2 {

struct RelocCounters {
    unsigned long long map_failures = 0, near_face = 0, searched = 0;
    uint32_t err = 0;
};

template <int DIM>
struct Vec {
    double v[DIM];
};

constexpr uint32_t SRCH_FOUND = 1u, SRCH_NEAR = 2u, SRCH_OVERFLOW = 4u;

struct SearchOut {
    double xi[3];
    uint32_t cell;
    uint32_t flags;
    uint32_t map_failures;
};

// Vertex-patch search for a particle that left cell c
// (sort_particles_into_subdomains_and_cells, src/pfem2particlehandler.cpp:438-491):
//  1. closest vertex of c seen from the previous position F(xi_old) along
//     velocity_ext (src/pfem2particle.cpp:186-211): strict '>' keeps the
//     first maximum, NaN never wins;
//  2. cells around that vertex by descending dot product of their centre
//     direction with the unit vertex->particle direction, ties in cell order
//     (stable, as libstdc++'s std::sort on <= 16 items) (:445-456);
//  3. the first cell whose inverse map lands inside wins (:458-478); the
//     particle's own cell is not retried (its inverse map is deterministic
//     and already failed).
// Out of line and by value, so the caller's registers stay registers.
template <int DIM>
__device__ __noinline__ SearchOut search64(const MeshDev m, uint32_t c, Vec<DIM> xo, Vec<DIM> ve, Vec<DIM> xp)
{
    constexpr int NV = 1 << DIM;
    constexpr int AFF = Dims<DIM>::AFF;
    SearchOut out;
    out.cell = c;
    out.flags = 0;
    out.map_failures = 0;
    double X[NV][DIM];
    load_cell64<DIM>(m.cellX, c, X);
    int cvx = 0;
    {
        double old[DIM], vn[DIM];
        fwd64<DIM>(X, xo.v, old);
        const double vnorm = sqrt(norm2_64<DIM>(ve.v));
#pragma unroll
        for (int d = 0; d < DIM; ++d) vn[d] = ve.v[d] / vnorm;
        double best = 0.0;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double ptv[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) ptv[d] = X[v][d] - old[d];
            const double pn = sqrt(norm2_64<DIM>(ptv));
#pragma unroll
            for (int d = 0; d < DIM; ++d) ptv[d] = ptv[d] / pn;
            double ang = vn[0] * ptv[0];
#pragma unroll
            for (int d = 1; d < DIM; ++d) ang = ang + vn[d] * ptv[d];
            if (v == 0) best = ang;
            else if (ang > best) {
                best = ang;
                cvx = v;
            }
        }
    }
    double vtp[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) vtp[d] = xp.v[d] - X[cvx][d];
    {
        const double vn = sqrt(norm2_64<DIM>(vtp));
#pragma unroll
        for (int d = 0; d < DIM; ++d) vtp[d] = vtp[d] / vn;
    }
    const int32_t vid = __ldg(m.cv + (size_t)c * NV + cvx);
    const int32_t b = __ldg(m.v2c_off + vid);
    int n = __ldg(m.v2c_off + vid + 1) - b;
    if (n > MAX_CAND) {
        out.flags |= SRCH_OVERFLOW;
        n = MAX_CAND;
    }
    double dots[MAX_CAND];
    uint8_t perm[MAX_CAND];
    for (int k = 0; k < n; ++k) {
        const double* cd = m.v2c_dirs + (size_t)(b + k) * DIM;
        double s = __ldg(cd) * vtp[0];
#pragma unroll
        for (int d = 1; d < DIM; ++d) s = s + __ldg(cd + d) * vtp[d];
        dots[k] = s;
        perm[k] = (uint8_t)k;
    }
    for (int i = 1; i < n; ++i) {  // stable insertion sort, descending
        const uint8_t pi = perm[i];
        const double key = dots[pi];
        int j = i;
        while (j > 0 && key > dots[perm[j - 1]]) {
            perm[j] = perm[j - 1];
            --j;
        }
        perm[j] = pi;
    }
    for (int k = 0; k < n; ++k) {
        const uint32_t cand = (uint32_t)__ldg(m.v2c_cells + b + perm[k]);
        if (cand == c) continue;
        load_cell64<DIM>(m.cellX, cand, X);
        double xin[DIM];
        const int st = inverse_map64<DIM>(X, m.aff + (size_t)cand * AFF, xp.v, xin);
        if (st) {
            out.map_failures++;
            continue;
        }
        if (inside_unit<DIM>(xin)) {
            out.cell = cand;
            out.flags |= SRCH_FOUND;
#pragma unroll
            for (int d = 0; d < DIM; ++d) out.xi[d] = xin[d];
            if (near_face64<DIM>(xin)) out.flags |= SRCH_NEAR;
            return out;
        }
    }
    return out;
}

template <int DIM>
__device__ __forceinline__ bool take_search(const SearchOut& so, uint32_t& c, double* xi, RelocCounters& rc)
{
    rc.searched++;
    rc.map_failures += so.map_failures;
    if (so.flags & SRCH_OVERFLOW) rc.err |= ERR_CAND_OVERFLOW;
    if (!(so.flags & SRCH_FOUND)) return false;
    if (so.flags & SRCH_NEAR) rc.near_face++;
    c = so.cell;
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi[d] = so.xi[d];
    return true;
}

// Full FP64 relocation of an FP32-form particle: rebuild x = F(xi) + u dt_p in
// FP64, inverse map in the own cell, then the vertex-patch search.
template <int DIM>
__device__ __noinline__ SearchOut fallback64(const MeshDev m, uint32_t c, Vec<DIM> xo, Vec<DIM> ue, double dtp)
{
    constexpr int AFF = Dims<DIM>::AFF;
    double X[1 << DIM][DIM], x[DIM], xin[DIM];
    load_cell64<DIM>(m.cellX, c, X);
    fwd64<DIM>(X, xo.v, x);
#pragma unroll
    for (int d = 0; d < DIM; ++d) x[d] = x[d] + ue.v[d] * dtp;
    const int st = inverse_map64<DIM>(X, m.aff + (size_t)c * AFF, x, xin);
    if (st == 0 && inside_unit<DIM>(xin)) {
        SearchOut out;
        out.cell = c;
        out.flags = SRCH_FOUND | (near_face64<DIM>(xin) ? SRCH_NEAR : 0u);
        out.map_failures = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) out.xi[d] = xin[d];
        return out;
    }
    Vec<DIM> xp;
#pragma unroll
    for (int d = 0; d < DIM; ++d) xp.v[d] = x[d];
    SearchOut out = search64<DIM>(m, c, xo, ue, xp);
    out.map_failures += st ? 1u : 0u;
    return out;
}

template <int DIM>
__device__ __forceinline__ void finish_counters(const StepArgs& a, unsigned long long lost, const RelocCounters& rc,
                                                unsigned long long fb)
{
    warp_count(&a.stats->lost, lost);
    warp_count(&a.stats->map_failures, rc.map_failures);
    warp_count(&a.stats->near_face, rc.near_face);
    warp_count(&a.stats->searched, rc.searched);
    warp_count(&a.stats->fallback64, fb);
    const unsigned e = __reduce_or_sync(0xffffffffu, rc.err);
    if ((threadIdx.x & 31) == 0 && e) atomicOr(&a.stats->error_flags, e);
}

// FP64 form: the reference's own state and arithmetic (global location x
// advanced as x + u*dt_p, reference coordinates re-derived by the inverse map).
template <int DIM>
__global__ void __launch_bounds__(256) k_advect64(StepArgs a)
{
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    const MeshDev& m = a.mesh;
    const uint32_t n = (uint32_t)a.stats->n_particles;
    const double* __restrict__ V = (const double*)a.Vaos;
    const double* __restrict__ dV = (const double*)a.dVaos;
    RelocCounters rc;
    unsigned long long lost = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t c = a.S0.cell[i];
        double x[DIM], xi[DIM], v[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            x[d] = ((const double*)a.S0.x[d])[i];
            xi[d] = ((const double*)a.S0.xi[d])[i];
            v[d] = ((const double*)a.S0.v[d])[i];
        }
        bool alive = c < (uint32_t)m.nC;
        if (!alive) rc.err |= ERR_BAD_CELL;
        if (alive) {
            double X[NV][DIM];
            load_cell64<DIM>(m.cellX, c, X);
            int32_t dof[NV];
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) dof[iv] = __ldg(m.cd + (size_t)c * NV + iv);
            if (a.do_correct) {  // src/pfem2particlehandler.cpp:126-138
                double N[NV], corr[DIM];
                shape64<DIM>(xi, N);
#pragma unroll
                for (int d = 0; d < DIM; ++d) corr[d] = 0.0;
#pragma unroll
                for (int iv = 0; iv < NV; ++iv)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) corr[d] = corr[d] + N[iv] * __ldg(dV + (size_t)dof[iv] * VS + d);
#pragma unroll
                for (int d = 0; d < DIM; ++d) v[d] = v[d] + corr[d];
            }
            for (int s = 0; s < a.pp.S; ++s) {  // :150-167
                double N[NV], u[DIM];
                shape64<DIM>(xi, N);
#pragma unroll
                for (int d = 0; d < DIM; ++d) u[d] = 0.0;
#pragma unroll
                for (int iv = 0; iv < NV; ++iv)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) u[d] = u[d] + N[iv] * __ldg(V + (size_t)dof[iv] * VS + d);
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const double st = u[d] * a.pp.dtp;
                    x[d] = x[d] + st;
                }
                // relocation, :420-491
                double xin[DIM];
                const int st = inverse_map64<DIM>(X, m.aff + (size_t)c * Dims<DIM>::AFF, x, xin);
                if (st) rc.map_failures++;
                if (st == 0 && inside_unit<DIM>(xin)) {
#pragma unroll
                    for (int d = 0; d < DIM; ++d) xi[d] = xin[d];
                    if (near_face64<DIM>(xin)) rc.near_face++;
                    continue;
                }
                Vec<DIM> xo, ve, xp;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    xo.v[d] = xi[d];
                    ve.v[d] = u[d];
                    xp.v[d] = x[d];
                }
                const SearchOut so = search64<DIM>(m, c, xo, ve, xp);
                if (!take_search<DIM>(so, c, xi, rc)) {
                    alive = false;
                    break;
                }
                load_cell64<DIM>(m.cellX, c, X);
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) dof[iv] = __ldg(m.cd + (size_t)c * NV + iv);
            }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            ((double*)a.T.x[d])[i] = x[d];
            ((double*)a.T.xi[d])[i] = xi[d];
            ((double*)a.T.v[d])[i] = v[d];
        }
        if (alive) {
            a.key[i] = c;
            a.slot[i] = atomicAdd(a.cell_count + c, 1u);
        } else {
            a.key[i] = LOST;
            lost++;
        }
    }
    finish_counters<DIM>(a, lost, rc, 0);
}

// FP32 form: state = (cell, xi, v) in FP32.  A sub-step converts u*dt_p to a
// reference-coordinate increment in FP32 (advance32); if the particle stays
// in its cell the step is done, otherwise the global position is rebuilt in
// FP64 (x = F(xi) + u dt_p) and relocated by the FP64 search above.
template <int DIM>
__global__ void __launch_bounds__(256) k_advect32(StepArgs a)
{
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    const MeshDev& m = a.mesh;
    const uint32_t n = (uint32_t)a.stats->n_particles;
    const float* __restrict__ V = (const float*)a.Vaos;
    const float* __restrict__ dV = (const float*)a.dVaos;
    RelocCounters rc;
    unsigned long long lost = 0, fb = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t c = a.S0.cell[i];
        float xi[DIM], v[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xi[d] = ((const float*)a.S0.xi[d])[i];
            v[d] = ((const float*)a.S0.v[d])[i];
        }
        bool alive = c < (uint32_t)m.nC;
        if (!alive) rc.err |= ERR_BAD_CELL;
        if (alive) {
            Geo32<DIM> g;
            load_geo32<DIM>(m.geo32, c, g);
            int32_t dof[NV];
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) dof[iv] = __ldg(m.cd + (size_t)c * NV + iv);
            if (a.do_correct) {
                float N[NV];
                shape32<DIM>(xi, N);
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) {
                    if constexpr (DIM == 3) {
                        const float4 t = __ldg(reinterpret_cast<const float4*>(dV) + dof[iv]);
                        v[0] += N[iv] * t.x;
                        v[1] += N[iv] * t.y;
                        v[2] += N[iv] * t.z;
                    } else {
                        const float2 t = __ldg(reinterpret_cast<const float2*>(dV) + dof[iv]);
                        v[0] += N[iv] * t.x;
                        v[1] += N[iv] * t.y;
                    }
                }
            }
            for (int s = 0; s < a.pp.S; ++s) {
                float N[NV], u[DIM];
                shape32<DIM>(xi, N);
#pragma unroll
                for (int d = 0; d < DIM; ++d) u[d] = 0.0f;
#pragma unroll
                for (int iv = 0; iv < NV; ++iv) {
                    if constexpr (DIM == 3) {
                        const float4 t = __ldg(reinterpret_cast<const float4*>(V) + dof[iv]);
                        u[0] += N[iv] * t.x;
                        u[1] += N[iv] * t.y;
                        u[2] += N[iv] * t.z;
                    } else {
                        const float2 t = __ldg(reinterpret_cast<const float2*>(V) + dof[iv]);
                        u[0] += N[iv] * t.x;
                        u[1] += N[iv] * t.y;
                    }
                }
                const float dtp = (float)a.pp.dtp;
                float dx[DIM], dl[DIM], y[DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d) dx[d] = u[d] * dtp;
                const bool ok = advance32<DIM>(g, xi, dx, dl);
#pragma unroll
                for (int d = 0; d < DIM; ++d) y[d] = xi[d] + dl[d];
                if (ok && inside_unit<DIM>(y)) {
#pragma unroll
                    for (int d = 0; d < DIM; ++d) xi[d] = y[d];
                    continue;
                }
                // face crossing (or unsettled Newton): FP64 relocation
                fb++;
                Vec<DIM> xo, ue;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    xo.v[d] = (double)xi[d];
                    ue.v[d] = (double)u[d];
                }
                const uint32_t c0 = c;
                const SearchOut so = fallback64<DIM>(m, c, xo, ue, a.pp.dtp);
                double xin[DIM];
                const bool searched = so.cell != c0 || !(so.flags & SRCH_FOUND);
                if (searched) {
                    if (!take_search<DIM>(so, c, xin, rc)) {
                        alive = false;
                        break;
                    }
                } else {
                    rc.map_failures += so.map_failures;
                    if (so.flags & SRCH_NEAR) rc.near_face++;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) xin[d] = so.xi[d];
                }
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const float t = (float)xin[d];
                    xi[d] = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
                }
                if (c != c0) {
                    load_geo32<DIM>(m.geo32, c, g);
#pragma unroll
                    for (int iv = 0; iv < NV; ++iv) dof[iv] = __ldg(m.cd + (size_t)c * NV + iv);
                }
            }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            ((float*)a.T.xi[d])[i] = xi[d];
            ((float*)a.T.v[d])[i] = v[d];
        }
        if (alive) {
            a.key[i] = c;
            a.slot[i] = atomicAdd(a.cell_count + c, 1u);
        } else {
            a.key[i] = LOST;
            lost++;
        }
    }
    finish_counters<DIM>(a, lost, rc, fb);
}

}  // namespace pfem2
