// Per-cell kernels: seeding, count correction (survivor/seed decisions and
// the final sorted layout), projection partial sums and the DoF gather.
//
// One warp owns one cell at a time.  Its particles arrive through the
// bucketed index list (cell-major), their extended part index is counted in
// shared memory, and the decisions of check_particle_distribution
// (src/pfem2particlehandler.cpp:356-410) follow from the counts alone:
// a part keeps min(count, max+1) particles, chosen by ascending key(id), and
// every real part left empty in a cell that had particles gets one new
// particle at its centre.  New ids continue the running count in
// (cell ascending, part x-major) order, the order in which the reference
// hands them out.  The output is sorted by (cell, part, key), so the layout
// and every floating-point sum taken over it are deterministic.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "geom32.cuh"
#include "geom64.cuh"

namespace pfem2 {

template <typename Real>
__device__ __forceinline__ Real ldr(const void* p, uint32_t i)
{
    return reinterpret_cast<const Real*>(p)[i];
}

template <typename Real>
__device__ __forceinline__ void str(void* p, uint32_t i, Real v)
{
    reinterpret_cast<Real*>(p)[i] = v;
}

// Velocity interpolation at xi, FP64 (reference arithmetic) or FP32.
template <int DIM, typename Real>
__device__ __forceinline__ void interp_v(const MeshDev& m, const void* Vaos, uint32_t c, const Real* xi, Real* u)
{
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    Real N[NV];
    if constexpr (std::is_same<Real, double>::value) shape64<DIM>(xi, N);
    else shape32<DIM>(xi, N);
#pragma unroll
    for (int d = 0; d < DIM; ++d) u[d] = Real(0);
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
        const int32_t dof = __ldg(m.cd + (size_t)c * NV + iv);
#pragma unroll
        for (int d = 0; d < DIM; ++d) u[d] = u[d] + N[iv] * __ldg(reinterpret_cast<const Real*>(Vaos) + (size_t)dof * VS + d);
    }
}

// A new particle at the centre of part idx of cell c (seed_particles
// :87-104 and check_particle_distribution :390-407): xi = (idx + 1/2) h,
// x = F(xi) (FP64 form), v = interpolated V.
template <int DIM, typename Real>
__device__ __forceinline__ void write_new_particle(const StepArgs& a, const PartState& S, uint32_t dst, uint32_t c,
                                                   const int* idx, uint32_t id)
{
    Real xi[DIM], v[DIM];
    double xid[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        xid[d] = (idx[d] + 0.5) * a.pp.h[d];
        xi[d] = (Real)xid[d];
    }
    interp_v<DIM, Real>(a.mesh, a.Vaos, c, xi, v);
    if constexpr (std::is_same<Real, double>::value) {
        double X[1 << DIM][DIM], x[DIM];
        load_cell64<DIM>(a.mesh.cellX, c, X);
        fwd64<DIM>(X, xid, x);
#pragma unroll
        for (int d = 0; d < DIM; ++d) str<double>(S.x[d], dst, x[d]);
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        str<Real>(S.xi[d], dst, xi[d]);
        str<Real>(S.v[d], dst, v[d]);
    }
    S.cell[dst] = c;
    S.id[dst] = id;
}

// seed_particles (:43-109): nC x npart particles, cell-major, parts x-major.
template <int DIM, typename Real>
__global__ void k_seed(StepArgs a, uint32_t* cell_start)
{
    const uint32_t total = (uint32_t)a.mesh.nC * a.pp.npart;
    const uint32_t id0 = a.stats->next_id;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t c = t / a.pp.npart;
        const int k = (int)(t % a.pp.npart);
        int idx[3] = {0, 0, 0};
        if (DIM == 2) {
            idx[0] = k / a.pp.q[1];
            idx[1] = k % a.pp.q[1];
        } else {
            idx[0] = k / (a.pp.q[1] * a.pp.q[2]);
            idx[1] = (k / a.pp.q[2]) % a.pp.q[1];
            idx[2] = k % a.pp.q[2];
        }
        write_new_particle<DIM, Real>(a, a.S0, t, c, idx, id0 + t + 1);
        if (k == 0) cell_start[c] = t;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cell_start[a.mesh.nC] = total;
}

template <int DIM, typename Real>
__device__ __forceinline__ uint2 part_key(const StepArgs& a, uint32_t i)
{
    Real xi[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) xi[d] = ldr<Real>(a.T.xi[d], i);
    return make_uint2((uint32_t)ext_part<DIM, Real>(xi, a.pp), key_of(a.S0.id[i], a.pp.seed));
}

__device__ __forceinline__ int survivors(int cnt, int maxpp, int apply)
{
    if (!apply) return cnt;
    if (maxpp < 0) return 0;
    return cnt < maxpp + 1 ? cnt : maxpp + 1;
}

// Count pass: per cell, seeds << 32 | (survivors + seeds).
template <int DIM, typename Real>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_count(StepArgs a)
{
    __shared__ int cnt_s[CELL_WARPS][NPE_MAX];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* cnt = cnt_s[warp];
    const int npe = a.pp.npe;
    for (int c = blockIdx.x * CELL_WARPS + warp; c < a.mesh.nC; c += gridDim.x * CELL_WARPS) {
        const uint32_t b = a.cell_off[c], e = a.cell_off[c + 1];
        if (b == e) {
            if (lane == 0) a.packed[c] = 0ull;
            continue;
        }
        for (int p = lane; p < npe; p += 32) cnt[p] = 0;
        __syncwarp();
        for (uint32_t j = b + lane; j < e; j += 32) {
            const uint2 pk = part_key<DIM, Real>(a, a.idx[j]);
            atomicAdd(cnt + pk.x, 1);
        }
        __syncwarp();
        unsigned surv = 0, seeds = 0;
        for (int p = lane; p < npe; p += 32) {
            const int s = survivors(cnt[p], a.pp.maxpp, a.apply_counts);
            int idx[3];
            surv += s;
            if (a.apply_counts && s == 0 && real_part<DIM>(p, a.pp, idx)) seeds++;
        }
        surv = __reduce_add_sync(0xffffffffu, surv);
        seeds = __reduce_add_sync(0xffffffffu, seeds);
        if (lane == 0) a.packed[c] = ((unsigned long long)seeds << 32) | (unsigned long long)(surv + seeds);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Projection partials: per cell and local vertex iv, sum_p N_iv v_p and
// sum_p N_iv over the cell's final particles in their sorted order
// (project_particle_fields :191-199 restricted to one cell).  Lane l sums
// particles l, l+32, ...; the 32 lanes are combined by a butterfly
// reduce-scatter after which lane k holds entry k = iv*4 + comp (comp = DIM
// is the weight).  FP32 sums are compensated (TwoSum pairs).
// ---------------------------------------------------------------------------

__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e)
{
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

template <int W, typename T>
__device__ __forceinline__ T reduce_scatter(T (&vals)[W], int lane)
{
    // after the loop lane l holds the total of entry (l & (W-1))
#pragma unroll
    for (int s = W / 2; s >= 1; s >>= 1) {
        const bool upper = lane & s;
#pragma unroll
        for (int k = 0; k < s; ++k) {
            const T send = upper ? vals[k] : vals[k + s];
            const T keep = upper ? vals[k + s] : vals[k];
            vals[k] = keep + __shfl_xor_sync(0xffffffffu, send, s);
        }
    }
    T r = vals[0];
#pragma unroll
    for (int s = W; s < 32; s <<= 1) r += __shfl_xor_sync(0xffffffffu, r, s);
    return r;
}

template <int W>
__device__ __forceinline__ float reduce_scatter_comp(float (&hi)[W], float (&lo)[W], int lane)
{
#pragma unroll
    for (int s = W / 2; s >= 1; s >>= 1) {
        const bool upper = lane & s;
#pragma unroll
        for (int k = 0; k < s; ++k) {
            const float sh = upper ? hi[k] : hi[k + s], sl = upper ? lo[k] : lo[k + s];
            const float kh = upper ? hi[k + s] : hi[k], kl = upper ? lo[k + s] : lo[k];
            const float rh = __shfl_xor_sync(0xffffffffu, sh, s);
            const float rl = __shfl_xor_sync(0xffffffffu, sl, s);
            float t, e;
            two_sum(kh, rh, t, e);
            hi[k] = t;
            lo[k] = e + (kl + rl);
        }
    }
    float h = hi[0], l = lo[0];
#pragma unroll
    for (int s = W; s < 32; s <<= 1) {
        const float rh = __shfl_xor_sync(0xffffffffu, h, s);
        const float rl = __shfl_xor_sync(0xffffffffu, l, s);
        float t, e;
        two_sum(h, rh, t, e);
        h = t;
        l = e + (l + rl);
    }
    return h + l;
}

template <int DIM, typename Real>
__device__ __forceinline__ void cell_partials(const StepArgs& a, const PartState& S, uint32_t c, uint32_t fb,
                                              uint32_t fcount, int lane)
{
    constexpr int NV = 1 << DIM, PW = Dims<DIM>::PW;
    if constexpr (std::is_same<Real, double>::value) {
        double vals[PW];
#pragma unroll
        for (int k = 0; k < PW; ++k) vals[k] = 0.0;
        for (uint32_t j = lane; j < fcount; j += 32) {
            double xi[DIM], v[DIM], N[NV];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                xi[d] = ldr<double>(S.xi[d], fb + j);
                v[d] = ldr<double>(S.v[d], fb + j);
            }
            shape64<DIM>(xi, N);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) {
#pragma unroll
                for (int d = 0; d < DIM; ++d) vals[iv * 4 + d] = vals[iv * 4 + d] + N[iv] * v[d];
                vals[iv * 4 + DIM] = vals[iv * 4 + DIM] + N[iv];
            }
        }
        const double r = reduce_scatter<PW, double>(vals, lane);
        if (lane < PW) reinterpret_cast<double*>(a.partials)[(size_t)c * PW + lane] = r;
    } else {
        float hi[PW], lo[PW];
#pragma unroll
        for (int k = 0; k < PW; ++k) hi[k] = lo[k] = 0.0f;
        for (uint32_t j = lane; j < fcount; j += 32) {
            float xi[DIM], v[DIM], N[NV];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                xi[d] = ldr<float>(S.xi[d], fb + j);
                v[d] = ldr<float>(S.v[d], fb + j);
            }
            shape32<DIM>(xi, N);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) {
#pragma unroll
                for (int d = 0; d <= DIM; ++d) {
                    const float term = d < DIM ? N[iv] * v[d] : N[iv];
                    float t, e;
                    two_sum(hi[iv * 4 + d], term, t, e);
                    hi[iv * 4 + d] = t;
                    lo[iv * 4 + d] += e;
                }
            }
        }
        const float r = reduce_scatter_comp<PW>(hi, lo, lane);
        if (lane < PW) reinterpret_cast<float*>(a.partials)[(size_t)c * PW + lane] = r;
    }
}

// Write pass: survivors in (part, key) order, then the new particles, into
// the next sorted state; then the cell's projection partials.
template <int DIM, typename Real>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_write(StepArgs a, uint32_t* cell_start)
{
    __shared__ int cnt_s[CELL_WARPS][NPE_MAX];
    __shared__ int pfx_s[CELL_WARPS][NPE_MAX];   // final position of each part's first particle
    __shared__ int spfx_s[CELL_WARPS][NPE_MAX];  // number of new particles in earlier parts
    __shared__ uint2 kc_s[CELL_WARPS][KEY_CACHE];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* cnt = cnt_s[warp];
    int* pfx = pfx_s[warp];
    int* spfx = spfx_s[warp];
    uint2* kc = kc_s[warp];
    const int npe = a.pp.npe;
    const uint32_t id0 = a.stats->next_id;
    const uint32_t cap = a.capacity;
    unsigned long long removed = 0;
    uint32_t err = 0;
    for (int c = blockIdx.x * CELL_WARPS + warp; c < a.mesh.nC; c += gridDim.x * CELL_WARPS) {
        const uint32_t b = a.cell_off[c], e = a.cell_off[c + 1];
        const uint32_t nseg = e - b;
        const unsigned long long po = a.packed_off[c];
        const uint32_t fb = (uint32_t)po, sb = (uint32_t)(po >> 32);
        if (lane == 0) cell_start[c] = fb;
        if (nseg == 0) {
            cell_partials<DIM, Real>(a, a.S1, (uint32_t)c, fb, 0, lane);
            continue;
        }
        for (int p = lane; p < npe; p += 32) cnt[p] = 0;
        __syncwarp();
        for (uint32_t j = lane; j < nseg; j += 32) {
            const uint2 pk = part_key<DIM, Real>(a, a.idx[b + j]);
            atomicAdd(cnt + pk.x, 1);
            if (j < KEY_CACHE) kc[j] = pk;
        }
        __syncwarp();
        int run = 0, srun = 0;
        for (int base = 0; base < npe; base += 32) {
            const int p = base + lane;
            int fc = 0, sf = 0;
            if (p < npe) {
                const int s = survivors(cnt[p], a.pp.maxpp, a.apply_counts);
                int idx[3];
                sf = (a.apply_counts && s == 0 && real_part<DIM>(p, a.pp, idx)) ? 1 : 0;
                fc = s + sf;
            }
            int ifc = fc, isf = sf;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t1 = __shfl_up_sync(0xffffffffu, ifc, o);
                const int t2 = __shfl_up_sync(0xffffffffu, isf, o);
                if (lane >= o) {
                    ifc += t1;
                    isf += t2;
                }
            }
            if (p < npe) {
                pfx[p] = run + ifc - fc;
                spfx[p] = srun + isf - sf;
            }
            run += __shfl_sync(0xffffffffu, ifc, 31);
            srun += __shfl_sync(0xffffffffu, isf, 31);
        }
        __syncwarp();
        // survivors
        for (uint32_t j = lane; j < nseg; j += 32) {
            const uint32_t i = a.idx[b + j];
            const uint2 pk = j < KEY_CACHE ? kc[j] : part_key<DIM, Real>(a, i);
            const int k = cnt[pk.x];
            int rank = 0;
            if (k > 1) {
                for (uint32_t jj = 0; jj < nseg; ++jj) {
                    const uint2 q = jj < KEY_CACHE ? kc[jj] : part_key<DIM, Real>(a, a.idx[b + jj]);
                    rank += (q.x == pk.x && q.y < pk.y) ? 1 : 0;
                }
            }
            if (rank < survivors(k, a.pp.maxpp, a.apply_counts)) {
                const uint32_t dst = fb + (uint32_t)pfx[pk.x] + (uint32_t)rank;
                if (dst < cap) {
                    a.S1.cell[dst] = (uint32_t)c;
                    a.S1.id[dst] = a.S0.id[i];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        if constexpr (std::is_same<Real, double>::value)
                            str<double>(a.S1.x[d], dst, ldr<double>(a.T.x[d], i));
                        str<Real>(a.S1.xi[d], dst, ldr<Real>(a.T.xi[d], i));
                        str<Real>(a.S1.v[d], dst, ldr<Real>(a.T.v[d], i));
                    }
                } else {
                    err |= ERR_CAPACITY;
                }
            } else {
                removed++;
            }
        }
        // new particles in the empty parts
        if (a.apply_counts) {
            for (int p = lane; p < npe; p += 32) {
                int idx[3] = {0, 0, 0};
                if (!real_part<DIM>(p, a.pp, idx)) continue;
                if (survivors(cnt[p], a.pp.maxpp, 1) != 0) continue;
                const uint32_t dst = fb + (uint32_t)pfx[p];
                if (dst < cap) write_new_particle<DIM, Real>(a, a.S1, dst, (uint32_t)c, idx, id0 + sb + (uint32_t)spfx[p] + 1);
                else err |= ERR_CAPACITY;
            }
        }
        __syncwarp();
        const uint32_t fcount = (uint32_t)run;
        cell_partials<DIM, Real>(a, a.S1, (uint32_t)c, fb, (fb + fcount <= cap) ? fcount : 0, lane);
    }
    warp_count(&a.stats->removed, removed);
    err = __reduce_or_sync(0xffffffffu, err);
    if (lane == 0 && err) atomicOr(&a.stats->error_flags, err);
}

// Partials of the current sorted state (after seeding or an upload).
template <int DIM, typename Real>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_partials(StepArgs a, const uint32_t* cell_start)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x * CELL_WARPS + warp; c < a.mesh.nC; c += gridDim.x * CELL_WARPS) {
        const uint32_t b = cell_start[c], e = cell_start[c + 1];
        cell_partials<DIM, Real>(a, a.S0, (uint32_t)c, b, e - b, lane);
    }
}

// Standalone velocity correction of the sorted state (when no move follows).
template <int DIM, typename Real>
__global__ void k_correct(StepArgs a)
{
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    const uint32_t n = (uint32_t)a.stats->n_particles;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = a.S0.cell[i];
        if (c >= (uint32_t)a.mesh.nC) continue;
        Real xi[DIM], N[NV], corr[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xi[d] = ldr<Real>(a.S0.xi[d], i);
            corr[d] = Real(0);
        }
        if constexpr (std::is_same<Real, double>::value) shape64<DIM>(xi, N);
        else shape32<DIM>(xi, N);
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) {
            const int32_t dof = __ldg(a.mesh.cd + (size_t)c * NV + iv);
#pragma unroll
            for (int d = 0; d < DIM; ++d)
                corr[d] = corr[d] + N[iv] * __ldg(reinterpret_cast<const Real*>(a.dVaos) + (size_t)dof * VS + d);
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) str<Real>(a.S0.v[d], i, ldr<Real>(a.S0.v[d], i) + corr[d]);
    }
}

// DoF gather: V_d = sum num_d / sum den over the cells sharing the DoF, in
// ascending cell order, FP64 sums and division (0/0 -> NaN as the reference,
// or the kept input value under empty_dof_policy 1).
template <int DIM, typename PReal>
__global__ void k_gather(StepArgs a, int keep_empty)
{
    constexpr int NV = 1 << DIM, PW = Dims<DIM>::PW;
    const PReal* P = reinterpret_cast<const PReal*>(a.partials);
    unsigned long long nan_dofs = 0;
    for (int dof = blockIdx.x * blockDim.x + threadIdx.x; dof < a.mesh.nD; dof += gridDim.x * blockDim.x) {
        double num[DIM], den = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) num[d] = 0.0;
        const int32_t b = __ldg(a.mesh.d2c_off + dof), e = __ldg(a.mesh.d2c_off + dof + 1);
        for (int32_t k = b; k < e; ++k) {
            const int32_t ent = __ldg(a.mesh.d2c_ent + k);
            const PReal* q = P + (size_t)(ent / NV) * PW + (ent % NV) * 4;
#pragma unroll
            for (int d = 0; d < DIM; ++d) num[d] = num[d] + (double)q[d];
            den = den + (double)q[DIM];
        }
        if (den == 0.0) nan_dofs++;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            double r = num[d] / den;
            if (den == 0.0 && keep_empty) r = a.Vkeep[(size_t)d * a.mesh.nD + dof];
            a.Vout[(size_t)d * a.mesh.nD + dof] = r;
        }
    }
    nan_dofs = warp_sum_u64(nan_dofs);
    if ((threadIdx.x & 31) == 0 && nan_dofs) atomicAdd(&a.stats->nan_dofs, nan_dofs);
}

// Global positions of the FP32 form for output: x = F(xi) in FP64.
template <int DIM>
__global__ void k_positions32(StepArgs a, double* xout)
{
    const uint32_t n = (uint32_t)a.stats->n_particles;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = a.S0.cell[i];
        double X[1 << DIM][DIM], xi[DIM], x[DIM];
        if (c >= (uint32_t)a.mesh.nC) continue;
        load_cell64<DIM>(a.mesh.cellX, c, X);
#pragma unroll
        for (int d = 0; d < DIM; ++d) xi[d] = (double)ldr<float>(a.S0.xi[d], i);
        fwd64<DIM>(X, xi, x);
#pragma unroll
        for (int d = 0; d < DIM; ++d) xout[(size_t)i * DIM + d] = x[d];
    }
}

}  // namespace pfem2
