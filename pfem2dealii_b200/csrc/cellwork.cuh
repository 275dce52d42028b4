// Per-cell kernels: seeding, count correction with the final sorted layout,
// projection partial sums and the DoF gather.
//
// Count correction (check_particle_distribution,
// src/pfem2particlehandler.cpp:356-410) depends on per-(cell, part) counts
// only: a part keeps min(count, max+1) particles, here the ones with the
// smallest key(id), and every real part left without particles in a cell
// that had any gets one new particle at its centre.  New ids continue the
// running count in (cell ascending, part x-major) order, the order in which
// the reference hands them out.  Output is sorted by (cell, part, key), so
// the layout and every floating-point sum over it are deterministic.
//
// The write pass is one cooperative launch: each block owns a contiguous
// range of cells, decides them (survivors, new particles, final count), adds
// the published totals of the earlier blocks to place its range, then writes
// its cells at their final offsets and sums the projection partials.
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

// Velocity interpolation at xi from the cell's vertex velocities, FP64
// (reference arithmetic) or FP32.
template <int DIM, typename Real>
__device__ __forceinline__ void interp_v(const void* Vc, uint32_t c, const Real* xi, Real* u)
{
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    const Real* p = reinterpret_cast<const Real*>(Vc) + (size_t)c * NV * VS;
    Real N[NV];
    if constexpr (std::is_same<Real, double>::value) shape64<DIM>(xi, N);
    else shape32<DIM>(xi, N);
#pragma unroll
    for (int d = 0; d < DIM; ++d) u[d] = Real(0);
#pragma unroll
    for (int iv = 0; iv < NV; ++iv)
#pragma unroll
        for (int d = 0; d < DIM; ++d) u[d] = u[d] + N[iv] * __ldg(p + iv * VS + d);
}

// A new particle at the centre of part idx of cell c (seed_particles
// :87-104 and check_particle_distribution :390-407): xi = (idx + 1/2) h,
// x = F(xi) (FP64 form), v = V interpolated at xi in FP64 (rounded to the
// form's precision).  Returns xi and v.
template <int DIM, typename Real>
__device__ __forceinline__ void new_particle(const StepArgs& a, const PartState& S, uint32_t dst, uint32_t c,
                                             const int* idx, uint32_t id, Real* xi, Real* v)
{
    double xid[DIM], vd[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        xid[d] = (idx[d] + 0.5) * a.pp.h[d];
        xi[d] = (Real)xid[d];
    }
    velocity_from_dofs<DIM>(a.mesh.cd, a.Vd, a.mesh.nD, c, xid, vd);
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = (Real)vd[d];
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

template <int DIM>
__device__ __forceinline__ void part_digits(int k, const PartParams& pp, int* idx)
{
    idx[2] = 0;
    if (DIM == 2) {
        idx[0] = k / pp.q[1];
        idx[1] = k % pp.q[1];
    } else {
        idx[0] = k / (pp.q[1] * pp.q[2]);
        idx[1] = (k / pp.q[2]) % pp.q[1];
        idx[2] = k % pp.q[2];
    }
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
        int idx[3];
        part_digits<DIM>(k, a.pp, idx);
        Real xi[DIM], v[DIM];
        new_particle<DIM, Real>(a, a.S0, t, c, idx, id0 + t + 1, xi, v);
        if (k == 0) cell_start[c] = t;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cell_start[a.mesh.nC] = total;
}

// Extended part of an advected particle (T arrays) and its removal key.
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

// Ascending bitonic sort of one 64-bit key per lane across the warp.
__device__ __forceinline__ unsigned long long warp_sort(unsigned long long x, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, j);
            const bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
            x = take_min ? (x < y ? x : y) : (x > y ? x : y);
        }
    return x;
}

// ---------------------------------------------------------------------------
// Projection partials: per cell and local vertex iv, sum_p N_iv v_p and
// sum_p N_iv (project_particle_fields :191-199 restricted to one cell), in
// the cell's final particle order.  Each lane writes one particle's 4*NV
// terms as a row of a per-warp shared array; lane e then adds column e row by
// row (FP32: compensated TwoSum).  Entry e = iv*4 + comp, comp = DIM is the
// weight.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e)
{
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

template <typename Real>
struct PartialAcc {
    Real s = Real(0), c = Real(0);
};

template <int DIM, typename Real>
__device__ __forceinline__ void partial_rows(Real (*tr)[33], bool valid, const Real* xi, const Real* v, int rows,
                                             int lane, PartialAcc<Real>& acc)
{
    constexpr int NV = 1 << DIM, PW = Dims<DIM>::PW;
    Real N[NV];
    if constexpr (std::is_same<Real, double>::value) shape64<DIM>(xi, N);
    else shape32<DIM>(xi, N);
    if (lane < rows) {
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) tr[lane][iv * 4 + d] = valid ? N[iv] * v[d] : Real(0);
            tr[lane][iv * 4 + DIM] = valid ? N[iv] : Real(0);
            if (DIM == 2) tr[lane][iv * 4 + 3] = Real(0);
        }
    }
    __syncwarp();
    if (lane < PW) {
        for (int r = 0; r < rows; ++r) {
            const Real t = tr[r][lane];
            if constexpr (std::is_same<Real, double>::value) {
                acc.s = acc.s + t;
            } else {
                float s, e;
                two_sum(acc.s, t, s, e);
                acc.s = s;
                acc.c += e;
            }
        }
    }
    __syncwarp();
}

template <int DIM, typename Real>
__device__ __forceinline__ void store_partial(const StepArgs& a, uint32_t c, const PartialAcc<Real>& acc, int lane)
{
    constexpr int PW = Dims<DIM>::PW;
    if (lane < PW) reinterpret_cast<Real*>(a.partials)[(size_t)c * PW + lane] = acc.s + acc.c;
}

// Partials of particles [b, b+count) of a sorted state, in order.
template <int DIM, typename Real>
__device__ __forceinline__ void partials_of_range(const StepArgs& a, const PartState& S, uint32_t c, uint32_t b,
                                                  uint32_t count, Real (*tr)[33], int lane)
{
    PartialAcc<Real> acc;
    for (uint32_t base = 0; base < count; base += 32) {
        const uint32_t j = base + lane;
        const bool valid = j < count;
        Real xi[DIM], v[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xi[d] = valid ? ldr<Real>(S.xi[d], b + j) : Real(0);
            v[d] = valid ? ldr<Real>(S.v[d], b + j) : Real(0);
        }
        const int rows = count - base < 32 ? (int)(count - base) : 32;
        partial_rows<DIM, Real>(tr, valid, xi, v, rows, lane, acc);
    }
    store_partial<DIM, Real>(a, c, acc, lane);
}

template <typename Real>
struct WriteSmem {
    int cnt[WR_WARPS][NPE_MAX];              // per-part counts (fast path: first 64)
    uint2 kc[WR_WARPS][KEY_CACHE];           // general path: (part, key) cache
    int fpfx[WR_WARPS][64];                  // fast path: first output slot of each part
    Real tr[WR_WARPS][32][33];               // partial rows; general path: part prefixes first
    uint32_t blk_f, blk_s;                   // block totals (particles, new particles)
    unsigned long long pre;                  // seeds << 32 | particles before this block
    uint32_t ws_f[WR_WARPS], ws_s[WR_WARPS]; // block scan workspace
};

__device__ __forceinline__ void store_release_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long load_acquire_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

constexpr unsigned long long BLK_READY = 1ull << 62;
constexpr uint32_t BLK_SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ unsigned long long blk_pack(uint32_t f, uint32_t s)
{
    return BLK_READY | ((unsigned long long)(f & 0x7fffffffu) << 31) | (unsigned long long)(s & 0x7fffffffu);
}

// Warp 0: publish this block's totals, then add up the totals of all earlier
// blocks (all blocks are co-resident: cooperative launch).  Every wait is
// bounded; on time-out the error flag is raised and the partial sum is used
// (the output is then wrong but every write stays in bounds).  Returns
// seeds << 32 | particles before this block.
static __device__ __noinline__ unsigned long long block_prefix(const StepArgs& a, uint32_t b, uint32_t f, uint32_t s,
                                                               int lane)
{
    if (lane == 0) store_release_u64(a.blk_status + b, blk_pack(f, s));
    uint32_t ef = 0, es = 0;
    uint32_t spins = 0;
    bool timed_out = false;
    for (uint32_t base = 0; base < b && !timed_out; base += 32) {
        const uint32_t t = base + lane;
        unsigned long long w = t < b ? load_acquire_u64(a.blk_status + t) : BLK_READY;
        while (__any_sync(0xffffffffu, !(w & BLK_READY))) {
            if (++spins > BLK_SPIN_LIMIT) {
                timed_out = true;
                break;
            }
            __nanosleep(64);
            if (!(w & BLK_READY)) w = load_acquire_u64(a.blk_status + t);
        }
        const bool use = t < b && (w & BLK_READY);
        ef += __reduce_add_sync(0xffffffffu, use ? (uint32_t)((w >> 31) & 0x7fffffffu) : 0u);
        es += __reduce_add_sync(0xffffffffu, use ? (uint32_t)(w & 0x7fffffffu) : 0u);
    }
    if (timed_out && lane == 0) atomicOr(&a.stats->error_flags, ERR_LOOKBACK);
    return ((unsigned long long)es << 32) | ef;
}

// The particles of cell c after the move: those of its old range [s0, s0+L)
// that stayed (key == c), then its arrival list.  Each particle is visited
// by one lane: f(i, ord) with ord = j in the range or L + t on the list.
// The list walk stops after `capacity` nodes (an unreset list can not loop).
template <typename F>
__device__ __forceinline__ void for_each_in_cell(const StepArgs& a, uint32_t c, uint32_t s0, uint32_t L, uint32_t h,
                                                 int lane, F&& f)
{
    for (uint32_t j = lane; j < L; j += 32) {
        const uint32_t i = s0 + j;
        if (a.key[i] == c) f(i, j);
    }
    uint32_t t = 0;
    for (uint32_t p = h; p != LOST && t < a.capacity; p = a.next[p], ++t)
        if ((t & 31u) == (uint32_t)lane) f(p, L + t);
}

// Every particle of the cell in one lane (for the rank loops).
template <typename F>
__device__ __forceinline__ void for_all_in_cell(const StepArgs& a, uint32_t c, uint32_t s0, uint32_t L, uint32_t h,
                                                F&& f)
{
    for (uint32_t j = 0; j < L; ++j) {
        const uint32_t i = s0 + j;
        if (a.key[i] == c) f(i, j);
    }
    uint32_t t = 0;
    for (uint32_t p = h; p != LOST && t < a.capacity; p = a.next[p], ++t) f(p, L + t);
}

// General-path phase 1: per-part counts of one cell (in cnt) and its
// (final, seeds).  Also caches (part, key) pairs by ord below KEY_CACHE.
template <int DIM, typename Real>
__device__ __forceinline__ uint2 count_cell(const StepArgs& a, int* cnt, uint2* kc, uint32_t c, uint32_t s0, uint32_t L,
                                            uint32_t h, int lane)
{
    const int npe = a.pp.npe;
    for (int p = lane; p < npe; p += 32) cnt[p] = 0;
    __syncwarp();
    unsigned nloc = 0;
    for_each_in_cell(a, c, s0, L, h, lane, [&](uint32_t i, uint32_t ord) {
        const uint2 pk = part_key<DIM, Real>(a, i);
        atomicAdd(cnt + pk.x, 1);
        if (ord < KEY_CACHE) kc[ord] = pk;
        nloc++;
    });
    const uint32_t nseg = __reduce_add_sync(0xffffffffu, nloc);
    __syncwarp();
    unsigned surv = 0, seeds = 0;
    for (int p = lane; p < npe; p += 32) {
        const int s = survivors(cnt[p], a.pp.maxpp, a.apply_counts);
        int idx[3];
        surv += s;
        if (a.apply_counts && nseg > 0 && s == 0 && real_part<DIM>(p, a.pp, idx)) seeds++;
    }
    surv = __reduce_add_sync(0xffffffffu, surv);
    seeds = __reduce_add_sync(0xffffffffu, seeds);
    return make_uint2(surv + seeds, seeds);
}

template <int DIM, typename Real>
__device__ __forceinline__ void copy_particle(const StepArgs& a, uint32_t i, uint32_t dst, uint32_t c, Real* xi, Real* v)
{
    a.S1.cell[dst] = c;
    a.S1.id[dst] = a.S0.id[i];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        if constexpr (std::is_same<Real, double>::value) str<double>(a.S1.x[d], dst, ldr<double>(a.T.x[d], i));
        xi[d] = ldr<Real>(a.T.xi[d], i);
        v[d] = ldr<Real>(a.T.v[d], i);
        str<Real>(a.S1.xi[d], dst, xi[d]);
        str<Real>(a.S1.v[d], dst, v[d]);
    }
}

// General-path phase 2 of one cell (any particle count, any part count).
template <int DIM, typename Real>
__device__ void write_cell_general(const StepArgs& a, WriteSmem<Real>& sm, int warp, uint32_t c, uint32_t s0,
                                   uint32_t L, uint32_t h, uint32_t fb, uint32_t sb, uint32_t id0, int lane,
                                   unsigned long long& removed, uint32_t& err)
{
    int* cnt = sm.cnt[warp];
    uint2* kc = sm.kc[warp];
    int* pfx = reinterpret_cast<int*>(&sm.tr[warp][0][0]);
    int* spfx = pfx + NPE_MAX;
    const int npe = a.pp.npe;
    const uint2 fs = count_cell<DIM, Real>(a, cnt, kc, c, s0, L, h, lane);
    bool has_any = false;
    for (int p = lane; p < npe; p += 32) has_any = has_any || cnt[p] > 0;
    has_any = __any_sync(0xffffffffu, has_any);
    int run = 0, srun = 0;
    for (int base = 0; base < npe; base += 32) {
        const int p = base + lane;
        int fc = 0, sf = 0;
        if (p < npe) {
            const int s = survivors(cnt[p], a.pp.maxpp, a.apply_counts);
            int idx[3];
            sf = (a.apply_counts && has_any && s == 0 && real_part<DIM>(p, a.pp, idx)) ? 1 : 0;
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
    const uint32_t cap = a.capacity;
    for_each_in_cell(a, c, s0, L, h, lane, [&](uint32_t i, uint32_t ord) {
        const uint2 pk = ord < KEY_CACHE ? kc[ord] : part_key<DIM, Real>(a, i);
        const int k = cnt[pk.x];
        int rank = 0;
        if (k > 1) {
            for_all_in_cell(a, c, s0, L, h, [&](uint32_t i2, uint32_t ord2) {
                const uint2 q = ord2 < KEY_CACHE ? kc[ord2] : part_key<DIM, Real>(a, i2);
                rank += (q.x == pk.x && q.y < pk.y) ? 1 : 0;
            });
        }
        if (rank < survivors(k, a.pp.maxpp, a.apply_counts)) {
            const uint32_t dst = fb + (uint32_t)pfx[pk.x] + (uint32_t)rank;
            Real xi[DIM], v[DIM];
            if (dst < cap) copy_particle<DIM, Real>(a, i, dst, c, xi, v);
            else err |= ERR_CAPACITY;
        } else {
            removed++;
        }
    });
    if (a.apply_counts && has_any) {
        for (int p = lane; p < npe; p += 32) {
            int idx[3] = {0, 0, 0};
            if (!real_part<DIM>(p, a.pp, idx)) continue;
            if (survivors(cnt[p], a.pp.maxpp, 1) != 0) continue;
            const uint32_t dst = fb + (uint32_t)pfx[p];
            Real xi[DIM], v[DIM];
            if (dst < cap) new_particle<DIM, Real>(a, a.S1, dst, c, idx, id0 + sb + (uint32_t)spfx[p] + 1, xi, v);
            else err |= ERR_CAPACITY;
        }
    }
    __syncwarp();
    __threadfence_block();
    const uint32_t fcount = fs.x;
    partials_of_range<DIM, Real>(a, a.S1, c, fb, (fb + fcount <= cap) ? fcount : 0, sm.tr[warp], lane);
}

// The write pass, one cooperative launch per step.  Block b owns the cell
// range [b R, (b+1) R).  Phase 1 decides every cell of the range (survivors,
// new particles, final count, output map) into global scratch; the block then
// publishes its totals, adds those of the earlier blocks and scans its own
// cells into final offsets; phase 2 writes each cell at its offset and sums
// its projection partials in final order.
template <int DIM, typename Real>
__global__ void __launch_bounds__(WR_WARPS * 32) k_write(StepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    WriteSmem<Real>& sm = *reinterpret_cast<WriteSmem<Real>*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int npe = a.pp.npe;
    const bool fast_ok = npe <= 64;
    const unsigned long long realmask = a.pp.realmask;
    const uint32_t id0 = a.stats->next_id;
    const uint32_t cap = a.capacity;
    const int apply = a.apply_counts;
    const int maxpp = a.pp.maxpp;
    const uint32_t nC = (uint32_t)a.mesh.nC;
    const uint32_t R = (nC + gridDim.x - 1) / gridDim.x;
    const uint32_t c0 = blockIdx.x * R < nC ? blockIdx.x * R : nC;
    const uint32_t c1 = c0 + R < nC ? c0 + R : nC;
    unsigned long long removed = 0;
    uint32_t err = 0;
    if (threadIdx.x == 0) {
        sm.blk_f = 0;
        sm.blk_s = 0;
    }
    __syncthreads();
    // ---- phase 1 ----
    for (uint32_t c = c0 + warp; c < c1; c += WR_WARPS) {
        const uint32_t s0 = a.cs_old[c], L = a.cs_old[c + 1] - s0;
        const uint32_t h = a.head[c];
        bool fast = fast_ok && L <= 32;
        uint32_t i = 0, n = 0, fin = 0, nsd = 0;
        unsigned long long seedm = 0;
        if (fast) {
            // stayers of the old range compacted to lanes 0..ns-1, then arrivals
            const bool stay = (uint32_t)lane < L && a.key[s0 + lane] == c;
            const unsigned stm = __ballot_sync(0xffffffffu, stay);
            const uint32_t ns = __popc(stm);
            i = s0 + (__fns(stm, 0, lane + 1) & 31u);
            uint32_t na = 0, p = h;
            while (p != LOST && ns + na < 32) {
                if ((uint32_t)lane == ns + na) i = p;
                ++na;
                p = a.next[p];
            }
            fast = p == LOST;
            n = ns + na;
        }
        if (fast) {
            const bool valid = (uint32_t)lane < n;
            const uint2 pk = valid ? part_key<DIM, Real>(a, i) : make_uint2(0u, 0u);
            int* cnt = sm.cnt[warp];
            int* fpfx = sm.fpfx[warp];
            cnt[lane] = 0;
            cnt[lane + 32] = 0;
            __syncwarp();
            if (valid) atomicAdd(cnt + pk.x, 1);
            __syncwarp();
            int run = 0;
#pragma unroll
            for (int ch = 0; ch < 2; ++ch) {
                const int p = ch * 32 + lane;
                const int k = p < npe ? cnt[p] : 0;
                const int sv = survivors(k, maxpp, apply);
                const bool sf = apply && n > 0 && p < npe && ((realmask >> p) & 1ull) && sv == 0;
                const int fc = sv + (sf ? 1 : 0);
                int inc = fc;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += t;
                }
                fpfx[p] = run + inc - fc;
                run += __shfl_sync(0xffffffffu, inc, 31);
                seedm |= (unsigned long long)__ballot_sync(0xffffffffu, sf) << (32 * ch);
            }
            fin = (uint32_t)run;
            nsd = __popcll(seedm);
            if (fin <= 32) {
                __syncwarp();
                const int kme = valid ? cnt[pk.x] : 0;
                int rank = 0;
                if (__any_sync(0xffffffffu, kme > 1)) {
                    for (int l = 0; l < 32; ++l) {
                        const uint32_t ol = __shfl_sync(0xffffffffu, pk.x, l);
                        const uint32_t kl = __shfl_sync(0xffffffffu, pk.y, l);
                        rank += ((uint32_t)l < n && ol == pk.x && kl < pk.y) ? 1 : 0;
                    }
                }
                const bool surv = valid && rank < survivors(kme, maxpp, apply);
                uint32_t* om = a.comap + (size_t)c * 32;
                if (surv) om[fpfx[pk.x] + rank] = i;
#pragma unroll
                for (int ch = 0; ch < 2; ++ch) {
                    const int p = ch * 32 + lane;
                    if ((seedm >> p) & 1ull) om[fpfx[p]] = 0x80000000u | (uint32_t)p;
                }
                removed += (valid && !surv) ? 1 : 0;
            } else {
                fast = false;
            }
            __syncwarp();
        }
        if (!fast) {
            const uint2 fs = count_cell<DIM, Real>(a, sm.cnt[warp], sm.kc[warp], c, s0, L, h, lane);
            fin = fs.x;
            nsd = fs.y;
            seedm = 0;
        }
        if (lane == 0) {
            a.cfin[c] = fin | (fast ? 0u : 0x80000000u);
            a.cseed[c] = nsd;
            a.cseedm[c] = seedm;
            atomicAdd(&sm.blk_f, fin);
            atomicAdd(&sm.blk_s, nsd);
        }
    }
    __syncthreads();
    // ---- block prefix over the earlier blocks ----
    if (warp == 0) {
        const unsigned long long pre = block_prefix(a, blockIdx.x, sm.blk_f, sm.blk_s, lane);
        if (lane == 0) {
            sm.pre = pre;
            if (blockIdx.x == gridDim.x - 1)
                *a.totals = (((pre >> 32) + sm.blk_s) << 32) | (unsigned long long)((uint32_t)pre + sm.blk_f);
        }
    }
    __syncthreads();
    // ---- final offsets of the range's cells (block scan) ----
    {
        uint32_t runf = (uint32_t)sm.pre, runs = (uint32_t)(sm.pre >> 32);
        for (uint32_t base = c0; base < c1; base += WR_WARPS * 32) {
            const uint32_t c = base + threadIdx.x;
            const uint32_t f = c < c1 ? (a.cfin[c] & 0x7fffffffu) : 0u;
            const uint32_t s = c < c1 ? a.cseed[c] : 0u;
            uint32_t fi = f, si = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t1 = __shfl_up_sync(0xffffffffu, fi, o);
                const uint32_t t2 = __shfl_up_sync(0xffffffffu, si, o);
                if (lane >= o) {
                    fi += t1;
                    si += t2;
                }
            }
            if (lane == 31) {
                sm.ws_f[warp] = fi;
                sm.ws_s[warp] = si;
            }
            __syncthreads();
            uint32_t wf = 0, wsum = 0, tf = 0, ts = 0;
            for (int w = 0; w < WR_WARPS; ++w) {
                if (w < warp) {
                    wf += sm.ws_f[w];
                    wsum += sm.ws_s[w];
                }
                tf += sm.ws_f[w];
                ts += sm.ws_s[w];
            }
            if (c < c1) {
                a.cs_new[c] = runf + wf + fi - f;
                a.cseedoff[c] = runs + wsum + si - s;
            }
            runf += tf;
            runs += ts;
            __syncthreads();
        }
    }
    // ---- phase 2 ----
    for (uint32_t c = c0 + warp; c < c1; c += WR_WARPS) {
        const uint32_t fb = a.cs_new[c], sb = a.cseedoff[c];
        const uint32_t fw = a.cfin[c];
        if (fw & 0x80000000u) {
            const uint32_t s0 = a.cs_old[c], L = a.cs_old[c + 1] - s0;
            write_cell_general<DIM, Real>(a, sm, warp, c, s0, L, a.head[c], fb, sb, id0, lane, removed, err);
        } else {
            const uint32_t fin = fw;
            const bool valid = (uint32_t)lane < fin;
            Real xi[DIM], v[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = v[d] = Real(0);
            if (valid) {
                const uint32_t ent = a.comap[(size_t)c * 32 + lane];
                const uint32_t dst = fb + lane;
                if (dst >= cap) {
                    err |= ERR_CAPACITY;
                } else if (ent & 0x80000000u) {
                    const int p = (int)(ent & 0x7fffffffu);
                    int idx[3] = {0, 0, 0};
                    real_part<DIM>(p, a.pp, idx);
                    const unsigned long long sdm = a.cseedm[c];
                    const uint32_t r = (uint32_t)__popcll(p == 0 ? 0ull : (sdm & ((1ull << p) - 1ull)));
                    new_particle<DIM, Real>(a, a.S1, dst, c, idx, id0 + sb + r + 1, xi, v);
                } else {
                    copy_particle<DIM, Real>(a, ent, dst, c, xi, v);
                }
            }
            PartialAcc<Real> acc;
            partial_rows<DIM, Real>(sm.tr[warp], valid && fb + lane < cap, xi, v, (int)fin, lane, acc);
            store_partial<DIM, Real>(a, c, acc, lane);
        }
        __syncwarp();
        if (lane == 0) a.head[c] = LOST;  // arrival list consumed
    }
    warp_count(&a.stats->removed, removed);
    err = __reduce_or_sync(0xffffffffu, err);
    if (lane == 0 && err) atomicOr(&a.stats->error_flags, err);
}

// Partials of the current sorted state (after seeding or an upload).
template <int DIM, typename Real>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_partials(StepArgs a, const uint32_t* cell_start)
{
    __shared__ Real tr_s[CELL_WARPS][32][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x * CELL_WARPS + warp; c < a.mesh.nC; c += gridDim.x * CELL_WARPS) {
        const uint32_t b = cell_start[c], e = cell_start[c + 1];
        partials_of_range<DIM, Real>(a, a.S0, (uint32_t)c, b, e - b, tr_s[warp], lane);
    }
}

// Standalone velocity correction of the sorted state (when no move follows).
template <int DIM, typename Real>
__global__ void k_correct(StepArgs a)
{
    const uint32_t n = (uint32_t)a.stats->n_particles;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = a.S0.cell[i];
        if (c >= (uint32_t)a.mesh.nC) continue;
        Real xi[DIM], corr[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) xi[d] = ldr<Real>(a.S0.xi[d], i);
        if constexpr (std::is_same<Real, double>::value) {
            interp_v<DIM, Real>(a.dVc, c, xi, corr);
        } else {
            Rec32<DIM> r;
            load_rec32<DIM>(a.dvrec32, c, r);
            eval_poly<DIM>(r.b, xi, corr);
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
    const int stride = gridDim.x * blockDim.x;
    const int nloop = (a.mesh.nD + stride - 1) / stride * stride;
    for (int dof = blockIdx.x * blockDim.x + threadIdx.x; dof < nloop; dof += stride) {
        if (dof >= a.mesh.nD) continue;
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
