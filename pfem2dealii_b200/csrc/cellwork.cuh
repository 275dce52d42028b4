// Per-cell kernels: seeding, count correction with the new layout,
// projection partial sums and the DoF gather.
//
// Count correction (check_particle_distribution,
// src/pfem2particlehandler.cpp:356-410) depends on per-(cell, part) counts
// only: a part keeps min(count, max+1) particles, here the ones with the
// smallest key(id), and every real part left without particles in a cell
// that had any gets one new particle at its centre.  New ids continue the
// running count in (cell ascending, part x-major) order, the order in which
// the reference hands them out.
//
// Layout after a step: cells in ascending order; inside a cell the particles
// that stayed (in their previous order), then the ones that moved in (by
// key), then the new ones (by part).  Each cell owns `count + new` slots,
// known from the move's per-cell count and part occupancy before the write
// pass starts; a cell whose over-full parts lose particles leaves that many
// empty slots (cell = HOLE) at the end of its range.  The layout and every
// floating-point sum taken over it are deterministic.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "geom32.cuh"
#include "geom64.cuh"
#include "staging.cuh"

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

// Velocity interpolation at xi from the cell's vertex velocities (FP64 form).
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

// seed_particles (:43-109): npart particles per owned cell, cell-major, parts
// x-major; ids by the global (cell, part) index, so a partitioned run hands
// out the ids of an unpartitioned one.  Cells outside [cbeg, cend) get empty
// ranges.
template <int DIM, typename Real>
__global__ void k_seed(StepArgs a, uint32_t* cell_start)
{
    const uint32_t cb = (uint32_t)a.cbeg, ce = (uint32_t)a.cend;
    const uint32_t total = (ce - cb) * a.pp.npart;
    const uint32_t id0 = a.stats->next_id + cb * a.pp.npart;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t c = cb + t / a.pp.npart;
        const int k = (int)(t % a.pp.npart);
        int idx[3];
        part_digits<DIM>(k, a.pp, idx);
        Real xi[DIM], v[DIM];
        new_particle<DIM, Real>(a, a.S0, t, c, idx, id0 + t + 1, xi, v);
        if (k == 0) cell_start[c] = t;
        if (a.chunk_first && t % ADV_CH == 0) a.chunk_first[t / ADV_CH] = c;
    }
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < (uint32_t)a.mesh.nC; c += gridDim.x * blockDim.x)
        if (c < cb || c >= ce) cell_start[c] = c < cb ? 0u : total;
    if (blockIdx.x == 0 && threadIdx.x == 0) cell_start[a.mesh.nC] = total;
}

__device__ __forceinline__ int survivors(int cnt, int maxpp, int apply)
{
    if (!apply) return cnt;
    if (maxpp < 0) return 0;
    return cnt < maxpp + 1 ? cnt : maxpp + 1;
}

// Does extended part p get a new particle?  (A real part with no survivor in
// a cell that had particles.)
__device__ __forceinline__ bool gets_seed(const StepArgs& a, int p, int cnt, uint32_t n)
{
    if (!a.apply_counts || n == 0 || p >= a.pp.npe) return false;
    if (!((a.pp.realmask[p >> 6] >> (p & 63)) & 1ull)) return false;
    return survivors(cnt, a.pp.maxpp, 1) == 0;
}

// ---------------------------------------------------------------------------
// Projection partials: per cell and local vertex iv, sum_p N_iv v_p and
// sum_p N_iv (project_particle_fields :191-199 restricted to one cell), in
// the cell's particle order.  Each lane writes one particle's 4*NV terms as a
// row of a per-warp shared array; lane e then adds column e row by row
// (FP32: Kahan-compensated).  Entry e = iv*4 + comp, comp = DIM is the weight.
// ---------------------------------------------------------------------------

// Row stride of the partial-row array: 36 keeps rows 16-byte aligned (vector
// stores) and the column reads (lane e reads entry e of row r) conflict-free.
constexpr int TRW = 36;

template <typename Real>
struct PartialAcc {
    Real s = Real(0), c = Real(0);
};

template <int DIM, typename Real>
__device__ __forceinline__ void partial_row(Real (*tr)[TRW], int row, const Real* xi, const Real* v)
{
    constexpr int NV = 1 << DIM;
    Real N[NV];
    if constexpr (std::is_same<Real, double>::value) shape64<DIM>(xi, N);
    else shape32<DIM>(xi, N);
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
        if constexpr (std::is_same<Real, float>::value) {
            float4 t;
            t.x = N[iv] * v[0];
            t.y = N[iv] * v[1];
            t.z = DIM == 3 ? N[iv] * v[DIM - 1] : N[iv];
            t.w = DIM == 3 ? N[iv] : 0.0f;
            *reinterpret_cast<float4*>(&tr[row][iv * 4]) = t;
        } else {
#pragma unroll
            for (int d = 0; d < DIM; ++d) tr[row][iv * 4 + d] = N[iv] * v[d];
            tr[row][iv * 4 + DIM] = N[iv];
            if (DIM == 2) tr[row][iv * 4 + 3] = 0.0;
        }
    }
}

// Column sums of up to 32 partial rows into acc (lane = column).  FP64:
// the rows in order, as the oracle adds them.  FP32: a pairwise tree over the
// 32 rows (empty rows read as 0), then one compensated add into acc.
template <int DIM, typename Real>
__device__ __forceinline__ void partial_sum_rows(Real (*tr)[TRW], int rows, int lane, PartialAcc<Real>& acc)
{
    constexpr int PW = Dims<DIM>::PW;
    if (lane < PW) {
        if constexpr (std::is_same<Real, double>::value) {
            for (int r = 0; r < rows; ++r) acc.s = acc.s + tr[r][lane];
        } else {
            float t[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) t[r] = r < rows ? tr[r][lane] : 0.0f;
#pragma unroll
            for (int w = 16; w >= 1; w >>= 1)
#pragma unroll
                for (int r = 0; r < w; ++r) t[r] = t[r] + t[r + w];
            const float y = t[0] - acc.c;
            const float s = acc.s + y;
            acc.c = (s - acc.s) - y;
            acc.s = s;
        }
    }
}

template <int DIM, typename Real>
__device__ __forceinline__ void store_partial(const StepArgs& a, uint32_t c, const PartialAcc<Real>& acc, int lane)
{
    constexpr int PW = Dims<DIM>::PW;
    if (lane < PW) reinterpret_cast<Real*>(a.partials)[(size_t)c * PW + lane] = acc.s - acc.c;
}

// Partials of the particles in slots [b, b+count) of a state, in order
// (empty slots contribute nothing).
template <int DIM, typename Real>
__device__ __forceinline__ void partials_of_range(const StepArgs& a, const PartState& S, uint32_t c, uint32_t b,
                                                  uint32_t count, Real (*tr)[TRW], int lane)
{
    PartialAcc<Real> acc;
    for (uint32_t base = 0; base < count; base += 32) {
        const uint32_t j = base + lane;
        const bool valid = j < count && S.cell[b + j] != HOLE;
        Real xi[DIM], v[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xi[d] = valid ? ldr<Real>(S.xi[d], b + j) : Real(0);
            v[d] = valid ? ldr<Real>(S.v[d], b + j) : Real(0);
        }
        const int rows = count - base < 32 ? (int)(count - base) : 32;
        if (valid) {
            partial_row<DIM, Real>(tr, lane, xi, v);
        } else if (lane < rows) {  // an empty slot adds nothing
#pragma unroll
            for (int k = 0; k < Dims<DIM>::PW; ++k) tr[lane][k] = Real(0);
        }
        __syncwarp();
        partial_sum_rows<DIM, Real>(tr, rows, lane, acc);
        __syncwarp();
    }
    store_partial<DIM, Real>(a, c, acc, lane);
}

// FP32 cells of at most 32 particles, one per lane (lanes without a particle
// add zeros): the first level of the pairwise tree, rows u + (u + 16), is
// taken through one shuffle instead of shared memory.  Lane u < 16 keeps the
// entries of the vertices whose highest reference-coordinate bit is clear,
// lane u + 16 those with it set, and receives them from its partner, so each
// entry crosses the warp once and 16 rows of PW entries are staged; the
// tree's other levels and the compensated add follow.  Shape values and
// products are those of partial_row (N = (x0 factor * x1 factor) * x2 factor).
template <int DIM>
__device__ __forceinline__ void partial_pairs32(float (*tr)[TRW], bool active, const float* xi, const float* v,
                                                int lane, PartialAcc<float>& acc)
{
    constexpr int NV = 1 << DIM, H = NV / 2, PW = Dims<DIM>::PW;
    const bool hi = lane >= 16;
    float x[DIM], w[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        x[d] = active ? xi[d] : 0.0f;
        w[d] = active ? v[d] : 0.0f;
    }
    float lowN[H];  // products of the factors below the highest direction
#pragma unroll
    for (int k = 0; k < H; ++k) {
        float n = (k & 1) ? x[0] : 1.0f - x[0];
        if (DIM > 2) n *= ((k >> 1) & 1) ? x[1] : 1.0f - x[1];
        lowN[k] = n;
    }
    // a lane without a particle adds nothing (its shape values are zero too)
    const float top = x[DIM - 1], bot = 1.0f - x[DIM - 1];
    const float fk = active ? (hi ? top : bot) : 0.0f, fs = active ? (hi ? bot : top) : 0.0f;
    float keep[4 * H];
#pragma unroll
    for (int k = 0; k < H; ++k) {
        const float nk = lowN[k] * fk, ns = lowN[k] * fs;
        float e[4], f[4];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            e[d] = nk * w[d];
            f[d] = ns * w[d];
        }
        e[DIM] = nk;
        f[DIM] = ns;
        if (DIM == 2) e[3] = f[3] = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) keep[4 * k + j] = e[j] + __shfl_xor_sync(0xffffffffu, f[j], 16);
    }
    const int row = lane & 15, col0 = hi ? 4 * H : 0;
#pragma unroll
    for (int k = 0; k < H; ++k)
        *reinterpret_cast<float4*>(&tr[row][col0 + 4 * k]) =
            make_float4(keep[4 * k], keep[4 * k + 1], keep[4 * k + 2], keep[4 * k + 3]);
    __syncwarp();
    if (lane < PW) {
        float t[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) t[r] = tr[r][lane];
#pragma unroll
        for (int wd = 8; wd >= 1; wd >>= 1)
#pragma unroll
            for (int r = 0; r < wd; ++r) t[r] = t[r] + t[r + wd];
        const float y = t[0] - acc.c;
        const float sm = acc.s + y;
        acc.c = (sm - acc.s) - y;
        acc.s = sm;
    }
}

// ---------------------------------------------------------------------------
// Write pass.  A warp takes CHC consecutive cells; their old ranges are
// contiguous, so the stayers' data (key, id, xi, v[, x]) of the whole chunk
// is loaded at once into shared memory (many independent loads in flight);
// arrivals are gathered from their slots.
// ---------------------------------------------------------------------------

template <int DIM, typename Real>
struct WrCfg {
    static constexpr bool HX = std::is_same<Real, double>::value;
    static constexpr int CHC = WR_CHC;   // cells per chunk on affine meshes
    static constexpr int CHC_UNEVEN = 2; // on other meshes (cells differ more in work)
    static constexpr int UCAP = 128;     // staged particles per chunk
};

template <int DIM, typename Real>
struct __align__(16) WrWarp {
    static constexpr int UCAP = WrCfg<DIM, Real>::UCAP;
    static constexpr bool HX = WrCfg<DIM, Real>::HX;
    uint32_t key[UCAP];
    uint32_t id[UCAP];
    Real xi[DIM][UCAP];
    Real v[DIM][UCAP];
    Real x[HX ? DIM : 1][HX ? UCAP : 4];
    int cnt[NPE_MAX];
    Real tr[32][TRW];
    uint64_t bar;  // completion of the chunk's bulk copies
};

template <int DIM, typename Real>
struct PData {
    uint32_t i, id;
    Real xi[DIM], v[DIM];
    Real x[std::is_same<Real, double>::value ? DIM : 1];
};

template <int DIM, typename Real>
__device__ __forceinline__ void load_global(const StepArgs& a, uint32_t i, PData<DIM, Real>& p)
{
    p.i = i;
    p.id = a.S0.id[i];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        p.xi[d] = ldr<Real>(a.T.xi[d], i);
        p.v[d] = ldr<Real>(a.T.v[d], i);
        if constexpr (std::is_same<Real, double>::value) p.x[d] = ldr<double>(a.T.x[d], i);
    }
}

template <int DIM, typename Real>
__device__ __forceinline__ void load_stage(const WrWarp<DIM, Real>& w, uint32_t u, uint32_t i, PData<DIM, Real>& p)
{
    p.i = i;
    p.id = w.id[u];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        p.xi[d] = w.xi[d][u];
        p.v[d] = w.v[d][u];
        if constexpr (std::is_same<Real, double>::value) p.x[d] = w.x[d][u];
    }
}

template <int DIM, typename Real>
__device__ __forceinline__ void store_particle(const StepArgs& a, uint32_t dst, uint32_t c, const PData<DIM, Real>& p)
{
    a.S1.cell[dst] = c;
    a.S1.id[dst] = p.id;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        str<Real>(a.S1.xi[d], dst, p.xi[d]);
        str<Real>(a.S1.v[d], dst, p.v[d]);
        if constexpr (std::is_same<Real, double>::value) str<double>(a.S1.x[d], dst, p.x[d]);
    }
}

// The k-th arrival of cell c: one of its ARRCAP slots, or further down the
// overflow list (walked from its head; bounded by the capacity).
__device__ __forceinline__ uint32_t arrival(const StepArgs& a, uint32_t c, uint32_t k, uint32_t h)
{
    if (k < (uint32_t)ARRCAP) return a.carrs[(size_t)c * ARRCAP + k];
    uint32_t p = h;
    for (uint32_t t = ARRCAP; t < k && p != LOST && t < a.capacity; ++t) p = a.next[p];
    return p;
}

__device__ __forceinline__ void reset_cell(const StepArgs& a, uint32_t c, int lane)
{
    if (lane == 0) {
        a.ccount[c] = 0;
        a.carr[c] = 0;
        a.head[c] = LOST;
    }
    if (lane < a.pp.occw) a.cocc[(size_t)c * a.pp.occw + lane] = 0ull;
}

// Empty slots [from, to) of a cell's range.
__device__ __forceinline__ void write_holes(const StepArgs& a, uint32_t from, uint32_t to, int lane)
{
    for (uint32_t j = from + lane; j < to; j += 32)
        if (j < a.capacity) a.S1.cell[j] = HOLE;
}

// New particles of one cell: the k-th seeded part (in part order) goes to
// slot base + k and gets id id0 + sb + k + 1.  With tr, its partial row is
// written at row0 + k.  Returns the number of new particles.
template <int DIM, typename Real>
__device__ __forceinline__ uint2 write_seeds(const StepArgs& a, uint32_t c, const int* cnt, uint32_t n, uint32_t base,
                                          uint32_t id0, uint32_t sb, Real (*tr)[TRW], int row0, int lane)
{
    uint32_t done = 0, err = 0;
    for (int p0 = 0; p0 < a.pp.npe; p0 += 32) {
        const int p = p0 + lane;
        const bool sf = p < a.pp.npe && gets_seed(a, p, cnt[p < a.pp.npe ? p : 0], n);
        const unsigned m = __ballot_sync(0xffffffffu, sf);
        if (sf) {
            const uint32_t k = done + __popc(m & ((1u << lane) - 1u));
            const uint32_t dst = base + k;
            int idx[3] = {0, 0, 0};
            real_part<DIM>(p, a.pp, idx);
            Real xi[DIM], v[DIM];
            if (dst < a.capacity) {
                new_particle<DIM, Real>(a, a.S1, dst, c, idx, id0 + sb + k + 1, xi, v);
                if (tr && row0 + (int)k < 32) partial_row<DIM, Real>(tr, row0 + (int)k, xi, v);
            } else {
                err |= ERR_CAPACITY;
            }
        }
        done += __popc(m);
    }
    return make_uint2(done, err);
}

// General path of one cell (any particle count).  Per-element data goes to
// the cell's own slot range of the scratch array; survivors and positions
// are found by counting.  Order: stayers by slot, arrivals by key, new
// particles by part -- the same as the fast path.
template <int DIM, typename Real>
__device__ uint2 write_cell_general(const StepArgs& a, WrWarp<DIM, Real>& w, uint32_t c, uint32_t s0,
                                                 uint32_t L, uint32_t na, uint32_t h, uint32_t off, uint32_t ub,
                                                 uint32_t nseed_expect, uint32_t sb, uint32_t id0, int lane)
{
    uint32_t removed = 0, err = 0;
    int* cnt = w.cnt;
    uint4* G = a.gscr + off;  // element -> (particle index, part, key, flags: 1 stayer, 2 survivor)
    const int npe = a.pp.npe;
    for (int p = lane; p < npe; p += 32) cnt[p] = 0;
    __syncwarp();
    if (off + ub > a.capacity) return make_uint2(0u, ERR_CAPACITY);
    // stayers: elements 0..ns-1 in slot order
    uint32_t ns = 0;
    for (uint32_t base = 0; base < L; base += 32) {
        const uint32_t j = base + lane;
        const bool stay = j < L && a.key[s0 + j] == c;
        const unsigned m = __ballot_sync(0xffffffffu, stay);
        if (stay) {
            const uint32_t i = s0 + j, e = ns + __popc(m & ((1u << lane) - 1u));
            Real xi[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = ldr<Real>(a.T.xi[d], i);
            const int pe = ext_part<DIM, Real>(xi, a.pp);
            if (e < ub) G[e] = make_uint4(i, (uint32_t)pe, key_of(a.S0.id[i], a.pp.seed), 1u);
            atomicAdd(cnt + pe, 1);
        }
        ns += __popc(m);
    }
    // arrivals: elements ns.. (slots lane-parallel; the overflow list walked by all lanes)
    uint32_t t = 0, p = h;
    for (; t < na && t < a.capacity; ++t) {
        uint32_t i;
        if (t < (uint32_t)ARRCAP) {
            i = a.carrs[(size_t)c * ARRCAP + t];
        } else {
            if (p == LOST) break;
            i = p;
            p = a.next[p];
        }
        if ((t & 31u) == (uint32_t)lane) {
            Real xi[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = ldr<Real>(a.T.xi[d], i);
            const int pe = ext_part<DIM, Real>(xi, a.pp);
            if (ns + t < ub) G[ns + t] = make_uint4(i, (uint32_t)pe, key_of(a.S0.id[i], a.pp.seed), 0u);
            atomicAdd(cnt + pe, 1);
        }
    }
    const uint32_t n = ns + t;
    __syncwarp();
    __threadfence_block();
    if (n > ub) return make_uint2(0u, ERR_COUNT_UB);
    // survivors: rank by key inside the part
    uint32_t nsurv = 0;
    for (uint32_t e = lane; e < n; e += 32) {
        const uint4 g = G[e];
        const int k = cnt[g.y];
        int rank = 0;
        if (a.apply_counts && k > a.pp.maxpp + 1)
            for (uint32_t m = 0; m < n; ++m) {
                const uint4 o = G[m];
                rank += (o.y == g.y && o.z < g.z) ? 1 : 0;
            }
        if (rank < survivors(k, a.pp.maxpp, a.apply_counts)) {
            G[e].w = g.w | 2u;
            nsurv++;
        } else {
            removed++;
        }
    }
    nsurv = __reduce_add_sync(0xffffffffu, nsurv);
    __syncwarp();
    __threadfence_block();
    // positions: survivors before in (stayers by slot | arrivals by key) order
    for (uint32_t e = lane; e < n; e += 32) {
        const uint4 g = G[e];
        if (!(g.w & 2u)) continue;
        const bool gs = g.w & 1u;
        uint32_t pos = 0;
        for (uint32_t m = 0; m < n; ++m) {
            const uint4 o = G[m];
            if (!(o.w & 2u)) continue;
            const bool os = o.w & 1u;
            pos += ((os && !gs) || (os && gs && o.x < g.x) || (!os && !gs && o.z < g.z)) ? 1u : 0u;
        }
        PData<DIM, Real> pd;
        load_global<DIM, Real>(a, g.x, pd);
        store_particle<DIM, Real>(a, off + pos, c, pd);
    }
    const uint2 sd = write_seeds<DIM, Real>(a, c, cnt, n, off + nsurv, id0, sb, nullptr, 0, lane);
    err |= sd.y;
    const uint32_t nseed = sd.x;
    const uint32_t fin = nsurv + nseed;
    if (nseed != nseed_expect) err |= ERR_COUNT;
    if (fin > ub) err |= ERR_COUNT_UB;
    write_holes(a, off + fin, off + ub, lane);
    __syncwarp();
    __threadfence_block();
    partials_of_range<DIM, Real>(a, a.S1, c, off, fin, w.tr, lane);
    return make_uint2(removed, err);
}

// Simple cell: no new particles, and no part can hold more than max+1
// particles (the cell's count exceeds its occupied parts by at most max), so
// every particle survives: the stayers in slot order, then the arrivals by
// key.  Stayers and arrivals fit one round of the warp (L + na <= 32).
template <int DIM, typename Real>
__device__ __forceinline__ void write_cell_simple(const StepArgs& a, WrWarp<DIM, Real>& w, uint32_t c, uint32_t s0,
                                                  uint32_t L, uint32_t na, uint32_t h, uint32_t off, uint32_t ub,
                                                  uint32_t S, bool staged, int lane, uint32_t& err)
{
    const uint32_t u = (uint32_t)lane;
    const bool st = u < L && (staged ? w.key[s0 - S + u] : a.key[s0 + u]) == c;
    const bool ar = u >= L && u < L + na;
    const unsigned m = __ballot_sync(0xffffffffu, st);
    const uint32_t ns = __popc(m);
    PData<DIM, Real> pd;
    bool loaded = st;
    uint32_t pos = 0, key = 0xffffffffu;
    if (st) {
        if (staged) load_stage<DIM, Real>(w, s0 - S + u, s0 + u, pd);
        else load_global<DIM, Real>(a, s0 + u, pd);
        pos = __popc(m & ((1u << lane) - 1u));
    } else if (ar) {
        const uint32_t ia = arrival(a, c, u - L, h);
        if (ia < a.capacity) {
            load_global<DIM, Real>(a, ia, pd);
            loaded = true;
            key = key_of(pd.id, a.pp.seed);
        } else {
            err |= ERR_ARRIVAL;
        }
    }
    uint32_t rank = 0;  // of an arrival among the cell's arrivals, by key
    if (na > 1) {
        for (uint32_t t = 0; t < na; ++t) {
            const uint32_t kl = __shfl_sync(0xffffffffu, key, (int)(L + t));
            rank += kl < key ? 1u : 0u;
        }
    }
    if (ar) pos = ns + rank;
    if (st || ar) {
        const uint32_t dst = off + pos;
        if (dst < a.capacity) store_particle<DIM, Real>(a, dst, c, pd);
        else err |= ERR_CAPACITY;
        if constexpr (!std::is_same<Real, float>::value) partial_row<DIM, Real>(w.tr, (int)pos, pd.xi, pd.v);
    }
    const uint32_t fin = ns + na;
    if (fin != ub) err |= ERR_COUNT_UB;
    PartialAcc<Real> acc;
    if constexpr (std::is_same<Real, float>::value) {
        // rows are lanes: stayers in slot order; the arrival of rank r moves
        // to lane L + r, so the sum's order does not depend on the order in
        // which the arrivals were recorded
        int from = lane;
        bool act = st;
        for (uint32_t t = 0; t < na; ++t) {
            const unsigned b = __ballot_sync(0xffffffffu, ar && loaded && rank == t);
            if (u == L + t) {
                from = b ? __ffs(b) - 1 : lane;
                act = b != 0;
            }
        }
        float xs[DIM], vs[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xs[d] = __shfl_sync(0xffffffffu, pd.xi[d], from);
            vs[d] = __shfl_sync(0xffffffffu, pd.v[d], from);
        }
        partial_pairs32<DIM>(w.tr, act, xs, vs, lane, acc);
    } else {
        __syncwarp();
        partial_sum_rows<DIM, Real>(w.tr, (int)fin, lane, acc);
    }
    store_partial<DIM, Real>(a, c, acc, lane);
    reset_cell(a, c, lane);
}

// Fast path of one cell (at most 96 old slots + arrivals and 96 output
// slots), R rounds of the warp: virtual slots u = 32 r + lane, u < L the
// cell's old slots (a stayer where its key is c), L <= u < L + na the
// arrivals.  R = ceil((L + na) / 32), so a cell issues only the rounds it
// fills.
template <int DIM, typename Real, int R>
__device__ __forceinline__ void write_cell_fast(const StepArgs& a, WrWarp<DIM, Real>& w, uint32_t c, uint32_t s0,
                                                uint32_t L, uint32_t na, uint32_t h, uint32_t off, uint32_t ub,
                                                uint32_t nseed_expect, uint32_t sb, uint32_t id0, uint32_t S,
                                                bool staged, int lane, unsigned long long& removed, uint32_t& err)
{
    const uint32_t cap = a.capacity;
    const int apply = a.apply_counts, maxpp = a.pp.maxpp;
    bool is_stay[R];
    unsigned stm[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t u = 32u * r + (uint32_t)lane;
        is_stay[r] = u < L && (staged ? w.key[s0 - S + u] : a.key[s0 + u]) == c;
        stm[r] = __ballot_sync(0xffffffffu, is_stay[r]);
    }
    uint32_t ns = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) ns += __popc(stm[r]);
    const uint32_t n = ns + na;
    PData<DIM, Real> pd[R];
    bool is_arr[R], valid[R];
    int pe[R];
    uint32_t key[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t u = 32u * r + (uint32_t)lane;
        is_arr[r] = u >= L && u < L + na;
        valid[r] = is_stay[r] || is_arr[r];
        pd[r].i = 0;
        pd[r].id = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) pd[r].xi[d] = pd[r].v[d] = Real(0);
        if (is_stay[r]) {
            if (staged) load_stage<DIM, Real>(w, s0 - S + u, s0 + u, pd[r]);
            else load_global<DIM, Real>(a, s0 + u, pd[r]);
        } else if (is_arr[r]) {
            const uint32_t ia = arrival(a, c, u - L, h);
            if (ia < cap) load_global<DIM, Real>(a, ia, pd[r]);
            else err |= ERR_ARRIVAL;
        }
        pe[r] = valid[r] ? ext_part<DIM, Real>(pd[r].xi, a.pp) : 0;
        key[r] = valid[r] ? key_of(pd[r].id, a.pp.seed) : 0xffffffffu;
    }
    int* cnt = w.cnt;
    for (int p = lane; p < a.pp.npe; p += 32) cnt[p] = 0;
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (valid[r]) atomicAdd(cnt + pe[r], 1);
    __syncwarp();
    int kme[R], rank[R];
    unsigned validm[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        kme[r] = valid[r] ? cnt[pe[r]] : 0;
        rank[r] = 0;
        validm[r] = __ballot_sync(0xffffffffu, valid[r]);
    }
    // rank inside an over-full part (by key)
    bool over = false;
#pragma unroll
    for (int r = 0; r < R; ++r) over = over || kme[r] > maxpp + 1;
    if (__any_sync(0xffffffffu, apply && over)) {
#pragma unroll
        for (int r2 = 0; r2 < R; ++r2) {
            for (int l = 0; l < 32; ++l) {
                const int pl = __shfl_sync(0xffffffffu, pe[r2], l);
                const uint32_t kl = __shfl_sync(0xffffffffu, key[r2], l);
                const bool vl = (validm[r2] >> l) & 1u;
#pragma unroll
                for (int r = 0; r < R; ++r) rank[r] += (vl && pl == pe[r] && kl < key[r]) ? 1 : 0;
            }
        }
    }
    // order: stayers (slot order), then arrivals by key
    const unsigned ltm = (1u << lane) - 1u;
    uint32_t seq[R];
    uint32_t before = 0;  // stayers in the earlier rounds
#pragma unroll
    for (int r = 0; r < R; ++r) {
        seq[r] = is_stay[r] ? before + (uint32_t)__popc(stm[r] & ltm) : ns + 32u * r + (uint32_t)lane - L;
        before += (uint32_t)__popc(stm[r]);
    }
    if (na > 1) {
        uint32_t ar[R];
#pragma unroll
        for (int r = 0; r < R; ++r) ar[r] = 0u;
        for (uint32_t t = 0; t < na; ++t) {
            const uint32_t u2 = L + t;
            uint32_t kl = 0u;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t kr = __shfl_sync(0xffffffffu, key[r], (int)(u2 & 31u));
                if ((u2 >> 5) == (uint32_t)r) kl = kr;
            }
#pragma unroll
            for (int r = 0; r < R; ++r) ar[r] += (kl < key[r]) ? 1u : 0u;
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (is_arr[r]) seq[r] = ns + ar[r];
    }
    bool surv[R];
    unsigned survm[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        surv[r] = valid[r] && rank[r] < survivors(kme[r], maxpp, apply);
        survm[r] = __ballot_sync(0xffffffffu, surv[r]);
    }
    uint32_t nsurv = 0, pos[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        nsurv += __popc(survm[r]);
        pos[r] = seq[r];
    }
    if (nsurv != n) {  // removals: survivors before in sequence order
#pragma unroll
        for (int r = 0; r < R; ++r) pos[r] = 0;
#pragma unroll
        for (int r2 = 0; r2 < R; ++r2) {
            for (int l = 0; l < 32; ++l) {
                const uint32_t sl = __shfl_sync(0xffffffffu, seq[r2], l);
                const bool bl = (survm[r2] >> l) & 1u;
#pragma unroll
                for (int r = 0; r < R; ++r) pos[r] += (bl && sl < seq[r]) ? 1u : 0u;
            }
        }
    }
    // partial rows in registers -> shared rows when the cell's final
    // particles fit one row block, else re-read from the new layout
    const bool rows = nsurv + nseed_expect <= 32u;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (surv[r]) {
            const uint32_t dst = off + pos[r];
            if (dst < cap) store_particle<DIM, Real>(a, dst, c, pd[r]);
            else err |= ERR_CAPACITY;
            if (rows) partial_row<DIM, Real>(w.tr, (int)pos[r], pd[r].xi, pd[r].v);
        }
        removed += (valid[r] && !surv[r]) ? 1 : 0;
    }
    uint32_t nseed = 0;
    if (nseed_expect) {
        const uint2 sd = write_seeds<DIM, Real>(a, c, cnt, n, off + nsurv, id0, sb, rows ? w.tr : nullptr,
                                                (int)nsurv, lane);
        nseed = sd.x;
        err |= sd.y;
    }
    const uint32_t fin = nsurv + nseed;
    if (nseed != nseed_expect) err |= ERR_COUNT;
    if (fin > ub) err |= ERR_COUNT_UB;
    write_holes(a, off + fin, off + ub, lane);
    __syncwarp();
    if (rows) {
        PartialAcc<Real> acc;
        partial_sum_rows<DIM, Real>(w.tr, fin < 32u ? (int)fin : 32, lane, acc);
        store_partial<DIM, Real>(a, c, acc, lane);
    } else {
        __threadfence_block();
        partials_of_range<DIM, Real>(a, a.S1, c, off, fin < ub ? fin : ub, w.tr, lane);
    }
    reset_cell(a, c, lane);
}

// BULK: stage each chunk's old slots by bulk copies (meshes whose chunks of
// CHC cells usually fit the stage); else by plain loads (a kernel without the
// bulk-copy code, faster where the chunks are too large to stage anyway).
template <int DIM, typename Real, bool BULK, int CHC>
__global__ void __launch_bounds__(WR_WARPS * 32) k_write(StepArgs a)
{
    pdl_entry();
    constexpr int UCAP = WrCfg<DIM, Real>::UCAP;
    extern __shared__ __align__(16) unsigned char wr_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WrWarp<DIM, Real>& w = reinterpret_cast<WrWarp<DIM, Real>*>(wr_raw)[warp];
    const uint32_t nC = (uint32_t)a.mesh.nC;
    const uint32_t nchunks = (nC + CHC - 1) / CHC;
    const uint32_t id0 = a.stats->next_id;
    const uint32_t cap = a.capacity;
    const int apply = a.apply_counts, maxpp = a.pp.maxpp;
    unsigned long long removed = 0;
    uint32_t err = 0;
    if (BULK && lane == 0) {
        mbar_init(&w.bar, 1);
        mbar_fence_init();
    }
    __syncwarp();
    uint32_t phase = 0;
    bool stage_ok = true;  // cleared for good if a copy ever fails to land in time
    // chunks of cells are handed out one at a time, so that warps that drew
    // cheap chunks take more (cells differ in particles and arrivals)
    while (true) {
        uint32_t ck = 0;
        if (lane == 0) ck = atomicAdd(&a.stats->write_next, 1u);
        ck = __shfl_sync(0xffffffffu, ck, 0);
        if (ck >= nchunks) break;
        const uint32_t c0 = ck * CHC;
        const uint32_t ncell = nC - c0 < (uint32_t)CHC ? nC - c0 : (uint32_t)CHC;
        // chunk headers, one cell per lane
        const uint32_t csl = (uint32_t)lane <= ncell ? a.cs_old[c0 + lane] : 0u;
        uint32_t h_na = 0, h_head = LOST, h_occ = 0;
        unsigned long long h_ub = 0, h_off = 0;
        if ((uint32_t)lane < ncell) {
            h_na = a.carr[c0 + lane];
            h_head = a.head[c0 + lane];
            h_ub = a.cub[c0 + lane];
            h_off = a.coff[c0 + lane];
            for (int q = 0; q < a.pp.occw; ++q) h_occ += __popcll(a.cocc[(size_t)(c0 + lane) * a.pp.occw + q]);
        }
        // the chunk's old slot range [S, E), staged by bulk copies of whole
        // 16-byte pieces [SA, EA) (the capacity is a multiple of 4 slots)
        const uint32_t S = __shfl_sync(0xffffffffu, csl, 0), E = __shfl_sync(0xffffffffu, csl, ncell);
        const uint32_t SA = BULK ? (S & ~3u) : S, EA = BULK ? ((E + 3u) & ~3u) : E;
        bool staged = stage_ok && EA - SA <= (uint32_t)UCAP;
        if constexpr (!BULK) {
            if (staged) {
                for (uint32_t j = lane; j < E - S; j += 32) {
                    const uint32_t i = S + j;
                    w.key[j] = a.key[i];
                    w.id[j] = a.S0.id[i];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        w.xi[d][j] = ldr<Real>(a.T.xi[d], i);
                        w.v[d][j] = ldr<Real>(a.T.v[d], i);
                        if constexpr (WrCfg<DIM, Real>::HX) w.x[d][j] = ldr<double>(a.T.x[d], i);
                    }
                }
            }
        } else if (staged && EA > SA) {
            const uint32_t nb = EA - SA;
            if (lane == 0) {
                fence_proxy_async();  // the previous chunk's reads of the stage come first
                constexpr uint32_t per = 8u + 2u * DIM * sizeof(Real) + (WrCfg<DIM, Real>::HX ? DIM * 8u : 0u);
                mbar_expect_tx(&w.bar, nb * per);
                bulk_g2s(w.key, a.key + SA, nb * 4u, &w.bar);
                bulk_g2s(w.id, a.S0.id + SA, nb * 4u, &w.bar);
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    bulk_g2s(w.xi[d], reinterpret_cast<const Real*>(a.T.xi[d]) + SA, nb * (uint32_t)sizeof(Real),
                             &w.bar);
                    bulk_g2s(w.v[d], reinterpret_cast<const Real*>(a.T.v[d]) + SA, nb * (uint32_t)sizeof(Real),
                             &w.bar);
                    if constexpr (WrCfg<DIM, Real>::HX)
                        bulk_g2s(w.x[d], reinterpret_cast<const double*>(a.T.x[d]) + SA, nb * 8u, &w.bar);
                }
            }
            const uint32_t par = phase;
            phase ^= 1u;
            if (!__all_sync(0xffffffffu, mbar_wait(&w.bar, par))) {
                // give the copy one more bounded wait, then stop staging
                err |= ERR_TIMEOUT;
                mbar_wait(&w.bar, par);
                staged = false;
                stage_ok = false;
            }
        }
        __syncwarp();
        for (uint32_t jc = 0; jc < ncell; ++jc) {
            const uint32_t c = c0 + jc;
            const uint32_t s0 = __shfl_sync(0xffffffffu, csl, jc);
            const uint32_t L = __shfl_sync(0xffffffffu, csl, jc + 1) - s0;
            const uint32_t na = __shfl_sync(0xffffffffu, h_na, jc);
            const uint32_t h = __shfl_sync(0xffffffffu, h_head, jc);
            const unsigned long long ubw = __shfl_sync(0xffffffffu, h_ub, jc);
            const unsigned long long ofw = __shfl_sync(0xffffffffu, h_off, jc);
            const uint32_t ub = (uint32_t)ubw, nseed_expect = (uint32_t)(ubw >> 32);
            const uint32_t off = (uint32_t)ofw, sb = (uint32_t)(ofw >> 32);
            if (lane == 0) {
                a.cs_new[c] = off;
                // the advect chunks that start in this cell's new range
                if (a.chunk_first)
                    for (uint32_t k = (off + ADV_CH - 1) / ADV_CH; (uint64_t)k * ADV_CH < (uint64_t)off + ub; ++k)
                        a.chunk_first[k] = c;
            }
            const uint32_t occ = __shfl_sync(0xffffffffu, h_occ, jc);
            // count - occupied parts <= max: no part above max + 1 particles
            const bool no_removal = !apply || (maxpp >= 0 && ub - nseed_expect <= occ + (uint32_t)maxpp);
            if (nseed_expect == 0 && no_removal && L + na <= 32u) {
                write_cell_simple<DIM, Real>(a, w, c, s0, L, na, h, off, ub, SA, staged, lane, err);
                __syncwarp();
                continue;
            }
            // Cells beyond 96 particles take the general path.
            if (!(L + na <= 96 && ub <= 96)) {
                const uint2 gr = write_cell_general<DIM, Real>(a, w, c, s0, L, na, h, off, ub, nseed_expect, sb, id0,
                                                               lane);
                removed += gr.x;
                err |= gr.y;
                __syncwarp();
                reset_cell(a, c, lane);
                __syncwarp();
                continue;
            }
            if (L + na > 64)
                write_cell_fast<DIM, Real, 3>(a, w, c, s0, L, na, h, off, ub, nseed_expect, sb, id0, SA, staged, lane,
                                              removed, err);
            else if (L + na > 32)
                write_cell_fast<DIM, Real, 2>(a, w, c, s0, L, na, h, off, ub, nseed_expect, sb, id0, SA, staged, lane,
                                              removed, err);
            else
                write_cell_fast<DIM, Real, 1>(a, w, c, s0, L, na, h, off, ub, nseed_expect, sb, id0, SA, staged, lane,
                                              removed, err);
            __syncwarp();
        }
    }
    warp_count(&a.stats->removed, removed);
    warp_count(&a.stats->step_holes, removed);
    err = __reduce_or_sync(0xffffffffu, err);
    if (lane == 0 && err) atomicOr(&a.stats->error_flags, err);
    // the last warp to finish finalises the step (no waiting: the others
    // have published their counters before counting themselves done)
    unsigned int last = 0;
    if (lane == 0) {
        __threadfence();
        last = atomicAdd(&a.stats->write_done, 1u) == gridDim.x * WR_WARPS - 1 ? 1u : 0u;
        if (last) {
            __threadfence();
            finalize_step(a);
            a.stats->write_done = 0;
            a.stats->write_next = 0;
        }
    }
    (void)last;
}

// Partials of the current state (after seeding or an upload).
template <int DIM, typename Real>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_partials(StepArgs a, const uint32_t* cell_start)
{
    __shared__ __align__(16) Real tr_s[CELL_WARPS][32][TRW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x * CELL_WARPS + warp; c < a.mesh.nC; c += gridDim.x * CELL_WARPS) {
        const uint32_t b = cell_start[c], e = cell_start[c + 1];
        partials_of_range<DIM, Real>(a, a.S0, (uint32_t)c, b, e - b, tr_s[warp], lane);
    }
}

// Standalone velocity correction of the current state (when no move follows).
template <int DIM, typename Real>
__global__ void k_correct(StepArgs a)
{
    const uint32_t n = (uint32_t)a.stats->n_slots;
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

// The 4 values of one (cell, vertex) partial entry (16-byte aligned).
__device__ __forceinline__ void load4(const float* p, float* q)
{
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    q[0] = t.x;
    q[1] = t.y;
    q[2] = t.z;
    q[3] = t.w;
}
__device__ __forceinline__ void load4(const double* p, double* q)
{
    const double2 t0 = __ldg(reinterpret_cast<const double2*>(p));
    const double2 t1 = __ldg(reinterpret_cast<const double2*>(p) + 1);
    q[0] = t0.x;
    q[1] = t0.y;
    q[2] = t1.x;
    q[3] = t1.y;
}

// DoF gather: V_d = sum num_d / sum den over the cells sharing the DoF, in
// ascending cell order, FP64 sums and division (0/0 -> NaN as the reference,
// or the kept input value under empty_dof_policy 1).  Up to 8 cell entries
// are fetched before any is summed; a thread's first DoF's entries (mesh
// data) are fetched before the kernel waits for the write pass.
template <int DIM, typename PReal>
__global__ void k_gather(StepArgs a, int keep_empty)
{
    constexpr int NV = 1 << DIM, PW = Dims<DIM>::PW;
    const int stride = gridDim.x * blockDim.x;
    const int nloop = (a.mesh.nD + stride - 1) / stride * stride;
    const int dof0 = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t b0 = 0, e0 = 0, ent0[8];
    if (dof0 < a.mesh.nD) {
        b0 = __ldg(a.mesh.d2c_off + dof0);
        e0 = __ldg(a.mesh.d2c_off + dof0 + 1);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) ent0[j] = b0 + j < e0 ? __ldg(a.mesh.d2c_ent + b0 + j) : -1;
    pdl_entry();
    const PReal* P = reinterpret_cast<const PReal*>(a.partials);
    unsigned long long nan_dofs = 0;
    for (int dof = dof0; dof < nloop; dof += stride) {
        if (dof >= a.mesh.nD) continue;
        double num[DIM], den = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) num[d] = 0.0;
        const bool first = dof == dof0;
        const int32_t b = first ? b0 : __ldg(a.mesh.d2c_off + dof), e = first ? e0 : __ldg(a.mesh.d2c_off + dof + 1);
        for (int32_t k0 = b; k0 < e; k0 += 8) {
            int32_t ent[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
                ent[j] = first && k0 == b ? ent0[j] : k0 + j < e ? __ldg(a.mesh.d2c_ent + k0 + j) : -1;
            PReal q[8][4];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int32_t en = ent[j] < 0 ? 0 : ent[j];
                load4(P + (size_t)(en / NV) * PW + (en % NV) * 4, q[j]);  // one vector load per entry
                if (ent[j] < 0) q[j][0] = q[j][1] = q[j][2] = q[j][3] = PReal(0);
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (ent[j] < 0) continue;
#pragma unroll
                for (int d = 0; d < DIM; ++d) num[d] = num[d] + (double)q[j][d];
                den = den + (double)q[j][DIM];
            }
        }
        if (den == 0.0) nan_dofs++;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            double r = num[d] / den;
            if (den == 0.0 && keep_empty) r = a.Vkeep[(size_t)d * a.mesh.nD + dof];
            a.Vout[(size_t)d * a.mesh.nD + dof] = r;
            if (a.Vout2) a.Vout2[(size_t)d * a.mesh.nD + dof] = r;
        }
    }
    nan_dofs = warp_sum_u64(nan_dofs);
    if ((threadIdx.x & 31) == 0 && nan_dofs) atomicAdd(&a.stats->nan_dofs, nan_dofs);
}

// Global positions of the FP32 form for output: x = F(xi) in FP64.
template <int DIM>
__global__ void k_positions32(StepArgs a, double* xout)
{
    const uint32_t n = (uint32_t)a.stats->n_slots;
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

// Output packing (output_particle_solution, src/pfem2particlehandler.cpp:
// 218-317, writes positions and velocities as Float32): for the k-th live
// particle (slot[k], in slot order) out[3k..3k+2] = x and
// out[3n + 3k..] = v as floats, x = the FP64 position (FP64 form) or F(xi)
// in FP64 (FP32 form); 2D pads the third component with 0.
template <int DIM, typename Real>
__global__ void k_pack_output(StepArgs a, const uint32_t* __restrict__ slot, uint32_t n, float* __restrict__ out)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = slot[k];
        double x[3] = {0.0, 0.0, 0.0};
        if constexpr (std::is_same<Real, double>::value) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) x[d] = ldr<double>(a.S0.x[d], i);
        } else {
            double X[1 << DIM][DIM], xi[DIM];
            load_cell64<DIM>(a.mesh.cellX, a.S0.cell[i], X);
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = (double)ldr<float>(a.S0.xi[d], i);
            fwd64<DIM>(X, xi, x);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            out[(size_t)3 * k + d] = (float)x[d];
            out[(size_t)3 * n + (size_t)3 * k + d] = d < DIM ? (float)ldr<Real>(a.S0.v[d], i) : 0.0f;
        }
    }
}

}  // namespace pfem2
