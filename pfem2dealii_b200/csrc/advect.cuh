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

#include <type_traits>

#include "common.cuh"
#include "geom64.cuh"
#include "geom32.cuh"
#include "staging.cuh"

namespace pfem2 {

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
// LIN (FP32 form on a mesh whose cells are all affine): the inverse map of a
// candidate is the cell's exact affine inverse xi = A^-1 (p - b), one
// matrix-vector product instead of the Newton iteration; the FP64 form
// always takes the Newton restatement (bit parity with its CPU restatement).
template <int DIM, bool LIN = false>
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
    if constexpr (LIN) {
        // Up to REG_CAND candidates stay in registers: the next one tried is
        // the untried maximum of the dot products, the first of equal ones
        // (the order of the stable descending sort below), selected only
        // when the ones before it have failed.
        if (n <= REG_CAND) {
            double dk[REG_CAND];
            uint32_t ck[REG_CAND];
#pragma unroll
            for (int k = 0; k < REG_CAND; ++k) {
                dk[k] = 0.0;
                ck[k] = c;
                if (k < n) {
                    const double* cd = m.v2c_dirs + (size_t)(b + k) * DIM;
                    double s = __ldg(cd) * vtp[0];
#pragma unroll
                    for (int d = 1; d < DIM; ++d) s = s + __ldg(cd + d) * vtp[d];
                    dk[k] = s;
                    ck[k] = (uint32_t)__ldg(m.v2c_cells + b + k);
                }
            }
            uint32_t tried = 0;
            for (int t = 0; t < n; ++t) {
                int bi = -1;
                double bv = 0.0;
                uint32_t cand = c;
#pragma unroll
                for (int k = 0; k < REG_CAND; ++k) {
                    const bool open = k < n && !((tried >> k) & 1u);
                    if (open && (bi < 0 || dk[k] > bv)) {
                        bi = k;
                        bv = dk[k];
                        cand = ck[k];
                    }
                }
                tried |= 1u << bi;
                if (cand == c) continue;
                double xin[DIM];
                if (inverse_affine64<DIM>(m.aff + (size_t)cand * AFF, xp.v, xin)) {
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
        double xin[DIM];
        int st;
        if constexpr (LIN) {
            st = inverse_affine64<DIM>(m.aff + (size_t)cand * AFF, xp.v, xin);
        } else {
            load_cell64<DIM>(m.cellX, cand, X);
            st = inverse_map64<DIM>(X, m.aff + (size_t)cand * AFF, xp.v, xin);
        }
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

// L1 prefetch of a cell's rows that the FP64 relocation reads (vertex
// coordinates, affine inverse, vertex and DoF ids), issued as soon as the
// cell is known so that the dependent steps after it find them on chip.
__device__ __forceinline__ void prefetch_l1(const void* p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
template <int DIM>
__device__ __forceinline__ void prefetch_cell64(const MeshDev& m, uint32_t c)
{
    constexpr int NV = 1 << DIM, AFF = Dims<DIM>::AFF;
    const double* X = m.cellX + (size_t)c * NV * DIM;
    prefetch_l1(X);
    prefetch_l1(X + NV * DIM - 1);
    if (DIM == 3) prefetch_l1(X + NV * DIM / 2);
    prefetch_l1(m.aff + (size_t)c * AFF);
    prefetch_l1(m.aff + (size_t)c * AFF + AFF - 1);
    prefetch_l1(m.cv + (size_t)c * NV);
    prefetch_l1(m.cd + (size_t)c * NV);
}

// Full FP64 relocation of an FP32-form particle: rebuild x = F(xi) + u dt_p in
// FP64, inverse map in the own cell, then the vertex-patch search of search64
// (LIN: the affine inverse) with two changes of arithmetic that keep its
// choices: the closest vertex maximises (u . p_v) / |p_v| (p_v = vertex -
// previous position) as one product with a reciprocal square root, which
// orders the vertices as the angle cos = (u/|u|) . (p_v/|p_v|) does (a
// positive factor per particle), and the candidates are ordered by their
// centre directions' dot products with the unnormalised vertex->particle
// vector.  Results differ from search64's only where two products tie to
// the last bits.  The vertex ids of the cell are loaded with its coordinates
// and the vertices' cell ranges are prefetched while the angles are
// computed.  A vertex with more than REG_CAND cells takes search64 itself.
template <int DIM, bool LIN = false>
__device__ __noinline__ SearchOut fallback64(const MeshDev m, uint32_t c, Vec<DIM> xo, Vec<DIM> ue, double dtp)
{
    constexpr int NV = 1 << DIM, AFF = Dims<DIM>::AFF;
    int32_t vids[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) vids[v] = __ldg(m.cv + (size_t)c * NV + v);
    double X[NV][DIM], x[DIM], xin[DIM];
    load_cell64<DIM>(m.cellX, c, X);
    fwd64<DIM>(X, xo.v, x);
#pragma unroll
    for (int d = 0; d < DIM; ++d) x[d] = x[d] + ue.v[d] * dtp;
    const int st = LIN ? inverse_affine64<DIM>(m.aff + (size_t)c * AFF, x, xin)
                       : inverse_map64<DIM>(X, m.aff + (size_t)c * AFF, x, xin);
    SearchOut out;
    out.cell = c;
    out.flags = 0;
    out.map_failures = st ? 1u : 0u;
    if (st == 0 && inside_unit<DIM>(xin)) {
        out.flags = SRCH_FOUND | (near_face64<DIM>(xin) ? SRCH_NEAR : 0u);
#pragma unroll
        for (int d = 0; d < DIM; ++d) out.xi[d] = xin[d];
        return out;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) prefetch_l1(m.v2c_off + vids[v]);
    int cvx = 0;
    {
        double old[DIM];
        fwd64<DIM>(X, xo.v, old);
        double best = 0.0;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double ptv[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) ptv[d] = X[v][d] - old[d];
            double dot = ue.v[0] * ptv[0];
#pragma unroll
            for (int d = 1; d < DIM; ++d) dot = dot + ue.v[d] * ptv[d];
            const double ang = dot * rsqrt(norm2_64<DIM>(ptv));
            if (v == 0) best = ang;
            else if (ang > best) {
                best = ang;
                cvx = v;
            }
        }
    }
    int32_t vid = vids[0];
#pragma unroll
    for (int v = 1; v < NV; ++v) vid = cvx == v ? vids[v] : vid;
    double vtp[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) vtp[d] = x[d] - X[cvx][d];
    const int32_t b = __ldg(m.v2c_off + vid);
    const int n = __ldg(m.v2c_off + vid + 1) - b;
    if (n > REG_CAND) {
        Vec<DIM> xp;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xp.v[d] = x[d];
        SearchOut o2 = search64<DIM, LIN>(m, c, xo, ue, xp);
        o2.map_failures += out.map_failures;
        return o2;
    }
    double dk[REG_CAND];
    uint32_t ck[REG_CAND];
#pragma unroll
    for (int k = 0; k < REG_CAND; ++k) {
        dk[k] = 0.0;
        ck[k] = c;
        if (k < n) {
            const double* cd = m.v2c_dirs + (size_t)(b + k) * DIM;
            double sdot = __ldg(cd) * vtp[0];
#pragma unroll
            for (int d = 1; d < DIM; ++d) sdot = sdot + __ldg(cd + d) * vtp[d];
            dk[k] = sdot;
            ck[k] = (uint32_t)__ldg(m.v2c_cells + b + k);
        }
    }
    uint32_t tried = 0;
    for (int t = 0; t < n; ++t) {
        int bi = -1;
        double bv = 0.0;
        uint32_t cand = c;
#pragma unroll
        for (int k = 0; k < REG_CAND; ++k) {
            const bool open = k < n && !((tried >> k) & 1u);
            if (open && (bi < 0 || dk[k] > bv)) {
                bi = k;
                bv = dk[k];
                cand = ck[k];
            }
        }
        tried |= 1u << bi;
        if (cand == c) continue;
        double xc[DIM];
        int sc;
        if constexpr (LIN) {
            sc = inverse_affine64<DIM>(m.aff + (size_t)cand * AFF, x, xc);
        } else {
            load_cell64<DIM>(m.cellX, cand, X);
            sc = inverse_map64<DIM>(X, m.aff + (size_t)cand * AFF, x, xc);
        }
        if (sc) {
            out.map_failures++;
            continue;
        }
        if (inside_unit<DIM>(xc)) {
            out.cell = cand;
            out.flags |= SRCH_FOUND | (near_face64<DIM>(xc) ? SRCH_NEAR : 0u);
#pragma unroll
            for (int d = 0; d < DIM; ++d) out.xi[d] = xc[d];
            return out;
        }
    }
    return out;
}

struct AdvCounters {
    uint32_t lost = 0, map_failures = 0, near_face = 0, searched = 0, fallback = 0;
    uint32_t err = 0;
};

__device__ __forceinline__ void flush_counters(const StepArgs& a, const AdvCounters& k)
{
    warp_count(&a.stats->lost, k.lost);
    warp_count(&a.stats->map_failures, k.map_failures);
    warp_count(&a.stats->near_face, k.near_face);
    warp_count(&a.stats->searched, k.searched);
    warp_count(&a.stats->fallback64, k.fallback);
    const unsigned e = __reduce_or_sync(0xffffffffu, k.err);
    if ((threadIdx.x & 31) == 0 && e) atomicOr(&a.stats->error_flags, e);
}

// Queue a particle whose sub-step s needs the vertex-patch search (FP64
// form) or the FP64 relocation (FP32 form); one atomic per warp.
__device__ __forceinline__ void defer(const StepArgs& a, bool want, uint32_t i, int s)
{
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(a.nxq, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) {
        const uint32_t k = base + __popc(m & ((1u << lane) - 1u));
        if (k < a.capacity) a.xq[k] = make_uint2(i, (uint32_t)s);
    }
}

// Record where particle i ended: its cell, or LOST.  A particle that changed
// cell is entered among its new cell's arrivals (ARRCAP slots, then the
// overflow list); the ones that stayed are found by the write pass in their
// old cell range.
__device__ __forceinline__ void arrive(const StepArgs& a, uint32_t i, uint32_t c, uint32_t c_old, bool alive)
{
    a.key[i] = alive ? c : LOST;
    if (alive && c != c_old) {
        const uint32_t k = atomicAdd(a.carr + c, 1u);
        if (k < (uint32_t)ARRCAP) a.carrs[(size_t)c * ARRCAP + k] = i;
        else a.next[i] = atomicExch(a.head + c, i);
    }
}

// Cell count and part occupancy of the particles a warp finished (pe = the
// particle's extended part): one atomic per distinct cell per word.
__device__ __forceinline__ void count_cells(const StepArgs& a, bool counted, uint32_t c, int pe)
{
    const unsigned am = __ballot_sync(0xffffffffu, counted);
    if (!counted) return;
    const unsigned grp = __match_any_sync(am, c);
    const int leader = __ffs(grp) - 1;
    const bool lead = (int)(threadIdx.x & 31) == leader;
    if (lead) atomicAdd(a.ccount + c, (uint32_t)__popc(grp));
    for (int w = 0; w < a.pp.occw; ++w) {
        const unsigned long long bit = (pe >> 6) == w ? (1ull << (pe & 63)) : 0ull;
        const unsigned lo = __reduce_or_sync(grp, (unsigned)bit);
        const unsigned hi = __reduce_or_sync(grp, (unsigned)(bit >> 32));
        if (lead && (lo | hi)) atomicOr(a.cocc + (size_t)c * a.pp.occw + w, ((unsigned long long)hi << 32) | lo);
    }
}

__device__ __forceinline__ void count_one(const StepArgs& a, uint32_t c, int pe)
{
    atomicAdd(a.ccount + c, 1u);
    atomicOr(a.cocc + (size_t)c * a.pp.occw + (pe >> 6), 1ull << (pe & 63));
}

// One chunk of particle state staged in shared memory by bulk copies.
template <int DIM, typename Real, int CH>
struct AdvStage {
    uint32_t cell[CH];
    Real xi[DIM][CH];
    Real v[DIM][CH];
    Real x[std::is_same<Real, double>::value ? DIM : 1][std::is_same<Real, double>::value ? CH : 4];
};

__device__ __forceinline__ uint32_t round16(uint32_t b) { return (b + 15u) & ~15u; }

// FP32 form: the velocity records (V and V - Vold) of the consecutive cells
// [cfirst, cfirst + ncell) that one chunk's particles lie in (they are
// sorted by cell), staged with the chunk.  ncell = 0: not staged.
template <int DIM>
struct AdvRecStage {
    static constexpr int MAXC = AdvRec<DIM>::MAXC, F4 = Dims<DIM>::REC4;
    float4 v[MAXC][F4];
    float4 dv[MAXC][F4];
    uint32_t cfirst, ncell;
};

// A chunk ticket and, for the record stage, the chunk's first and last
// cells: the cells from the chunk's first cell to the next chunk's first
// cell, as the seed and write passes recorded them.  Thread 0 draws tickets
// ahead and issues these loads early, so their latency passes while the
// block works on earlier chunks.
struct ChunkTicket {
    uint32_t tk, cf, cl;
};

template <int CH>
__device__ __forceinline__ void ticket_cells(const StepArgs& a, uint32_t n, ChunkTicket& t, bool recs)
{
    const uint32_t nchunks = (n + CH - 1) / CH;
    t.cf = 1u;
    t.cl = 0u;  // no range unless loaded
    if (recs && t.tk < nchunks) {
        t.cf = a.chunk_first[t.tk];
        t.cl = t.tk + 1 < nchunks ? a.chunk_first[t.tk + 1] : (uint32_t)a.mesh.nC - 1;
    }
}

// Thread 0: bulk-copy particles [chunk*CH, chunk*CH + cnt) of S0 into stage
// st, and (rs not null) the records of the chunk's cells [t.cf, t.cl] into
// rs (a range that is out of order or too long is not staged; the particles
// then read their records from global memory).
template <int DIM, typename Real, int CH>
__device__ __forceinline__ void stage_chunk(const StepArgs& a, AdvStage<DIM, Real, CH>& st, uint64_t* bar,
                                            const ChunkTicket& t, uint32_t n, AdvRecStage<DIM>* rs = nullptr)
{
    constexpr bool HX = std::is_same<Real, double>::value;
    const uint32_t chunk = t.tk;
    const uint32_t base = chunk * CH;
    const uint32_t cnt = n - base < (uint32_t)CH ? n - base : (uint32_t)CH;
    const uint32_t b4 = round16(cnt * 4u), br = round16(cnt * (uint32_t)sizeof(Real));
    uint32_t cf = 0, nrec = 0;
    if (rs) {
        const uint32_t nC = (uint32_t)a.mesh.nC;
        cf = t.cf;
        if (t.cf <= t.cl && t.cl < nC && t.cl - t.cf < (uint32_t)AdvRecStage<DIM>::MAXC) nrec = t.cl - t.cf + 1;
        rs->cfirst = cf;
        rs->ncell = nrec;
    }
    constexpr uint32_t RB = Dims<DIM>::REC4 * 16u;  // bytes of one cell's record
    const uint32_t recb = nrec * RB * (a.do_correct ? 2u : 1u);
    mbar_expect_tx(bar, b4 + (2 + (HX ? 1 : 0)) * DIM * br + recb);
    if (nrec) {
        bulk_g2s(rs->v, a.vrec32 + (size_t)cf * Dims<DIM>::REC4 * 4, nrec * RB, bar);
        if (a.do_correct) bulk_g2s(rs->dv, a.dvrec32 + (size_t)cf * Dims<DIM>::REC4 * 4, nrec * RB, bar);
    }
    bulk_g2s(st.cell, a.S0.cell + base, b4, bar);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        bulk_g2s(st.xi[d], reinterpret_cast<const Real*>(a.S0.xi[d]) + base, br, bar);
        bulk_g2s(st.v[d], reinterpret_cast<const Real*>(a.S0.v[d]) + base, br, bar);
        if (HX) bulk_g2s(st.x[d], reinterpret_cast<const Real*>(a.S0.x[d]) + base, br, bar);
    }
}

// The chunk loop shared by both forms: double-buffered staging, f(stage,
// buffer, t, i, active) per particle slot (every lane of every warp calls it,
// so warp collectives are allowed inside).  Chunks are handed out one at a
// time from a counter (stats->adv_next, reset when the step is finalised), so
// blocks that drew cheap chunks take more.  A block holds the chunks it works
// on and stages, and thread 0 keeps one more ticket in hand: it loads that
// chunk's cell range and draws the ticket after it while the block works, so
// restaging a buffer waits on no memory.  One barrier per chunk: the reads of
// a buffer end there, and a ticket written after it is read only after the
// next chunk's barrier.
template <int DIM, typename Real, int CH, typename F>
__device__ __forceinline__ void staged_loop(const StepArgs& a, AdvStage<DIM, Real, CH>* st, uint64_t* bar, F&& f,
                                            AdvRecStage<DIM>* rs = nullptr)
{
    __shared__ uint32_t tk[2];
    const uint32_t n = (uint32_t)a.stats->n_slots;
    const uint32_t nchunks = (n + CH - 1) / CH;
    const bool recs = rs != nullptr;
    ChunkTicket hand{0u, 1u, 0u};  // thread 0: the next chunk to stage
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            ChunkTicket t{atomicAdd(&a.stats->adv_next, 1u), 1u, 0u};
            ticket_cells<CH>(a, n, t, recs);
            tk[b] = t.tk;
            if (t.tk < nchunks) stage_chunk<DIM, Real, CH>(a, st[b], &bar[b], t, n, recs ? rs + b : nullptr);
        }
        hand.tk = atomicAdd(&a.stats->adv_next, 1u);
    }
    __syncthreads();
    for (uint32_t it = 0;; ++it) {
        const int sidx = it & 1;
        const uint32_t chunk = tk[sidx];
        if (chunk >= nchunks) break;  // tickets grow: the other buffer holds nothing in flight
        const bool ok = mbar_wait(&bar[sidx], (it >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(&a.stats->error_flags, ERR_TIMEOUT);
            // let the copy still in flight land before the block leaves
            if (tk[sidx ^ 1] < nchunks) mbar_wait(&bar[sidx ^ 1], ((it + 1) >> 1) & 1u);
            return;
        }
        uint32_t after = 0;
        if (threadIdx.x == 0) {  // loads and a ticket in flight while the block works
            ticket_cells<CH>(a, n, hand, recs);
            after = hand.tk < nchunks ? atomicAdd(&a.stats->adv_next, 1u) : 0xffffffffu;
        }
        const uint32_t base = chunk * CH;
        const uint32_t cnt = n - base < (uint32_t)CH ? n - base : (uint32_t)CH;
#pragma unroll 1
        for (uint32_t t = threadIdx.x; t < (uint32_t)CH; t += blockDim.x) f(st[sidx], sidx, t, base + t, t < cnt);
        __syncthreads();
        if (threadIdx.x == 0) {
            tk[sidx] = hand.tk;
            if (hand.tk < nchunks) {
                fence_proxy_async();
                stage_chunk<DIM, Real, CH>(a, st[sidx], &bar[sidx], hand, n, recs ? rs + sidx : nullptr);
            }
            hand.tk = after;
        }
    }
}

// ---------------------------------------------------------------------------
// FP64 form.  Per sub-step (src/pfem2particlehandler.cpp:150-167): u = sum N V,
// x += u dt_p, inverse map in the own cell (:424-431).  A particle that leaves
// its cell is queued with the sub-step index; k_search64 runs the
// vertex-patch search for it and finishes its remaining sub-steps.  Values
// are the same as running everything in one place: every operation is
// repeated in the same order.
// ---------------------------------------------------------------------------

// u = sum_i N_i(xi) V_i with V_i the cell's vertex velocities (a per-step
// copy of V[dof_i], so the values are V's own).
template <int DIM>
__device__ __forceinline__ void velocity64(const double* __restrict__ Vc, uint32_t c, const double* xi, double* u)
{
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    const double* p = Vc + (size_t)c * NV * VS;
    double N[NV];
    shape64<DIM>(xi, N);
#pragma unroll
    for (int d = 0; d < DIM; ++d) u[d] = 0.0;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv)
#pragma unroll
        for (int d = 0; d < DIM; ++d) u[d] = u[d] + N[iv] * __ldg(p + iv * VS + d);
}

// The transport velocity of a sub-step from xi in cell c (vertices X).
// Euler (move_particles :151-159): u(xi).  RK2 (PFEM2GPU_RK2, no reference
// counterpart): u(xi_mid), xi_mid = xi + (h/2) J(xi)^-1 u(xi), the cell's Q1
// field extrapolated where xi_mid leaves the unit cell; a non-positive
// Jacobian determinant keeps u(xi).  The oracle's transport_velocity does the
// same operations in the same order.
template <int DIM, bool RK>
__device__ __forceinline__ void transport64(const StepArgs& a, const double (*X)[DIM], uint32_t c, const double* xi,
                                            double* u)
{
    velocity64<DIM>((const double*)a.Vc, c, xi, u);
    if constexpr (!RK) return;
    double J[DIM][DIM], Ji[DIM][DIM], dl[DIM], xm[DIM];
    jac64<DIM>(X, xi, J);
    const double det = invert64<DIM>(J, Ji);
    if (!(det > 0.0)) return;
    matvec64<DIM>(Ji, u, dl);
    const double half = a.pp.dtp * 0.5;
#pragma unroll
    for (int d = 0; d < DIM; ++d) xm[d] = xi[d] + half * dl[d];
    velocity64<DIM>((const double*)a.Vc, c, xm, u);
}

// Sub-steps s0.. of one FP64 particle starting in cell c; returns the
// sub-step at which it leaves its cell (S if it never does).
template <int DIM, bool RK>
__device__ __forceinline__ int substeps64(const StepArgs& a, uint32_t c, int s0, double* x, double* xi, double* u,
                                          AdvCounters& k)
{
    constexpr int NV = 1 << DIM;
    const MeshDev& m = a.mesh;
    double X[NV][DIM];
    load_cell64<DIM>(m.cellX, c, X);
    int s = s0;
    for (; s < a.pp.S; ++s) {
        transport64<DIM, RK>(a, X, c, xi, u);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const double st = u[d] * a.pp.dtp;
            x[d] = x[d] + st;
        }
        double xin[DIM];
        const int st = inverse_map64<DIM>(X, m.aff + (size_t)c * Dims<DIM>::AFF, x, xin);
        if (st) k.map_failures++;
        if (st == 0 && inside_unit<DIM>(xin)) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = xin[d];
            if (near_face64<DIM>(xin)) k.near_face++;
            continue;
        }
        break;
    }
    return s;
}

constexpr int ADV64_CH = 512;

template <int DIM, bool RK>
__global__ void __launch_bounds__(256) k_advect64(StepArgs a)
{
    pdl_entry();
    extern __shared__ __align__(128) unsigned char adv_raw[];
    __shared__ uint64_t bar[2];
    auto* st = reinterpret_cast<AdvStage<DIM, double, ADV64_CH>*>(adv_raw);
    const MeshDev& m = a.mesh;
    AdvCounters k;
    staged_loop<DIM, double, ADV64_CH>(a, st, bar, [&](AdvStage<DIM, double, ADV64_CH>& sg, int, uint32_t t,
                                                       uint32_t i, bool in) {
        const uint32_t c = in ? sg.cell[t] : HOLE;
        const bool act = c != HOLE && in;
        bool want = false, counted = false;
        int s = 0, pe = 0;
        if (in && c == HOLE) a.key[i] = LOST;
        if (act) {
            double x[DIM], xi[DIM], v[DIM], u[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                x[d] = sg.x[d][t];
                xi[d] = sg.xi[d][t];
                v[d] = sg.v[d][t];
            }
            const bool alive = c < (uint32_t)m.nC;
            if (!alive) k.err |= ERR_BAD_CELL;
            if (alive) {
                if (a.do_correct) {  // :126-138, deltaV = V - Vold per vertex
                    double corr[DIM];
                    velocity64<DIM>((const double*)a.dVc, c, xi, corr);
#pragma unroll
                    for (int d = 0; d < DIM; ++d) v[d] = v[d] + corr[d];
                }
                s = substeps64<DIM, RK>(a, c, 0, x, xi, u, k);
                want = s < a.pp.S;
            }
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                ((double*)a.T.x[d])[i] = x[d];
                ((double*)a.T.xi[d])[i] = xi[d];
                ((double*)a.T.v[d])[i] = v[d];
            }
            if (want) a.key[i] = c;
            else {
                arrive(a, i, c, c, alive);
                if (!alive) k.lost++;
                counted = alive;
                if (counted) pe = ext_part<DIM, double>(xi, a.pp);
            }
        }
        defer(a, want, i, s);
        count_cells(a, counted, c, pe);
    });
    flush_counters(a, k);
}

// Deferred FP64 particles: the search of sub-step s (:438-491), then the
// remaining sub-steps (searching again whenever needed).
template <int DIM, bool RK>
__global__ void __launch_bounds__(128) k_search64(StepArgs a)
{
    pdl_entry();
    const uint32_t nq = *a.nxq < a.capacity ? *a.nxq : a.capacity;
    const MeshDev& m = a.mesh;
    AdvCounters k;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const uint2 e = a.xq[q];
        const uint32_t i = e.x;
        int s = (int)e.y;
        uint32_t c = a.key[i];
        const uint32_t c_old = a.S0.cell[i];
        double x[DIM], xi[DIM], u[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            x[d] = ((const double*)a.T.x[d])[i];
            xi[d] = ((const double*)a.T.xi[d])[i];
        }
        bool alive = true;
        while (true) {
            // velocity_ext of sub-step s, recomputed from the start-of-sub-step state
            if constexpr (RK) {
                double X[1 << DIM][DIM];
                load_cell64<DIM>(m.cellX, c, X);
                transport64<DIM, RK>(a, X, c, xi, u);
            } else {
                velocity64<DIM>((const double*)a.Vc, c, xi, u);
            }
            Vec<DIM> xo, ve, xp;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                xo.v[d] = xi[d];
                ve.v[d] = u[d];
                xp.v[d] = x[d];
            }
            const SearchOut so = search64<DIM>(m, c, xo, ve, xp);
            k.searched++;
            k.map_failures += so.map_failures;
            if (so.flags & SRCH_OVERFLOW) k.err |= ERR_CAND_OVERFLOW;
            if (!(so.flags & SRCH_FOUND)) {
                alive = false;
                break;
            }
            if (so.flags & SRCH_NEAR) k.near_face++;
            c = so.cell;
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = so.xi[d];
            s = substeps64<DIM, RK>(a, c, s + 1, x, xi, u, k);
            if (s >= a.pp.S) break;
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            ((double*)a.T.x[d])[i] = x[d];
            ((double*)a.T.xi[d])[i] = xi[d];
        }
        arrive(a, i, c, c_old, alive);
        if (alive) count_one(a, c, ext_part<DIM, double>(xi, a.pp));
        else k.lost++;
    }
    flush_counters(a, k);
}

// ---------------------------------------------------------------------------
// FP32 form.  The per-step cell record holds the cell's trilinear velocity
// field as monomial coefficients b_k (bit d of k selects xi_d):
//   affine cells:     the reference-space velocity w = J^-1 u, so a sub-step
//                     is  xi += dt_p w(xi)  (7 FMAs per component);
//   non-affine cells: u itself; the increment solves x(xi + d) - x(xi) = u dt_p
//                     by Newton (out of line).
// A particle that leaves its cell is queued for k_cross32, which rebuilds its
// position in FP64 and relocates it there.
// ---------------------------------------------------------------------------

template <int DIM>
struct Rec32 {
    float b[1 << DIM][DIM];
    bool affine;
};

template <int DIM>
__device__ __forceinline__ void load_rec32(const float* __restrict__ rec, uint32_t c, Rec32<DIM>& r)
{
    constexpr int F4 = Dims<DIM>::REC4;
    const float4* p = reinterpret_cast<const float4*>(rec) + (size_t)c * F4;
    float buf[F4 * 4];
#pragma unroll
    for (int k = 0; k < F4; ++k) {
        const float4 t = __ldg(p + k);
        buf[4 * k] = t.x;
        buf[4 * k + 1] = t.y;
        buf[4 * k + 2] = t.z;
        buf[4 * k + 3] = t.w;
    }
#pragma unroll
    for (int k = 0; k < (1 << DIM); ++k)
#pragma unroll
        for (int d = 0; d < DIM; ++d) r.b[k][d] = buf[k * DIM + d];
    r.affine = buf[(1 << DIM) * DIM] != 0.0f;
}

// The same record from a shared-memory stage.
template <int DIM>
__device__ __forceinline__ void load_rec32_s(const float4* p, Rec32<DIM>& r)
{
    constexpr int F4 = Dims<DIM>::REC4;
    float buf[F4 * 4];
#pragma unroll
    for (int k = 0; k < F4; ++k) {
        const float4 t = p[k];
        buf[4 * k] = t.x;
        buf[4 * k + 1] = t.y;
        buf[4 * k + 2] = t.z;
        buf[4 * k + 3] = t.w;
    }
#pragma unroll
    for (int k = 0; k < (1 << DIM); ++k)
#pragma unroll
        for (int d = 0; d < DIM; ++d) r.b[k][d] = buf[k * DIM + d];
    r.affine = buf[(1 << DIM) * DIM] != 0.0f;
}

// f(xi) = sum_k b_k prod_{d in k} xi_d, nested: 3 (2D) / 7 (3D) FMAs per component.
template <int DIM>
__device__ __forceinline__ void eval_poly(const float (*b)[DIM], const float* xi, float* f)
{
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        if constexpr (DIM == 2) {
            const float t0 = fmaf(b[1][d], xi[0], b[0][d]);
            const float t1 = fmaf(b[3][d], xi[0], b[2][d]);
            f[d] = fmaf(t1, xi[1], t0);
        } else {
            const float t0 = fmaf(b[1][d], xi[0], b[0][d]);
            const float t1 = fmaf(b[3][d], xi[0], b[2][d]);
            const float t2 = fmaf(b[5][d], xi[0], b[4][d]);
            const float t3 = fmaf(b[7][d], xi[0], b[6][d]);
            f[d] = fmaf(fmaf(t3, xi[1], t2), xi[2], fmaf(t1, xi[1], t0));
        }
    }
}

template <int DIM>
struct F3 {
    float v[DIM];
    bool ok;
};

// Newton on a non-affine cell, out of line (by value).
template <int DIM>
__device__ __noinline__ F3<DIM> newton32(const float* __restrict__ geo, uint32_t c, F3<DIM> xi, F3<DIM> dx)
{
    Geo32<DIM> g;
    load_geo32<DIM>(geo, c, g);
    F3<DIM> out;
    out.ok = advance32<DIM>(g, xi.v, dx.v, out.v);
    return out;
}

// A sub-step that moves a particle by less than 2^-46 (1.4e-14) of its
// cell in every reference direction is taken as no motion.  The FP64 form,
// like the reference, advances the physical position, and at |x| / h of
// 10^2..10^3 cells its rounding leaves x unchanged for such a step: a
// particle that the flow drives into a no-slip wall stops about 1e-14 of a
// cell from it and stays in its cell.  The FP32 form's reference coordinate
// would instead keep shrinking into subnormal floats, where the increment
// keeps only a few bits and can come out with the wrong sign; the particle
// then lands outside its cell, and the FP64 relocation finds it just beyond
// the wall and drops it while the FP64 form holds it at rest.  Such particles
// carry large velocities (the correction pulls them towards the wall's zero
// velocity step after step while they no longer move), so dropping one moves
// the projection at the wall's DoFs by up to 1e-1.  Affine cells need no
// pin: towards a xi = 0 wall their increment is a product of the coordinate
// itself (the face's velocity terms are exact zeros), which rounds towards
// the face but never past it, and towards a xi = 1 wall the spacing of FP32
// numbers below 1 (6e-8) stops the particle long before subnormals.
constexpr float XI_PIN = 1.4210855e-14f;

template <int DIM>
__device__ __forceinline__ void pin32(float* dl)
{
    float m = 0.0f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) m = fmaxf(m, fabsf(dl[d]));
    if (m < XI_PIN) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) dl[d] = 0.0f;
    }
}

// Euler sub-steps s0.. of a particle in a non-affine cell (FP32 form), out of
// line: the cell's FP32 geometry is loaded and its inverse Jacobian at the
// particle's start taken once, and every sub-step solves
// x(xi + d) - x(xi) = u dt_p by the chord iteration with that inverse (a
// particle moves a few hundredths of the cell per sub-step, so the
// iteration still contracts by the cell's twist times that distance).  The
// sub-step that leaves the cell, or whose solve does not settle, is returned
// (S if none) with xi where it stopped; the caller relocates it in FP64.
template <int DIM>
struct SubOut {
    float xi[DIM];
    int s;
};

template <int DIM>
__device__ __noinline__ SubOut<DIM> twisted_substeps32(const float* __restrict__ geo, uint32_t c, int s0, int S,
                                                       float dtp, const Rec32<DIM> r, F3<DIM> x0)
{
    Geo32<DIM> g;
    load_geo32<DIM>(geo, c, g);
    SubOut<DIM> out;
#pragma unroll
    for (int d = 0; d < DIM; ++d) out.xi[d] = x0.v[d];
    out.s = s0;
    float J[DIM][DIM], Ji[DIM][DIM];
    jac32<DIM>(g, out.xi, J);
    if (!(invert32<DIM>(J, Ji) > 0.0f)) return out;
    for (; out.s < S; ++out.s) {
        float w[DIM], dx[DIM], dl[DIM], y[DIM];
        eval_poly<DIM>(r.b, out.xi, w);
#pragma unroll
        for (int d = 0; d < DIM; ++d) dx[d] = w[d] * dtp;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            float t = 0.0f;
#pragma unroll
            for (int d = 0; d < DIM; ++d) t += Ji[k][d] * dx[d];
            dl[k] = t;
        }
        bool ok = g.affine;
        for (int it = 0; it < 8 && !ok; ++it) {
            float q[DIM];
            delta32<DIM>(g, out.xi, dl, q);
            float mx = 0.0f;
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                float t = 0.0f;
#pragma unroll
                for (int d = 0; d < DIM; ++d) t += Ji[k][d] * (q[d] - dx[d]);
                dl[k] -= t;
                mx = fmaxf(mx, fabsf(t));
            }
            ok = mx <= 2e-7f;
        }
        if (!ok) break;
        pin32<DIM>(dl);
#pragma unroll
        for (int d = 0; d < DIM; ++d) y[d] = out.xi[d] + dl[d];
        if (!inside_unit<DIM>(y)) break;
#pragma unroll
        for (int d = 0; d < DIM; ++d) out.xi[d] = y[d];
    }
    return out;
}

// RK2 midpoint of a non-affine cell in the FP32 form: xi + (h/2) J(xi)^-1 u
// with the cell's FP32 geometry, out of line (by value); xi itself when the
// Jacobian determinant is not positive.
template <int DIM>
__device__ __noinline__ F3<DIM> midpoint32(const float* __restrict__ geo, uint32_t c, F3<DIM> xi, F3<DIM> u, float hh)
{
    Geo32<DIM> g;
    load_geo32<DIM>(geo, c, g);
    float J[DIM][DIM], Ji[DIM][DIM];
    jac32<DIM>(g, xi.v, J);
    F3<DIM> out = xi;
    if (!(invert32<DIM>(J, Ji) > 0.0f)) return out;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        float s = 0.0f;
#pragma unroll
        for (int d = 0; d < DIM; ++d) s += Ji[k][d] * u.v[d];
        out.v[k] = xi.v[k] + hh * s;
    }
    return out;
}

// FP32 sub-steps s0.. in cell c; returns the sub-step that leaves the cell
// (S if none).  xi is advanced in place.  AFF: every cell of the mesh is
// affine, so the Newton branch (an out-of-line call whose saved registers
// would spill in the hot loop) is left out.
template <int DIM, bool AFF = false, bool RK = false>
__device__ __forceinline__ int substeps32(const StepArgs& a, uint32_t c, int s0, float* xi, const Rec32<DIM>& r)
{
    const float dtp = (float)a.pp.dtp;
    if constexpr (!AFF && !RK) {
        if (!r.affine) {
            F3<DIM> x0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) x0.v[d] = xi[d];
            const SubOut<DIM> o = twisted_substeps32<DIM>(a.mesh.geo32, c, s0, a.pp.S, dtp, r, x0);
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = o.xi[d];
            return o.s;
        }
    }
    int s = s0;
    for (; s < a.pp.S; ++s) {
        float w[DIM], dl[DIM], y[DIM];
        eval_poly<DIM>(r.b, xi, w);
        if constexpr (RK) {  // the midpoint rule: w (or u) at xi + (h/2) J^-1 u
            float xm[DIM];
            if (AFF || r.affine) {
#pragma unroll
                for (int d = 0; d < DIM; ++d) xm[d] = xi[d] + (0.5f * dtp) * w[d];
            } else {
                F3<DIM> x0, u0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    x0.v[d] = xi[d];
                    u0.v[d] = w[d];
                }
                const F3<DIM> mid = midpoint32<DIM>(a.mesh.geo32, c, x0, u0, 0.5f * dtp);
#pragma unroll
                for (int d = 0; d < DIM; ++d) xm[d] = mid.v[d];
            }
            eval_poly<DIM>(r.b, xm, w);
        }
        bool ok = true;
        if (AFF || r.affine) {
#pragma unroll
            for (int d = 0; d < DIM; ++d) dl[d] = dtp * w[d];
        } else {
            F3<DIM> x0, dx;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                x0.v[d] = xi[d];
                dx.v[d] = w[d] * dtp;
            }
            const F3<DIM> res = newton32<DIM>(a.mesh.geo32, c, x0, dx);
            ok = res.ok;
#pragma unroll
            for (int d = 0; d < DIM; ++d) dl[d] = res.v[d];
        }
        if (!(AFF || r.affine)) pin32<DIM>(dl);
#pragma unroll
        for (int d = 0; d < DIM; ++d) y[d] = xi[d] + dl[d];
        if (!(ok && inside_unit<DIM>(y))) break;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xi[d] = y[d];
    }
    return s;
}

template <int DIM, bool AFF = false, bool RK = false>
__device__ __forceinline__ int substeps32(const StepArgs& a, uint32_t c, int s0, float* xi)
{
    Rec32<DIM> r;
    load_rec32<DIM>(a.vrec32, c, r);
    return substeps32<DIM, AFF, RK>(a, c, s0, xi, r);
}

template <int DIM, bool AFF, bool RK = false>
__global__ void __launch_bounds__(256, AFF ? 4 : 3) k_advect32(StepArgs a)
{
    pdl_entry();
    extern __shared__ __align__(128) unsigned char adv_raw[];
    __shared__ uint64_t bar[2];
    auto* st = reinterpret_cast<AdvStage<DIM, float, ADV_CH>*>(adv_raw);
    auto* rs = reinterpret_cast<AdvRecStage<DIM>*>(adv_raw + 2 * sizeof(AdvStage<DIM, float, ADV_CH>));
    const MeshDev& m = a.mesh;
    AdvCounters k;
    staged_loop<DIM, float, ADV_CH>(a, st, bar, [&](AdvStage<DIM, float, ADV_CH>& sg, int sidx, uint32_t t, uint32_t i,
                                                    bool in) {
        const uint32_t c = in ? sg.cell[t] : HOLE;
        const bool act = c != HOLE && in;
        bool want = false, counted = false;
        int s = 0, pe = 0;
        if (in && c == HOLE) a.key[i] = LOST;
        if (act) {
            float xi[DIM], v[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                xi[d] = sg.xi[d][t];
                v[d] = sg.v[d][t];
            }
            const bool alive = c < (uint32_t)m.nC;
            if (!alive) k.err |= ERR_BAD_CELL;
            if (alive) {
                // the cell's records: staged with the chunk, or from global memory
                const AdvRecStage<DIM>& rsg = rs[sidx];
                const uint32_t lc = c - rsg.cfirst;
                const bool srec = a.chunk_first && lc < rsg.ncell;
                if (a.do_correct) {  // v += sum N_i (V - Vold)_i, src/pfem2particlehandler.cpp:126-138
                    Rec32<DIM> dr;
                    if (srec) load_rec32_s<DIM>(rsg.dv[lc], dr);
                    else load_rec32<DIM>(a.dvrec32, c, dr);
                    float dv[DIM];
                    eval_poly<DIM>(dr.b, xi, dv);
#pragma unroll
                    for (int d = 0; d < DIM; ++d) v[d] += dv[d];
                }
                Rec32<DIM> r;
                if (srec) load_rec32_s<DIM>(rsg.v[lc], r);
                else load_rec32<DIM>(a.vrec32, c, r);
                s = substeps32<DIM, AFF, RK>(a, c, 0, xi, r);
                want = s < a.pp.S;
            }
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                ((float*)a.T.xi[d])[i] = xi[d];
                ((float*)a.T.v[d])[i] = v[d];
            }
            if (want) a.key[i] = c;
            else {
                arrive(a, i, c, c, alive);
                if (!alive) k.lost++;
                counted = alive;
                if (counted) pe = ext_part<DIM, float>(xi, a.pp);
            }
        }
        defer(a, want, i, s);
        count_cells(a, counted, c, pe);
    }, a.chunk_first ? rs : nullptr);
    flush_counters(a, k);
}

// Queued FP32 particles: FP64 relocation of sub-step s (x = F(xi) + u dt_p,
// own cell first, then the vertex-patch search), then the remaining
// sub-steps in FP32 (relocating in FP64 again whenever needed).
template <int DIM, bool AFF, bool RK>
__device__ __forceinline__ void cross32(const StepArgs& a)
{
    const uint32_t nq = *a.nxq < a.capacity ? *a.nxq : a.capacity;
    const MeshDev& m = a.mesh;
    AdvCounters k;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        const uint2 e = a.xq[q];
        const uint32_t i = e.x;
        int s = (int)e.y;
        uint32_t c = a.key[i];
        const uint32_t c_old = a.S0.cell[i];
        float xi[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) xi[d] = ((const float*)a.T.xi[d])[i];
        bool alive = true;
        while (true) {
            prefetch_cell64<DIM>(m, c);
            Vec<DIM> xo, ue;
#pragma unroll
            for (int d = 0; d < DIM; ++d) xo.v[d] = (double)xi[d];
            velocity_from_dofs<DIM>(m.cd, a.Vd, m.nD, c, xo.v, ue.v);
            if constexpr (RK) {  // the midpoint rule in FP64 (transport64's operations)
                double X[1 << DIM][DIM], J[DIM][DIM], Ji[DIM][DIM], dl[DIM], xm[DIM];
                load_cell64<DIM>(m.cellX, c, X);
                jac64<DIM>(X, xo.v, J);
                if (invert64<DIM>(J, Ji) > 0.0) {
                    matvec64<DIM>(Ji, ue.v, dl);
#pragma unroll
                    for (int d = 0; d < DIM; ++d) xm[d] = xo.v[d] + (a.pp.dtp * 0.5) * dl[d];
                    velocity_from_dofs<DIM>(m.cd, a.Vd, m.nD, c, xm, ue.v);
                }
            }
            k.fallback++;
            const uint32_t c0 = c;
            const SearchOut so = fallback64<DIM, AFF>(m, c, xo, ue, a.pp.dtp);
            k.map_failures += so.map_failures;
            if (so.flags & SRCH_OVERFLOW) k.err |= ERR_CAND_OVERFLOW;
            if (so.cell != c0 || !(so.flags & SRCH_FOUND)) k.searched++;
            if (!(so.flags & SRCH_FOUND)) {
                alive = false;
                break;
            }
            if (so.flags & SRCH_NEAR) k.near_face++;
            c = so.cell;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const float t = (float)so.xi[d];
                xi[d] = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
            }
            s = substeps32<DIM, AFF, RK>(a, c, s + 1, xi);
            if (s >= a.pp.S) break;
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) ((float*)a.T.xi[d])[i] = xi[d];
        arrive(a, i, c, c_old, alive);
        if (alive) count_one(a, c, ext_part<DIM, float>(xi, a.pp));
        else k.lost++;
    }
    flush_counters(a, k);
}

template <int DIM, bool AFF = false, bool RK = false>
__global__ void __launch_bounds__(128) k_cross32(StepArgs a)
{
    pdl_entry();
    cross32<DIM, AFF, RK>(a);
}

// The same for 2D meshes with non-affine cells (many crossers, each a chain
// of dependent loads): 6 blocks per SM (80 registers, a few spills); more
// blocks cost the 3D forms about 10 %.
template <int DIM, bool RK = false>
__global__ void __launch_bounds__(128, 6) k_cross32_occ(StepArgs a)
{
    pdl_entry();
    cross32<DIM, false, RK>(a);
}

}  // namespace pfem2
