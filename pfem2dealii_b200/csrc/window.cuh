// Differentiated window of the particle path: K time steps of velocity
// correction and sub-stepped transport with relocation, from the handle's
// current particles, with count correction left out, then the projection;
// and its adjoint.  No counterpart in the reference (it has no adjoint); the
// forward arithmetic per particle is the same as the product kernels
// (k_advect64/k_search64, k_advect32/k_cross32), i.e. correct_particle_velocity
// (src/pfem2particlehandler.cpp:112-139), move_particles (:142-167) and
// sort_particles_into_subdomains_and_cells (:413-503); the projection is
// project_particle_fields (:174-215) with deterministic FP64 sums.
//
// Adjoint.  Each particle's cell sequence is frozen (cell assignment is the
// discrete, non-differentiated part).  With h = dt/S, one sub-step maps
//   x' = F_c(xi) + h u_c(xi),   xi' = F_c'^-1(x'),   u_c(xi) = sum_i N_i(xi) V_i
// so, for the adjoint g of xi and y = J_c'(xi')^-T g',
//   g = J_c(xi)^T y + h (grad_xi u_c)^T y,   dJ/dV_i += h N_i(xi) y,
// the correction v += sum_i N_i(xi) (V - Vold)_i adds
//   g += sum_i grad N_i(xi) ((V - Vold)_i . gv),   dJ/d(V - Vold)_i += N_i(xi) gv,
// and the projection U_j = num_j / den_j seeds
//   gv = sum_i N_i gnum_j(i),   g = sum_i grad N_i (gnum_j(i) . v + gden_j(i)),
//   gnum_j = gU_j / den_j,   gden_j = -(gU_j . U_j) / den_j.
// The particle velocity drives no motion, so gv is constant over the window
// and is the gradient with respect to the starting velocities.  Particles
// deleted inside the window get zero gradient.
//
// Memory: the state at the start of every segment of C steps is kept
// (checkpoints); the backward pass recomputes one segment per launch from its
// checkpoint, holding the segment's sub-step states in shared memory, and
// walks it in reverse.  Gradients with respect to nodal velocities are summed
// per (cell, vertex) with FP64 atomics after a per-warp reduction in lane
// order (their last bits can vary between runs); the projection, U and the
// per-particle gradients are deterministic.
#pragma once

#include <type_traits>

#include "advect.cuh"

namespace pfem2 {

template <typename Real>
__device__ __forceinline__ Real ldw(const void* p, size_t i) { return reinterpret_cast<const Real*>(p)[i]; }
template <typename Real>
__device__ __forceinline__ void stw(void* p, size_t i, Real v) { reinterpret_cast<Real*>(p)[i] = v; }

// ---------------------------------------------------------------------------
// Sub-steps.  Like the product (k_advect64/k_search64, k_advect32/k_cross32),
// a time step runs as two kernels: every particle's sub-steps inside its own
// cell, a particle that leaves its cell being queued with the sub-step
// index; then the queued particles' relocation and remaining sub-steps.
// The same kernels replay one segment of the window for the backward pass,
// recording the state before every sub-step.
// ---------------------------------------------------------------------------

// The FP64 vertex values of one cell from a padded per-cell table (VS per vertex).
template <int DIM>
__device__ __forceinline__ void load_vcell(const double* __restrict__ T, uint32_t c, double (*Vv)[DIM])
{
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    const double2* p = reinterpret_cast<const double2*>(T + (size_t)c * NV * VS);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double2 a = __ldg(p + i * (VS / 2));
        Vv[i][0] = a.x;
        Vv[i][1] = a.y;
        if constexpr (DIM == 3) Vv[i][2] = __ldg(p + i * (VS / 2) + 1).x;
    }
}

// State arrays of the forward (running = end state) or of a replay.
template <int DIM, typename Real>
struct WinView {
    uint32_t* cell;
    void* const* xi;
    double* const* x;
};

template <int DIM, typename Real, bool REPLAY>
__device__ __forceinline__ WinView<DIM, Real> win_view(const WinArgs& w)
{
    if constexpr (REPLAY) return {w.r_cell, w.r_xi, w.r_x};
    else return {w.fin_cell, w.fin_xi, w.fin_x};
}

template <int DIM, typename Real>
__device__ __forceinline__ void win_record(const WinArgs& w, int t, uint32_t p, uint32_t c, const Real* xi)
{
    const size_t o = (size_t)t * w.n + p;
    w.rec_cell[o] = c;
#pragma unroll
    for (int d = 0; d < DIM; ++d) stw<Real>(w.rec_xi[d], o, xi[d]);
}

// In-cell sub-steps s0.. of one particle in cell c (records the state before
// each when t0 >= 0); returns the sub-step that leaves the cell, S if none.
// FP64 form: on leaving, x has moved and xi is the sub-step's start.
template <int DIM, typename Real>
__device__ __forceinline__ int win_incell(const WinArgs& w, uint32_t p, uint32_t c, int s0, Real* xi, double* x,
                                          int t0)
{
    const StepArgs& a = w.a;
    const int S = a.pp.S;
    int s = s0;
    if constexpr (std::is_same<Real, double>::value) {
        constexpr int NV = 1 << DIM;
        double X[NV][DIM];
        load_cell64<DIM>(a.mesh.cellX, c, X);
        for (; s < S; ++s) {
            if (t0 >= 0) win_record<DIM, Real>(w, t0 + s, p, c, xi);
            double u[DIM], xin[DIM];
            velocity64<DIM>((const double*)a.Vc, c, xi, u);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const double st = u[d] * a.pp.dtp;
                x[d] = x[d] + st;
            }
            const int st = inverse_map64<DIM>(X, a.mesh.aff + (size_t)c * Dims<DIM>::AFF, x, xin);
            if (!(st == 0 && inside_unit<DIM>(xin))) break;
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = xin[d];
        }
    } else {
        Rec32<DIM> r;
        load_rec32<DIM>(a.vrec32, c, r);
        const float dtp = (float)a.pp.dtp;
        for (; s < S; ++s) {
            if (t0 >= 0) win_record<DIM, Real>(w, t0 + s, p, c, xi);
            float wv[DIM], dl[DIM], y[DIM];
            eval_poly<DIM>(r.b, xi, wv);
            bool ok = true;
            if (r.affine) {
#pragma unroll
                for (int d = 0; d < DIM; ++d) dl[d] = dtp * wv[d];
            } else {
                F3<DIM> x0, dx;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    x0.v[d] = xi[d];
                    dx.v[d] = wv[d] * dtp;
                }
                const F3<DIM> res = newton32<DIM>(a.mesh.geo32, c, x0, dx);
                ok = res.ok;
#pragma unroll
                for (int d = 0; d < DIM; ++d) dl[d] = res.v[d];
            }
#pragma unroll
            for (int d = 0; d < DIM; ++d) y[d] = xi[d] + dl[d];
            if (!(ok && inside_unit<DIM>(y))) break;
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = y[d];
        }
    }
    return s;
}

// Relocation of sub-step s of a particle that left cell c (false: deleted).
// FP64 form: the vertex-patch search from the moved x (k_search64); FP32
// form: the FP64 relocation of F(xi) + u dt_p (k_cross32).
template <int DIM, typename Real>
__device__ __forceinline__ bool win_relocate(const WinArgs& w, uint32_t& c, Real* xi, double* x)
{
    const StepArgs& a = w.a;
    if constexpr (std::is_same<Real, double>::value) {
        double u[DIM];
        velocity64<DIM>((const double*)a.Vc, c, xi, u);
        Vec<DIM> xo, ve, xp;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xo.v[d] = xi[d];
            ve.v[d] = u[d];
            xp.v[d] = x[d];
        }
        const SearchOut so = search64<DIM>(a.mesh, c, xo, ve, xp);
        if (!(so.flags & SRCH_FOUND)) return false;
        c = so.cell;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xi[d] = so.xi[d];
    } else {
        Vec<DIM> xo, ue;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xo.v[d] = (double)xi[d];
        velocity_from_dofs<DIM>(a.mesh.cd, a.Vd, a.mesh.nD, c, xo.v, ue.v);
        const SearchOut so = a.mesh.all_affine ? fallback64<DIM, true>(a.mesh, c, xo, ue, a.pp.dtp)
                                               : fallback64<DIM, false>(a.mesh, c, xo, ue, a.pp.dtp);
        if (!(so.flags & SRCH_FOUND)) return false;
        c = so.cell;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const float t = (float)so.xi[d];
            xi[d] = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
        }
    }
    return true;
}

// v += sum_i N_i(xi) (V - Vold)_i in FP64.  The window keeps the particle
// velocities (the differentiated variables) in FP64 in both forms: the FP64
// form with k_advect64's arithmetic, the FP32 form from its FP32 xi and the
// FP64 per-cell table of V - Vold.
template <int DIM, typename Real>
__device__ __forceinline__ void win_correct(const WinArgs& w, uint32_t c, const Real* xi, double* v)
{
    double corr[DIM];
    if constexpr (std::is_same<Real, double>::value) {
        velocity64<DIM>((const double*)w.a.dVc, c, xi, corr);
    } else {
        double x[DIM], Dv[1 << DIM][DIM], N[1 << DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) x[d] = (double)xi[d];
        shape64<DIM>(x, N);
        load_vcell<DIM>(w.dVcell, c, Dv);
#pragma unroll
        for (int d = 0; d < DIM; ++d) corr[d] = 0.0;
#pragma unroll
        for (int i = 0; i < (1 << DIM); ++i)
#pragma unroll
            for (int d = 0; d < DIM; ++d) corr[d] = corr[d] + N[i] * Dv[i][d];
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = v[d] + corr[d];
}

// Queue a face crosser (one atomic per warp; all lanes call it).
__device__ __forceinline__ void win_defer(const WinArgs& w, bool want, uint32_t p, int s)
{
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(w.nq, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) w.q[base + __popc(m & ((1u << lane) - 1u))] = make_uint2(p, (uint32_t)s);
}

// Window particles from the live slots of the handle's current state, with
// their starting velocities (v0: n x dim, or the particles' own).
template <int DIM, typename Real>
__global__ void k_win_init(WinArgs w, const double* __restrict__ v0)
{
    const PartState& S = w.a.S0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < w.n; p += gridDim.x * blockDim.x) {
        const uint32_t s = w.slot[p];
        w.fin_cell[p] = S.cell[s];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            stw<Real>(w.fin_xi[d], p, ldw<Real>(S.xi[d], s));
            if constexpr (std::is_same<Real, double>::value) w.fin_x[d][p] = ldw<double>(S.x[d], s);
            w.fin_v[d][p] = v0 ? v0[(size_t)p * DIM + d] : (double)ldw<Real>(S.v[d], s);
        }
    }
}

// Step k, first kernel.  Forward (REPLAY false): the state at the start of a
// segment goes to its checkpoint, then the correction, then the in-cell
// sub-steps.  Replay of the segment starting at step k0: the particles alive
// at the window's end, from the checkpoint at k == k0.  With `record`, the
// states before every sub-step of the segment starting at k0 (and its end
// state) are recorded: always in a replay, and in the forward's last segment.
template <int DIM, typename Real, bool REPLAY>
__global__ void __launch_bounds__(256) k_win_adv(WinArgs w, int k, int k0, int record)
{
    const WinView<DIM, Real> V = win_view<DIM, Real, REPLAY>(w);
    const int S = w.a.pp.S;
    const bool seg_start = k % w.C == 0;
    const bool seg_end = record && (k + 1 == w.K || (k + 1) % w.C == 0);
    const int t0 = record ? (k - k0) * S : -1;
    const uint32_t nloop = (w.n + 31u) & ~31u;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < nloop; p += gridDim.x * blockDim.x) {
        bool want = false;
        int s = 0;
        if (p < w.n) {
            uint32_t c;
            Real xi[DIM];
            double x[DIM];
            bool act;
            const bool from_ck = REPLAY && k == k0;
            if (from_ck) {
                const size_t o = (size_t)(k / w.C) * w.n + p;
                act = w.fin_cell[p] < (uint32_t)w.a.mesh.nC;
                c = w.ck_cell[o];
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    xi[d] = ldw<Real>(w.ck_xi[d], o);
                    if constexpr (std::is_same<Real, double>::value) x[d] = w.ck_x[d][o];
                }
            } else {
                c = V.cell[p];
                act = c < (uint32_t)w.a.mesh.nC && (!REPLAY || w.fin_cell[p] < (uint32_t)w.a.mesh.nC);
                if (act)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        xi[d] = ldw<Real>(V.xi[d], p);
                        if constexpr (std::is_same<Real, double>::value) x[d] = V.x[d][p];
                    }
            }
            if (act) {
                if (!REPLAY && seg_start) {
                    const size_t o = (size_t)(k / w.C) * w.n + p;
                    w.ck_cell[o] = c;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        stw<Real>(w.ck_xi[d], o, xi[d]);
                        if constexpr (std::is_same<Real, double>::value) w.ck_x[d][o] = x[d];
                    }
                }
                if (!REPLAY && w.do_correct) {
                    double v[DIM];
#pragma unroll
                    for (int d = 0; d < DIM; ++d) v[d] = w.fin_v[d][p];
                    win_correct<DIM, Real>(w, c, xi, v);
#pragma unroll
                    for (int d = 0; d < DIM; ++d) w.fin_v[d][p] = v[d];
                }
                s = win_incell<DIM, Real>(w, p, c, 0, xi, x, t0);
                want = s < S;
                if (!want && seg_end) win_record<DIM, Real>(w, t0 + S, p, c, xi);
                if (from_ck) V.cell[p] = c;
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    stw<Real>(V.xi[d], p, xi[d]);
                    if constexpr (std::is_same<Real, double>::value) V.x[d][p] = x[d];
                }
            }
        }
        win_defer(w, want, p, s);
    }
}

// Step k, second kernel: the queued particles' relocations and remaining
// sub-steps (relocating again whenever they leave a cell).
template <int DIM, typename Real, bool REPLAY>
__global__ void __launch_bounds__(128) k_win_cross(WinArgs w, int k, int k0, int record)
{
    const WinView<DIM, Real> V = win_view<DIM, Real, REPLAY>(w);
    const int S = w.a.pp.S;
    const bool seg_end = record && (k + 1 == w.K || (k + 1) % w.C == 0);
    const int t0 = record ? (k - k0) * S : -1;
    const uint32_t nq = *w.nq;
    unsigned int err = 0;
    for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += gridDim.x * blockDim.x) {
        const uint2 e = w.q[qi];
        const uint32_t p = e.x;
        int s = (int)e.y;
        uint32_t c = V.cell[p];
        Real xi[DIM];
        double x[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xi[d] = ldw<Real>(V.xi[d], p);
            if constexpr (std::is_same<Real, double>::value) x[d] = V.x[d][p];
        }
        bool alive = true;
        while (true) {
            if (!win_relocate<DIM, Real>(w, c, xi, x)) {
                alive = false;
                break;
            }
            s = win_incell<DIM, Real>(w, p, c, s + 1, xi, x, t0);
            if (s >= S) break;
        }
        if (!alive) {
            c = LOST;
            if (REPLAY) err |= ERR_REPLAY;  // alive at the window's end, so never deleted before
        } else if (seg_end) {
            win_record<DIM, Real>(w, t0 + S, p, c, xi);
        }
        V.cell[p] = c;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            stw<Real>(V.xi[d], p, xi[d]);
            if constexpr (std::is_same<Real, double>::value) V.x[d][p] = x[d];
        }
    }
    if (err) atomicOr(w.err, err);
}

// One warp per cell: the cell's particles in ascending index (rank by
// counting), then the FP64 projection partials summed in that order: lane l
// takes particles l, l+32, ..., then a fixed butterfly.
template <int DIM, typename Real>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_win_cellsum(WinArgs w)
{
    constexpr int NV = 1 << DIM, NP = NV * (DIM + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x * CELL_WARPS + warp; c < w.a.mesh.nC; c += gridDim.x * CELL_WARPS) {
        const uint32_t b = w.cstart[c], e = w.cstart[c + 1], cnt = e - b;
        for (uint32_t i = lane; i < cnt; i += 32) {
            const uint32_t key = w.order[b + i];
            uint32_t rank = 0;
            for (uint32_t j = 0; j < cnt; ++j) rank += w.order[b + j] < key ? 1u : 0u;
            w.order2[b + rank] = key;
        }
        __syncwarp();
        double acc[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) acc[k] = 0.0;
        for (uint32_t i = lane; i < cnt; i += 32) {
            const uint32_t p = w.order2[b + i];
            double xi[DIM], v[DIM], N[NV];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                xi[d] = (double)ldw<Real>(w.fin_xi[d], p);
                v[d] = w.fin_v[d][p];
            }
            shape64<DIM>(xi, N);
#pragma unroll
            for (int iv = 0; iv < NV; ++iv) {
#pragma unroll
                for (int d = 0; d < DIM; ++d) acc[iv * (DIM + 1) + d] = acc[iv * (DIM + 1) + d] + N[iv] * v[d];
                acc[iv * (DIM + 1) + DIM] = acc[iv * (DIM + 1) + DIM] + N[iv];
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int k = 0; k < NP; ++k) acc[k] = acc[k] + __shfl_xor_sync(0xffffffffu, acc[k], o);
        if (lane < NV) {
            double* q = w.part + ((size_t)c * NV + lane) * 4;
#pragma unroll
            for (int iv = 0; iv < NV; ++iv)
                if (iv == lane) {
#pragma unroll
                    for (int k = 0; k <= DIM; ++k) q[k] = acc[iv * (DIM + 1) + k];
                }
        }
    }
}

// ---------------------------------------------------------------------------
// Backward pass.
// ---------------------------------------------------------------------------

// Per particle: gv and the adjoint of the final xi from the projection;
// g_v0 (n x dim) gets gv.
template <int DIM, typename Real>
__global__ void k_win_bwd_init(WinArgs w, double* __restrict__ g_v0)
{
    constexpr int NV = 1 << DIM;
    const int nD = w.a.mesh.nD;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < w.n; p += gridDim.x * blockDim.x) {
        const uint32_t c = w.fin_cell[p];
        double gv[DIM], g[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) gv[d] = g[d] = 0.0;
        if (c < (uint32_t)w.a.mesh.nC) {
            double xi[DIM], v[DIM], N[NV], G[NV][DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                xi[d] = (double)ldw<Real>(w.fin_xi[d], p);
                v[d] = w.fin_v[d][p];
            }
            shape64<DIM>(xi, N);
            shape_grad64<DIM>(xi, G);
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                const int32_t j = w.a.mesh.cd[(size_t)c * NV + i];
                double s = w.gden[j];
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    const double gn = w.gnum[(size_t)d * nD + j];
                    gv[d] = gv[d] + N[i] * gn;
                    s = s + gn * v[d];
                }
#pragma unroll
                for (int k = 0; k < DIM; ++k) g[k] = g[k] + G[i][k] * s;
            }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            w.gv[(size_t)d * w.n + p] = gv[d];
            w.gxi[(size_t)d * w.n + p] = g[d];
            if (g_v0) g_v0[(size_t)p * DIM + d] = gv[d];
        }
    }
}

// Warp-cooperative add of each lane's NV x DIM values into acc[key * NV*DIM + m]:
// lanes in order, one atomic per run of equal keys per value (lanes with
// key LOST add nothing).  All 32 lanes call it.
template <int NVD>
__device__ __forceinline__ void warp_flush(double* buf, uint32_t* keys, uint32_t key, const double* vals,
                                           double* acc)
{
    const int lane = threadIdx.x & 31;
    keys[lane] = key;
#pragma unroll
    for (int m = 0; m < NVD; ++m) buf[m * 32 + lane] = vals[m];
    __syncwarp();
    if (lane < NVD) {
        uint32_t cur = LOST;
        double s = 0.0;
        for (int l = 0; l < 32; ++l) {
            const uint32_t k = keys[l];
            if (k != cur) {
                if (cur != LOST) atomicAdd(acc + (size_t)cur * NVD + lane, s);
                cur = k;
                s = 0.0;
            }
            s = s + buf[lane * 32 + l];
        }
        if (cur != LOST) atomicAdd(acc + (size_t)cur * NVD + lane, s);
    }
    __syncwarp();
}

// Reverse sweep over segment j (steps j*C .. min(K, (j+1)*C) - 1) from the
// recorded sub-step states.  With W_i = X_i + h V_i (the vertices of the
// sub-step map x' = sum N_i(xi) W_i), the adjoint of xi before a sub-step is
// g = sum_i grad N_i(xi) (W_i . y), y = J_c'(xi')^-T g'.  AFF: every cell is
// affine, J^-1 is the cell's constant inverse.  Gradients with respect to
// nodal values accumulate per particle while it stays in one cell; a change
// of cell adds the sum alone, the segment's end adds it warp-cooperatively.
// The thread loop is uniform across a warp (warp_flush).
// N_i and grad N_i of one vertex from the pairwise products of the 1D
// factors L_m = (1 - xi_m, xi_m); the products are taken in shape64's and
// shape_grad64's order, so the values are theirs.
template <int DIM>
struct ShapeF {
    double L[DIM][2];
    double P01[2][2], P02[2][2], P12[2][2];
    __device__ __forceinline__ explicit ShapeF(const double* xi)
    {
#pragma unroll
        for (int m = 0; m < DIM; ++m) {
            L[m][0] = 1.0 - xi[m];
            L[m][1] = xi[m];
        }
        if constexpr (DIM == 3) {
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    P01[a][b] = L[0][a] * L[1][b];
                    P02[a][b] = L[0][a] * L[2][b];
                    P12[a][b] = L[1][a] * L[2][b];
                }
        }
    }
    __device__ __forceinline__ double value_and_grad(int i, double* G) const
    {
        const int b0 = i & 1, b1 = (i >> 1) & 1;
        if constexpr (DIM == 2) {
            G[0] = b0 ? L[1][b1] : -L[1][b1];
            G[1] = b1 ? L[0][b0] : -L[0][b0];
            return L[0][b0] * L[1][b1];
        } else {
            const int b2 = (i >> 2) & 1;
            G[0] = b0 ? P12[b1][b2] : -P12[b1][b2];
            G[1] = b1 ? P02[b0][b2] : -P02[b0][b2];
            G[2] = b2 ? P01[b0][b1] : -P01[b0][b1];
            return P01[b0][b1] * L[2][b2];
        }
    }
};

template <int DIM, typename Real, bool AFF>
__global__ void __launch_bounds__(128, 3) k_win_rev(WinArgs w, int j)
{
    constexpr int NV = 1 << DIM, NVD = NV * DIM, VS = Dims<DIM>::VS;
    __shared__ double fbuf_s[4][32 * NVD];
    __shared__ uint32_t fkey_s[4][32];
    const int warp = threadIdx.x >> 5;
    double* fbuf = fbuf_s[warp];
    uint32_t* fkey = fkey_s[warp];
    const int k0 = j * w.C, k1 = min(w.K, k0 + w.C), S = w.a.pp.S;
    const int tseg = (k1 - k0) * S;
    const double h = w.a.pp.dtp;
    const MeshDev& m = w.a.mesh;
    unsigned int err = 0;
    const uint32_t nloop = (w.n + 31u) & ~31u;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < nloop; p += gridDim.x * blockDim.x) {
        bool act = p < w.n && w.fin_cell[p] < (uint32_t)m.nC;
        double g[DIM], gv[DIM], acc[NVD], accN[NV], Bi[DIM][DIM];
        uint32_t acc_c = LOST, bi_c = LOST;
#pragma unroll
        for (int k = 0; k < NVD; ++k) acc[k] = 0.0;
#pragma unroll
        for (int i = 0; i < NV; ++i) accN[i] = 0.0;
        if (act) {
            // the replay must have ended where the forward did
            const size_t oe = (size_t)tseg * w.n + p;
            const uint32_t ce = w.rec_cell[oe];
            bool same;
            if (k1 < w.K) {
                const size_t o = (size_t)(j + 1) * w.n + p;
                same = w.ck_cell[o] == ce;
#pragma unroll
                for (int d = 0; d < DIM; ++d) same = same && ldw<Real>(w.ck_xi[d], o) == ldw<Real>(w.rec_xi[d], oe);
            } else {
                same = w.fin_cell[p] == ce;
#pragma unroll
                for (int d = 0; d < DIM; ++d) same = same && ldw<Real>(w.fin_xi[d], p) == ldw<Real>(w.rec_xi[d], oe);
            }
            if (!same) {
                err |= ERR_REPLAY;
                act = false;
            }
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            g[d] = act ? w.gxi[(size_t)d * w.n + p] : 0.0;
            gv[d] = act ? w.gv[(size_t)d * w.n + p] : 0.0;
        }
        // J^-1 at the segment's end state
        if (act) {
            const size_t oe = (size_t)tseg * w.n + p;
            const uint32_t cb = w.rec_cell[oe];
            if constexpr (AFF) {
#pragma unroll
                for (int r = 0; r < DIM; ++r)
#pragma unroll
                    for (int q = 0; q < DIM; ++q) Bi[r][q] = __ldg(m.aff + (size_t)cb * Dims<DIM>::AFF + r * DIM + q);
                bi_c = cb;
            } else {
                double X[NV][DIM], xb[DIM], Jb[DIM][DIM];
                load_cell64<DIM>(m.cellX, cb, X);
#pragma unroll
                for (int d = 0; d < DIM; ++d) xb[d] = (double)ldw<Real>(w.rec_xi[d], oe);
                jac64<DIM>(X, xb, Jb);
                invert64<DIM>(Jb, Bi);
            }
        }
        for (int t = tseg - 1; t >= 0; --t) {
            if (!act) continue;
            const size_t o = (size_t)t * w.n + p;
            const uint32_t ca = w.rec_cell[o];
            double xa[DIM], y[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) xa[d] = (double)ldw<Real>(w.rec_xi[d], o);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {  // y = J^-T g
                double sy = 0.0;
#pragma unroll
                for (int k = 0; k < DIM; ++k) sy = sy + Bi[k][d] * g[k];
                y[d] = sy;
            }
            if (ca != acc_c) {  // the accumulators belong to a later cell: add them alone
                if (acc_c != LOST) {
#pragma unroll
                    for (int k = 0; k < NVD; ++k) atomicAdd(w.gadv + (size_t)acc_c * NVD + k, acc[k]);
                    if (w.do_correct)
#pragma unroll
                        for (int i = 0; i < NV; ++i)
#pragma unroll
                            for (int d = 0; d < DIM; ++d)
                                atomicAdd(w.gdv + (size_t)acc_c * NVD + i * DIM + d, accN[i] * gv[d]);
                }
#pragma unroll
                for (int k = 0; k < NVD; ++k) acc[k] = 0.0;
#pragma unroll
                for (int i = 0; i < NV; ++i) accN[i] = 0.0;
                acc_c = ca;
            }
            // shape values and gradients per vertex from the pairwise products of
            // the 1D factors, in shape64's / shape_grad64's multiplication order
            ShapeF<DIM> sf(xa);
            double gn[DIM];
#pragma unroll
            for (int k = 0; k < DIM; ++k) gn[k] = 0.0;
            const double2* Wp = reinterpret_cast<const double2*>(w.Wcell + (size_t)ca * NV * VS);
            const bool corr = w.do_correct && t % S == 0;
            const double2* Dp = reinterpret_cast<const double2*>(w.dVcell + (size_t)ca * NV * VS);
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                double Gi[DIM];
                const double Ni = sf.value_and_grad(i, Gi);
                double Wi[DIM];
                const double2 a0 = __ldg(Wp + i * (VS / 2));
                Wi[0] = a0.x;
                Wi[1] = a0.y;
                if constexpr (DIM == 3) Wi[2] = __ldg(Wp + i * (VS / 2) + 1).x;
                double si = 0.0;
#pragma unroll
                for (int d = 0; d < DIM; ++d) si = si + Wi[d] * y[d];
                if (corr) {  // the correction at the start of step t / S
                    double Di[DIM];
                    const double2 b0 = __ldg(Dp + i * (VS / 2));
                    Di[0] = b0.x;
                    Di[1] = b0.y;
                    if constexpr (DIM == 3) Di[2] = __ldg(Dp + i * (VS / 2) + 1).x;
                    double ci = 0.0;
#pragma unroll
                    for (int d = 0; d < DIM; ++d) ci = ci + Di[d] * gv[d];
                    si = si + ci;
                    accN[i] = accN[i] + Ni;
                }
#pragma unroll
                for (int k = 0; k < DIM; ++k) gn[k] = gn[k] + Gi[k] * si;
                const double hn = h * Ni;
#pragma unroll
                for (int d = 0; d < DIM; ++d) acc[i * DIM + d] = acc[i * DIM + d] + hn * y[d];
            }
#pragma unroll
            for (int k = 0; k < DIM; ++k) g[k] = gn[k];
            // J^-1 at this state, for the sub-step before it
            if constexpr (AFF) {
                if (ca != bi_c) {
#pragma unroll
                    for (int r = 0; r < DIM; ++r)
#pragma unroll
                        for (int q = 0; q < DIM; ++q) Bi[r][q] = __ldg(m.aff + (size_t)ca * Dims<DIM>::AFF + r * DIM + q);
                    bi_c = ca;
                }
            } else {
                double X[NV][DIM], Ja[DIM][DIM], G[NV][DIM];
                load_cell64<DIM>(m.cellX, ca, X);
#pragma unroll
                for (int i = 0; i < NV; ++i) sf.value_and_grad(i, G[i]);
#pragma unroll
                for (int d = 0; d < DIM; ++d)
#pragma unroll
                    for (int k = 0; k < DIM; ++k) {
                        double sj = 0.0;
#pragma unroll
                        for (int i = 0; i < NV; ++i) sj = sj + G[i][k] * X[i][d];
                        Ja[d][k] = sj;
                    }
                invert64<DIM>(Ja, Bi);
            }
        }
        double cv[NVD];
#pragma unroll
        for (int i = 0; i < NV; ++i)
#pragma unroll
            for (int d = 0; d < DIM; ++d) cv[i * DIM + d] = accN[i] * gv[d];
        const uint32_t key = act ? acc_c : LOST;
        warp_flush<NVD>(fbuf, fkey, key, acc, w.gadv);
        if (w.do_correct) warp_flush<NVD>(fbuf, fkey, key, cv, w.gdv);
        if (act)
#pragma unroll
            for (int d = 0; d < DIM; ++d) w.gxi[(size_t)d * w.n + p] = g[d];
    }
    err = __reduce_or_sync(0xffffffffu, err);
    if ((threadIdx.x & 31) == 0 && err) atomicOr(w.err, err);
}

// Per cell: W_i = X_i + h V_i (padded like Vcell).
template <int DIM>
__global__ void k_win_wcell(WinArgs w, const double* __restrict__ Vcell, double* __restrict__ Wout)
{
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    const int total = w.a.mesh.nC * NV;
    const double h = w.a.pp.dtp;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < VS; ++d) {
            const double x = d < DIM ? w.a.mesh.cellX[(size_t)t * DIM + d] : 0.0;
            const double v = Vcell[(size_t)t * VS + d];
            Wout[(size_t)t * VS + d] = x + h * v;
        }
    }
}

// ---------------------------------------------------------------------------
// Host-side sequences of one form (instantiated in window_f64.cu / window_f32.cu).
// ---------------------------------------------------------------------------
template <typename K>
inline int win_grid(K kernel, int threads)
{
    return occupancy_grid((const void*)kernel, threads);
}

template <int DIM, typename Real, bool REPLAY>
inline int win_step(const WinArgs& w, int k, int k0, int record, cudaStream_t s)
{
    cudaMemsetAsync(w.nq, 0, sizeof(uint32_t), s);
    k_win_adv<DIM, Real, REPLAY><<<win_grid(k_win_adv<DIM, Real, REPLAY>, 256), 256, 0, s>>>(w, k, k0, record);
    k_win_cross<DIM, Real, REPLAY><<<win_grid(k_win_cross<DIM, Real, REPLAY>, 128), 128, 0, s>>>(w, k, k0, record);
    return 2;
}

// The forward records its last segment (the backward's first).
template <int DIM, typename Real>
inline int win_forward_t(const WinArgs& w, cudaStream_t s)
{
    int n = 0;
    const int klast = (w.nseg - 1) * w.C;
    for (int k = 0; k < w.K; ++k) n += win_step<DIM, Real, false>(w, k, klast, k >= klast ? 1 : 0, s);
    return n;
}

// Segments in reverse: replay (recording) unless the record buffer holds the
// segment already (rec_seg), then the reverse sweep.
template <int DIM, typename Real>
inline int win_backward_t(const WinArgs& w, double* g_v0, int rec_seg, cudaStream_t s)
{
    k_win_bwd_init<DIM, Real><<<win_grid(k_win_bwd_init<DIM, Real>, 256), 256, 0, s>>>(w, g_v0);
    int n = 1;
    if (w.K == 0) return n;
    for (int j = w.nseg - 1; j >= 0; --j) {
        const int k0 = j * w.C, k1 = k0 + w.C < w.K ? k0 + w.C : w.K;
        if (j != rec_seg)
            for (int k = k0; k < k1; ++k) n += win_step<DIM, Real, true>(w, k, k0, 1, s);
        if (w.a.mesh.all_affine)
            k_win_rev<DIM, Real, true><<<win_grid(k_win_rev<DIM, Real, true>, 128), 128, 0, s>>>(w, j);
        else
            k_win_rev<DIM, Real, false><<<win_grid(k_win_rev<DIM, Real, false>, 128), 128, 0, s>>>(w, j);
        n += 1;
    }
    return n;
}

// ---------------------------------------------------------------------------
// Form-independent kernels (compiled once, in window_f64.cu).
// ---------------------------------------------------------------------------
#ifdef PFEM2_WINDOW_GENERIC
// ---------------------------------------------------------------------------
// Scans (exclusive, u32) and compaction of the live slots.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < nw ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    const uint32_t base = warp ? sh[warp - 1] : 0u;
    if (total) *total = sh[nw - 1];
    __syncthreads();
    return base + inc - v;
}

// Tile sums of in[0..n) (in == null: 1 for each live slot of `cells`).
__global__ void __launch_bounds__(256) k_win_tilesum(const uint32_t* __restrict__ in, const uint32_t* __restrict__ cells,
                                                     uint32_t n, uint32_t nC, uint32_t* __restrict__ tsum)
{
    __shared__ uint32_t sh[32];
    const uint32_t base = blockIdx.x * WIN_TILE;
    uint32_t s = 0;
    for (uint32_t k = threadIdx.x; k < WIN_TILE; k += blockDim.x) {
        const uint32_t i = base + k;
        if (i < n) s += in ? in[i] : (cells[i] < nC ? 1u : 0u);
    }
    uint32_t tot;
    block_excl_scan(s, sh, &tot);
    if (threadIdx.x == 0) tsum[blockIdx.x] = tot;
}

// Exclusive scan of the tile sums in place (one block); tsum[ntiles] = total.
__global__ void __launch_bounds__(1024) k_win_tilescan(uint32_t* tsum, uint32_t ntiles)
{
    __shared__ uint32_t sh[32];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < ntiles; b += blockDim.x) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < ntiles ? tsum[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(v, sh, &tot);
        if (i < ntiles) tsum[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) tsum[ntiles] = carry;
}

// out[i] = exclusive prefix of in (out[n] = total), or, with in == null, the
// compaction slot_out[k] = k-th live slot of `cells`.
__global__ void __launch_bounds__(256) k_win_apply(const uint32_t* __restrict__ in, const uint32_t* __restrict__ cells,
                                                   uint32_t n, uint32_t nC, const uint32_t* __restrict__ tsum,
                                                   uint32_t* __restrict__ out)
{
    __shared__ uint32_t sh[32];
    constexpr int PER = WIN_TILE / 256;
    const uint32_t base = blockIdx.x * WIN_TILE + threadIdx.x * PER;
    uint32_t v[PER], s = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const uint32_t i = base + k;
        v[k] = i < n ? (in ? in[i] : (cells[i] < nC ? 1u : 0u)) : 0u;
        s += v[k];
    }
    uint32_t pre = tsum[blockIdx.x] + block_excl_scan(s, sh, nullptr);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const uint32_t i = base + k;
        if (i < n) {
            if (in) out[i] = pre;
            else if (v[k]) out[pre] = i;
        }
        pre += v[k];
    }
    if (in && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = tsum[gridDim.x];
}

// Particles per final cell.
__global__ void k_win_count(WinArgs w)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < w.n; p += gridDim.x * blockDim.x) {
        const uint32_t c = w.fin_cell[p];
        if (c < (uint32_t)w.a.mesh.nC) atomicAdd(w.ccnt + c, 1u);
    }
}

// Particles into their final cell's range (arbitrary order inside a cell).
__global__ void k_win_place(WinArgs w)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < w.n; p += gridDim.x * blockDim.x) {
        const uint32_t c = w.fin_cell[p];
        if (c < (uint32_t)w.a.mesh.nC) w.order[w.cstart[c] + atomicAdd(w.ccnt + c, 1u)] = p;
    }
}

// Per DoF: num and den over its cells in ascending order, U = num / den.
template <int DIM>
__global__ void k_win_gather(WinArgs w)
{
    constexpr int NV = 1 << DIM;
    const int nD = w.a.mesh.nD;
    unsigned long long empty = 0;
    const int stride = gridDim.x * blockDim.x;
    const int nloop = (nD + stride - 1) / stride * stride;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nloop; j += stride) {
        if (j < nD) {
            double num[DIM], den = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) num[d] = 0.0;
            const int32_t b = w.a.mesh.d2c_off[j], e = w.a.mesh.d2c_off[j + 1];
            for (int32_t k = b; k < e; ++k) {
                const int32_t en = w.a.mesh.d2c_ent[k];
                const double* q = w.part + ((size_t)(en / NV) * NV + en % NV) * 4;
#pragma unroll
                for (int d = 0; d < DIM; ++d) num[d] = num[d] + q[d];
                den = den + q[DIM];
            }
            w.den[j] = den;
            if (den == 0.0) empty++;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                const size_t o = (size_t)d * nD + j;
                w.U[o] = (den == 0.0 && w.keep_empty) ? w.V[o] : num[d] / den;
            }
        }
    }
    empty = warp_sum_u64(empty);
    if ((threadIdx.x & 31) == 0 && empty) atomicAdd(w.nempty, empty);
}

// gnum = gU / den, gden = -(gU . U) / den per DoF (0 where den = 0).
template <int DIM>
__global__ void k_win_gseed(WinArgs w, const double* __restrict__ gU)
{
    const int nD = w.a.mesh.nD;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nD; j += gridDim.x * blockDim.x) {
        const double den = w.den[j];
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const size_t o = (size_t)d * nD + j;
            w.gnum[o] = den == 0.0 ? 0.0 : gU[o] / den;
            s = s + gU[o] * w.U[o];
        }
        w.gden[j] = den == 0.0 ? 0.0 : -s / den;
    }
}

// Per DoF: g_V = sum (gadv + gdv), g_Vold = -sum gdv over the DoF's (cell,
// vertex) entries in ascending cell order; under empty_dof_policy 1 the DoFs
// without particle weight pass gU through to g_V (U = V there).
template <int DIM>
__global__ void k_win_gV(WinArgs w, const double* __restrict__ gU, double* __restrict__ gV, double* __restrict__ gVold)
{
    constexpr int NV = 1 << DIM;
    const int nD = w.a.mesh.nD;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nD; j += gridDim.x * blockDim.x) {
        double a[DIM], b[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) a[d] = b[d] = 0.0;
        const int32_t e0 = w.a.mesh.d2c_off[j], e1 = w.a.mesh.d2c_off[j + 1];
        for (int32_t k = e0; k < e1; ++k) {
            const int32_t en = w.a.mesh.d2c_ent[k];
            const size_t o = ((size_t)(en / NV) * NV + en % NV) * DIM;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                a[d] = a[d] + w.gadv[o + d];
                b[d] = b[d] + w.gdv[o + d];
            }
        }
        const bool pass = w.keep_empty && w.den[j] == 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const size_t o = (size_t)d * nD + j;
            if (gV) gV[o] = a[d] + b[d] + (pass ? gU[o] : 0.0);
            if (gVold) gVold[o] = -b[d];
        }
    }
}

#endif  // PFEM2_WINDOW_GENERIC

}  // namespace pfem2
