// Small kernels of the particle cycle: arrival-list set-up for an uploaded
// particle set, finalisation of the step's counters, and the staging of nodal
// velocities (component-major doubles, one vector per component as the
// reference's std::array<TrilinosWrappers::MPI::Vector,dim>) into per-cell
// vertex records the particle kernels read.
#include "launch.h"
#include "geom64.cuh"

namespace pfem2 {

namespace {

constexpr int SB = 512;              // scan block: one cell per thread
constexpr int SI = SCAN_TILE / SB;   // rows of SB cells per tile
constexpr int STILE = SCAN_TILE;     // cells per tile

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T x)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Exclusive block scan of one value per thread; returns the prefix and the
// block total.
template <typename T, int NT>
__device__ __forceinline__ T block_excl_scan(T v, T& total)
{
    __shared__ T ws[NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const T inc = warp_incl_scan(v);
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < NT / 32 ? ws[lane] : T(0);
        w = warp_incl_scan(w);
        if (lane < NT / 32) ws[lane] = w;
    }
    __syncthreads();
    const T wp = warp ? ws[warp - 1] : T(0);
    total = ws[NT / 32 - 1];
    __syncthreads();
    return wp + inc - v;
}

// Slots needed per cell after the move (particles + new particles) and the
// new particles alone, from the cell's count and part occupancy, packed as
// new << 32 | slots so that one u64 scan gives both offsets.
__device__ __forceinline__ unsigned long long cell_slot_word(const StepArgs& a, uint32_t c)
{
    const uint32_t n = a.ccount[c];
    uint32_t seeds = 0;
    if (a.apply_counts && n > 0) {
        if (a.pp.maxpp < 0) {
            seeds = (uint32_t)a.pp.npart;
        } else {
            for (int w = 0; w < a.pp.occw; ++w)
                seeds += __popcll(a.pp.realmask[w] & ~a.cocc[(size_t)c * a.pp.occw + w]);
        }
    }
    return ((unsigned long long)seeds << 32) | (unsigned long long)(n + seeds);
}

// Pass 1: every cell's slot word (stored to cub) and each tile's sum.
__global__ void __launch_bounds__(SB) k_slots_reduce(StepArgs a, unsigned long long* __restrict__ tiles)
{
    pdl_entry();
    const uint32_t n = (uint32_t)a.mesh.nC;
    unsigned long long s = 0;
#pragma unroll
    for (int k = 0; k < SI; ++k) {
        const uint32_t c = blockIdx.x * STILE + k * SB + threadIdx.x;
        if (c < n) {
            const unsigned long long w = cell_slot_word(a, c);
            a.cub[c] = w;
            s += w;
        }
    }
    unsigned long long total;
    block_excl_scan<unsigned long long, SB>(s, total);
    if (threadIdx.x == 0) tiles[blockIdx.x] = total;
}

// Pass 2: each tile adds the sums of the tiles before it (read by one warp)
// and scans its rows of SB cells; coff[nC] = the grand total.
__global__ void __launch_bounds__(SB) k_slots_down(StepArgs a, const unsigned long long* __restrict__ tiles)
{
    pdl_entry();
    __shared__ unsigned long long carry_s;
    const uint32_t n = (uint32_t)a.mesh.nC;
    if (threadIdx.x < 32) {
        unsigned long long p = 0;
        for (uint32_t t = threadIdx.x; t < blockIdx.x; t += 32) p += tiles[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (threadIdx.x == 0) carry_s = p;
    }
    __syncthreads();
    unsigned long long carry = carry_s;
#pragma unroll 1
    for (int k = 0; k < SI; ++k) {
        const uint32_t i = blockIdx.x * STILE + k * SB + threadIdx.x;
        const unsigned long long v = i < n ? a.cub[i] : 0ull;
        unsigned long long total;
        const unsigned long long p = block_excl_scan<unsigned long long, SB>(v, total);
        if (i < n) a.coff[i] = carry + p;
        if (i == n - 1) a.coff[n] = carry + p + v;
        carry += total;
    }
}

// An uploaded particle set: every particle is an arrival of its cell (the old
// ranges are empty), counted with its part.
template <typename Real, int DIM>
__global__ void k_rekey(StepArgs a)
{
    const uint32_t n = (uint32_t)a.stats->n_slots;
    uint32_t err = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t nloop = (n + stride - 1) / stride * stride;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nloop; i += stride) {
        if (i >= n) continue;
        const uint32_t c = a.S0.cell[i];
        if (c < (uint32_t)a.mesh.nC) {
            a.key[i] = c;
            const uint32_t k = atomicAdd(a.carr + c, 1u);
            if (k < (uint32_t)ARRCAP) a.carrs[(size_t)c * ARRCAP + k] = i;
            else a.next[i] = atomicExch(a.head + c, i);
            Real xi[DIM];
#pragma unroll
            for (int d = 0; d < DIM; ++d) xi[d] = reinterpret_cast<const Real*>(a.T.xi[d])[i];
            const int pe = ext_part<DIM, Real>(xi, a.pp);
            atomicAdd(a.ccount + c, 1u);
            atomicOr(a.cocc + (size_t)c * a.pp.occw + (pe >> 6), 1ull << (pe & 63));
        } else {
            a.key[i] = LOST;
            err = ERR_BAD_CELL;
        }
    }
    err = __reduce_or_sync(0xffffffffu, err);
    if ((threadIdx.x & 31) == 0 && err) atomicOr(&a.stats->error_flags, err);
}

template <typename T>
__global__ void k_fill(T* p, uint32_t n, T v)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_set_state(DevStats* st, long long n, long long next_id, long long add_id)
{
    if (n >= 0) {
        st->n_particles = (unsigned long long)n;
        st->n_slots = (unsigned long long)n;
    }
    if (next_id >= 0) st->next_id = (unsigned)next_id;
    st->next_id += (unsigned)add_id;
}

// Per-cell copy of the nodal velocity (and V - Vold, deltaV of
// src/pfem2particlehandler.cpp:120-124) for every cell vertex, padded to
// VS components (FP64 form).
// The staged copy of V (component-major, ncopy values) written by the kernel
// that reads V first, so a step needs no separate copy.
__device__ __forceinline__ void copy_v(const double* __restrict__ V, double* __restrict__ Vcopy, size_t ncopy)
{
    if (!Vcopy) return;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < ncopy; i += (size_t)gridDim.x * blockDim.x)
        Vcopy[i] = V[i];
}

template <int DIM, typename Real>
__global__ void k_cell_v(const double* __restrict__ V, const double* __restrict__ Vold, const int32_t* __restrict__ cd,
                         int nC, int nD, Real* __restrict__ Vc, Real* __restrict__ dVc, double* __restrict__ Vcopy,
                         size_t ncopy)
{
    pdl_entry();
    copy_v(V, Vcopy, ncopy);
    constexpr int NV = 1 << DIM, VS = Dims<DIM>::VS;
    const int total = nC * NV;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int dof = __ldg(cd + t);
#pragma unroll
        for (int d = 0; d < VS; ++d) {
            const double v = d < DIM ? V[(size_t)d * nD + dof] : 0.0;
            Vc[(size_t)t * VS + d] = (Real)v;
            if (Vold) {
                const double dv = d < DIM ? v - Vold[(size_t)d * nD + dof] : 0.0;
                dVc[(size_t)t * VS + d] = (Real)dv;
            }
        }
    }
}

// FP32 form: per-cell polynomial of the velocity field, one thread per cell
// (a warp reads 32 consecutive cells' vertex values: coalesced on structured
// numberings).  b_k = nested differences of the vertex values (bit d of k
// selects xi_d); on affine cells mapped to reference space, w_k = J^-1 b_k,
// with the cell's exact FP64 inverse.  The increment record (V - Vold) stays
// in physical space.
template <int DIM>
__device__ __forceinline__ void moebius(double (*f)[DIM])
{
    constexpr int NV = 1 << DIM;
#pragma unroll
    for (int b = 0; b < DIM; ++b)
#pragma unroll
        for (int k = NV - 1; k >= 0; --k)
            if ((k >> b) & 1)
#pragma unroll
                for (int d = 0; d < DIM; ++d) f[k][d] = f[k][d] - f[k ^ (1 << b)][d];
}

template <int DIM>
__device__ __forceinline__ void store_rec(float* r, const float* w, float flag)
{
    constexpr int F4 = Dims<DIM>::REC4, NW = (1 << DIM) * DIM;
    float4* q = reinterpret_cast<float4*>(r);
#pragma unroll
    for (int k = 0; k < F4; ++k) {
        float t[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int i = 4 * k + j;
            t[j] = i < NW ? w[i < NW ? i : 0] : (i == NW ? flag : 0.0f);
        }
        q[k] = make_float4(t[0], t[1], t[2], t[3]);
    }
}

// One thread per cell, tiles of REC_TILE consecutive cells per block: the
// records are built in shared memory and written back as contiguous float4
// rows (the per-cell 112-byte records would otherwise be stored at a 112-byte
// stride, half sectors per instruction).
constexpr int REC_TILE = 128;

template <int DIM>
__global__ void __launch_bounds__(REC_TILE, 4) k_cell_rec32(const double* __restrict__ V, const double* __restrict__ Vold,
                                                         const int32_t* __restrict__ cd, const double* __restrict__ aff,
                                                         const float* __restrict__ jinv32, int nC, int nD,
                                                         float* __restrict__ vrec, float* __restrict__ dvrec,
                                                         double* __restrict__ Vcopy, size_t ncopy)
{
    constexpr int NV = 1 << DIM, F = Dims<DIM>::REC4 * 4, F4 = Dims<DIM>::REC4, AFF = Dims<DIM>::AFF;
    __shared__ __align__(16) float rec_s[2][REC_TILE * F];
    // the first tile's cell DoFs are mesh data, which no kernel of the step
    // writes: loaded before the wait on the previous kernel, so only the
    // velocity loads remain after it (the copy of V goes last)
    const int cf = blockIdx.x * REC_TILE + threadIdx.x;
    int dof0[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) dof0[k] = cf < nC ? __ldg(cd + (size_t)cf * NV + k) : 0;
    pdl_entry();
    for (int c0 = blockIdx.x * REC_TILE; c0 < nC; c0 += gridDim.x * REC_TILE) {
        const int c = c0 + threadIdx.x;
        if (c < nC) {
            int dof[NV];
#pragma unroll
            for (int k = 0; k < NV; ++k) dof[k] = c == cf ? dof0[k] : __ldg(cd + (size_t)c * NV + k);
            double f[NV][DIM], g[NV][DIM];
#pragma unroll
            for (int k = 0; k < NV; ++k)
#pragma unroll
                for (int d = 0; d < DIM; ++d) {
                    f[k][d] = __ldg(V + (size_t)d * nD + dof[k]);
                    g[k][d] = Vold ? f[k][d] - __ldg(Vold + (size_t)d * nD + dof[k]) : 0.0;
                }
            moebius<DIM>(f);
            const bool affine = __ldg(jinv32 + (size_t)c * Dims<DIM>::JS + DIM * DIM) != 0.0f;
            float w[NV * DIM];
            if (affine) {
                double A[DIM][DIM];
#pragma unroll
                for (int d = 0; d < DIM; ++d)
#pragma unroll
                    for (int e = 0; e < DIM; ++e) A[d][e] = __ldg(aff + (size_t)c * AFF + d * DIM + e);
#pragma unroll
                for (int k = 0; k < NV; ++k)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        double t = 0.0;
#pragma unroll
                        for (int e = 0; e < DIM; ++e) t += A[d][e] * f[k][e];
                        w[k * DIM + d] = (float)t;
                    }
            } else {
#pragma unroll
                for (int k = 0; k < NV; ++k)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) w[k * DIM + d] = (float)f[k][d];
            }
            store_rec<DIM>(&rec_s[0][threadIdx.x * F], w, affine ? 1.0f : 0.0f);
            if (Vold) {
                moebius<DIM>(g);
#pragma unroll
                for (int k = 0; k < NV; ++k)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) w[k * DIM + d] = (float)g[k][d];
                store_rec<DIM>(&rec_s[1][threadIdx.x * F], w, 0.0f);
            }
        }
        __syncthreads();
        const int ncell = nC - c0 < REC_TILE ? nC - c0 : REC_TILE;
        const float4* s0 = reinterpret_cast<const float4*>(rec_s[0]);
        const float4* s1 = reinterpret_cast<const float4*>(rec_s[1]);
        float4* d0 = reinterpret_cast<float4*>(vrec + (size_t)c0 * F);
        float4* d1 = reinterpret_cast<float4*>(dvrec + (size_t)c0 * F);
        for (int j = threadIdx.x; j < ncell * F4; j += REC_TILE) {
            d0[j] = s0[j];
            if (Vold) d1[j] = s1[j];
        }
        __syncthreads();
    }
    copy_v(V, Vcopy, ncopy);
}

int grid_for(const void* k, int threads) { return occupancy_grid(k, threads); }

}  // namespace

int launch_slots_scan(const StepArgs& a, unsigned long long* tiles, cudaStream_t s)
{
    const uint32_t ntiles = ((uint32_t)a.mesh.nC + STILE - 1) / STILE;
    const int r0 = launch_pdl(k_slots_reduce, (int)ntiles, SB, 0, s, a, tiles);
    const int r1 = launch_pdl(k_slots_down, (int)ntiles, SB, 0, s, a, (const unsigned long long*)tiles);
    if (r0 < 0 || r1 < 0) return -1;
    return 2;
}

int launch_rekey(int dim, int prec, const StepArgs& a, cudaStream_t s)
{
    if (prec == 0 && dim == 2) k_rekey<double, 2><<<grid_for((const void*)k_rekey<double, 2>, 256), 256, 0, s>>>(a);
    else if (prec == 0) k_rekey<double, 3><<<grid_for((const void*)k_rekey<double, 3>, 256), 256, 0, s>>>(a);
    else if (dim == 2) k_rekey<float, 2><<<grid_for((const void*)k_rekey<float, 2>, 256), 256, 0, s>>>(a);
    else k_rekey<float, 3><<<grid_for((const void*)k_rekey<float, 3>, 256), 256, 0, s>>>(a);
    return 1;
}

int launch_fill_u32(uint32_t* p, uint32_t n, uint32_t v, cudaStream_t s)
{
    k_fill<uint32_t><<<grid_for((const void*)k_fill<uint32_t>, 256), 256, 0, s>>>(p, n, v);
    return 1;
}


int launch_set_state(DevStats* st, long long n, long long next_id, long long add_id, cudaStream_t s)
{
    k_set_state<<<1, 1, 0, s>>>(st, n, next_id, add_id);
    return 1;
}

int launch_cell_v(int dim, int prec, const double* V, const double* Vold, const int32_t* cd, int nC, int nD, void* Vc,
                  void* dVc, double* Vcopy, cudaStream_t s)
{
    const size_t nc = Vcopy ? (size_t)dim * nD : 0;
    const int total = nC * (1 << dim);
    const int g = (total + 255) / 256 < 8192 ? (total + 255) / 256 : 8192;
    const int grid = g > 0 ? g : 1;
    if (dim == 2 && prec == 0) return launch_pdl(k_cell_v<2, double>, grid, 256, 0, s, V, Vold, cd, nC, nD, (double*)Vc, (double*)dVc, Vcopy, nc);
    if (dim == 3 && prec == 0) return launch_pdl(k_cell_v<3, double>, grid, 256, 0, s, V, Vold, cd, nC, nD, (double*)Vc, (double*)dVc, Vcopy, nc);
    if (dim == 2) return launch_pdl(k_cell_v<2, float>, grid, 256, 0, s, V, Vold, cd, nC, nD, (float*)Vc, (float*)dVc, Vcopy, nc);
    return launch_pdl(k_cell_v<3, float>, grid, 256, 0, s, V, Vold, cd, nC, nD, (float*)Vc, (float*)dVc, Vcopy, nc);
    return 1;
}

// Non-finite entries of an uploaded host vector (16-byte aligned, n doubles):
// any sets *flag, a mapped host word the caller cleared.  One pass over the
// vector in HBM replaces a host scan of it.
__global__ void k_nonfinite(const double* __restrict__ v, size_t n, unsigned* flag)
{
    bool bad = false;
    const size_t stride = (size_t)gridDim.x * blockDim.x, t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const double2* v2 = reinterpret_cast<const double2*>(v);
    for (size_t i = t0; i < n / 2; i += stride) {
        const double2 q = v2[i];
        bad = bad || !isfinite(q.x) || !isfinite(q.y);
    }
    if (t0 == 0 && (n & 1)) bad = bad || !isfinite(v[n - 1]);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) *reinterpret_cast<volatile unsigned*>(flag) = 1u;
}

int launch_nonfinite(const double* v, size_t n, unsigned* flag, cudaStream_t s)
{
    const size_t g = (n / 2 + 255) / 256;
    const int grid = g < 1 ? 1 : (g > 148 * 8 ? 148 * 8 : (int)g);
    k_nonfinite<<<grid, 256, 0, s>>>(v, n, flag);
    return 1;
}

int launch_cell_rec32(int dim, const double* V, const double* Vold, const int32_t* cd, const double* aff,
                      const float* jinv32, int nC, int nD, float* vrec, float* dvrec, double* Vcopy, cudaStream_t s)
{
    const size_t nc = Vcopy ? (size_t)dim * nD : 0;
    const int g = (nC + REC_TILE - 1) / REC_TILE;
    const int grid = g < 1 ? 1 : g;
    if (dim == 2) return launch_pdl(k_cell_rec32<2>, grid, REC_TILE, 0, s, V, Vold, cd, aff, jinv32, nC, nD, vrec, dvrec, Vcopy, nc);
    return launch_pdl(k_cell_rec32<3>, grid, REC_TILE, 0, s, V, Vold, cd, aff, jinv32, nC, nD, vrec, dvrec, Vcopy, nc);
    return 1;
}

}  // namespace pfem2
