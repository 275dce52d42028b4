// pfem2gpu_project_noalloc: projection of a caller-owned particle set onto the
// mesh DoFs that allocates no device memory.
//
// The work memory is one file-scope __device__ array (na_scratch), whose
// address is taken with cudaGetSymbolAddress on every call, with the call's
// device current, under a per-device lock: the address belongs to the context
// that is current, and a cached one would go stale after cudaDeviceReset or
// under another context on the same device.  A call validates its sizes against the
// array first and returns PFEM2GPU_ERR_SCRATCH when the mesh does not fit.
// Nothing in the array needs to hold any value on entry: the call zeroes the
// counters it accumulates into (the status block and the per-DoF entry
// counts) with cudaMemsetAsync before its first kernel, and every other word
// is written before it is read.  The per-device lock is held until the call's
// kernels have finished (the call ends by synchronising its stream), so calls
// from several host threads on one device run one after the other instead of
// sharing the array; calls on different devices use different arrays.
//
// Arithmetic: the per-cell sums are the FP64 form's own device code
// (partials_of_range), compiled with --fmad=false as the FP64 form is; the
// per-DoF gather adds the cell entries in ascending (cell, vertex) order, the
// order of the handle's DoF -> cell map (rebuilt here on the device by a
// counting sort), and divides once, as the handle's gather does.  So the
// result equals pfem2gpu_project of an FP64 handle holding the same
// particles in the same order bit for bit.  Every kernel of this file has
// internal linkage: no launch elsewhere in the library can resolve to this
// file's device image (and with it, to the scratch array).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "advect.cuh"
#include "cellwork.cuh"
#include "launch.h"
#include "pfem2gpu.h"

namespace pfem2 {
namespace {

constexpr size_t NA_BYTES = PFEM2GPU_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char na_scratch[NA_BYTES];

constexpr uint32_t NA_BAD_DOF = 1u;    // a cell_dofs entry outside [0, n_dofs)
constexpr uint32_t NA_BAD_CELL = 2u;   // a particle cell outside [0, n_cells)
constexpr uint32_t NA_UNSORTED = 4u;   // particle cells not in ascending order

constexpr int NA_THREADS = 256;
constexpr int NA_PER = 8;                       // scan items per thread
constexpr int NA_TILE = NA_THREADS * NA_PER;    // scan items per block
constexpr int NA_MAX_DEVICES = 64;

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

struct Layout {
    size_t stats, cnt, off, tsum, ent, partials, total;
};

Layout layout(int dim, int64_t nC, int64_t nD)
{
    const int64_t NV = 1 << dim, PW = NV * 4, ntiles = (nD + NA_TILE - 1) / NA_TILE;
    Layout L;
    L.stats = 0;
    L.cnt = al256(sizeof(DevStats));  // status block and counts are zeroed together
    L.off = L.cnt + al256(4 * nD);
    L.tsum = L.off + al256(4 * (nD + 1));
    L.ent = L.tsum + al256(4 * ntiles);
    L.partials = L.ent + al256(4 * nC * NV);
    L.total = L.partials + al256(8 * nC * PW);
    return L;
}

// Per-DoF entry counts; particle cell range and order checks.
__global__ void k_na_count(int nC, int NV, int nD, const int32_t* cell_dofs, int64_t np, const int32_t* pcell,
                           int32_t* cnt, DevStats* st)
{
    const int64_t nE = (int64_t)nC * NV, n = nE > np ? nE : np;
    uint32_t err = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < nE) {
            const int32_t d = cell_dofs[i];
            if (d < 0 || d >= nD) err |= NA_BAD_DOF;
            else atomicAdd(&cnt[d], 1);
        }
        if (i < np) {
            const int32_t c = pcell[i];
            if (c < 0 || c >= nC) err |= NA_BAD_CELL;
            else if (i > 0 && pcell[i - 1] > c) err |= NA_UNSORTED;
        }
    }
    err = __reduce_or_sync(0xffffffffu, err);
    if ((threadIdx.x & 31) == 0 && err) atomicOr(&st->error_flags, err);
}

// Exclusive block scan of one value per thread; returns the block total.
__device__ int32_t block_scan(int32_t v, int32_t& excl)
{
    __shared__ int32_t wsum[NA_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    int32_t base = 0, total = 0;
    for (int w = 0; w < NA_THREADS / 32; ++w) {
        if (w < warp) base += wsum[w];
        total += wsum[w];
    }
    __syncthreads();
    excl = base + inc - v;
    return total;
}

__global__ void k_na_scan_tiles(const int32_t* cnt, int nD, int32_t* tsum)
{
    const int64_t i0 = (int64_t)blockIdx.x * NA_TILE + threadIdx.x * NA_PER;
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < NA_PER; ++k)
        if (i0 + k < nD) s += cnt[i0 + k];
    int32_t excl;
    const int32_t total = block_scan(s, excl);
    if (threadIdx.x == 0) tsum[blockIdx.x] = total;
}

// One block: exclusive scan of the tile sums, in place.
__global__ void k_na_scan_top(int32_t* tsum, int ntiles)
{
    __shared__ int32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b = 0; b < ntiles; b += NA_THREADS) {
        const int i = b + threadIdx.x;
        const int32_t v = i < ntiles ? tsum[i] : 0;
        int32_t excl;
        const int32_t total = block_scan(v, excl);
        if (i < ntiles) tsum[i] = carry + excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void k_na_scan_apply(const int32_t* cnt, int nD, const int32_t* tsum, int32_t* off)
{
    const int64_t i0 = (int64_t)blockIdx.x * NA_TILE + threadIdx.x * NA_PER;
    int32_t v[NA_PER], s = 0;
#pragma unroll
    for (int k = 0; k < NA_PER; ++k) {
        v[k] = i0 + k < nD ? cnt[i0 + k] : 0;
        s += v[k];
    }
    int32_t excl;
    block_scan(s, excl);
    int32_t run = tsum[blockIdx.x] + excl;
#pragma unroll
    for (int k = 0; k < NA_PER; ++k) {
        if (i0 + k < nD) off[i0 + k] = run;
        run += v[k];
        if (i0 + k == nD - 1) off[nD] = run;
    }
}

// Entries (cell * NV + vertex) into their DoF's range; leaves cnt at zero.
__global__ void k_na_fill(int nC, int NV, int nD, const int32_t* cell_dofs, int32_t* cnt, const int32_t* off,
                          int32_t* ent)
{
    const int64_t nE = (int64_t)nC * NV;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nE; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = cell_dofs[e];
        if (d < 0 || d >= nD) continue;
        const int32_t k = atomicSub(&cnt[d], 1) - 1;
        ent[off[d] + k] = (int32_t)e;
    }
}

// Each DoF's entries in ascending order (insertion sort; a DoF has a few).
__global__ void k_na_sort(int nD, const int32_t* off, int32_t* ent)
{
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nD; d += gridDim.x * blockDim.x) {
        const int32_t b = off[d], e = off[d + 1];
        for (int32_t i = b + 1; i < e; ++i) {
            const int32_t x = ent[i];
            int32_t j = i - 1;
            while (j >= b && ent[j] > x) {
                ent[j + 1] = ent[j];
                --j;
            }
            ent[j + 1] = x;
        }
    }
}

__device__ __forceinline__ int64_t lower_bound(const int32_t* a, int64_t n, int32_t x)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t m = (lo + hi) >> 1;
        if (a[m] < x) lo = m + 1;
        else hi = m;
    }
    return lo;
}

// Warp per cell: the cell's particle range by binary search in the sorted
// cell array, then the FP64 form's per-cell sums over it, in order.
// Skipped, like the gather, when k_na_count flagged bad input.
template <int DIM>
__global__ void __launch_bounds__(CELL_WARPS * 32) k_na_partials(StepArgs a, PartState S, int64_t np,
                                                                 const DevStats* st)
{
    __shared__ __align__(16) double tr_s[CELL_WARPS][32][TRW];
    if (*(volatile const unsigned int*)&st->error_flags) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int32_t* pc = reinterpret_cast<const int32_t*>(S.cell);
    for (int c = blockIdx.x * CELL_WARPS + warp; c < a.mesh.nC; c += gridDim.x * CELL_WARPS) {
        const int64_t b = lower_bound(pc, np, c);
        int64_t e = lower_bound(pc, np, c + 1);
        if (e < b) e = b;  // unsorted input (reported by k_na_count): keep the range inside the arrays
        partials_of_range<DIM, double>(a, S, (uint32_t)c, (uint32_t)b, (uint32_t)(e - b), tr_s[warp], lane);
    }
}

// V_d = sum num_d / sum den over the DoF's entries in ascending order; 0/0
// gives NaN, or the value on entry under empty_dof_policy 1.  Bad input
// flagged by k_na_count leaves V untouched.
template <int DIM>
__global__ void k_na_gather(int nD, const int32_t* off, const int32_t* ent, const double* P, int keep_empty,
                            double* V, DevStats* st)
{
    constexpr int NV = 1 << DIM, PW = Dims<DIM>::PW;
    if (*(volatile const unsigned int*)&st->error_flags) return;
    unsigned long long empty = 0;
    const int stride = gridDim.x * blockDim.x;
    const int nloop = (nD + stride - 1) / stride * stride;
    for (int dof = blockIdx.x * blockDim.x + threadIdx.x; dof < nloop; dof += stride) {
        if (dof >= nD) continue;
        double num[DIM], den = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) num[d] = 0.0;
        for (int32_t k = off[dof]; k < off[dof + 1]; ++k) {
            const int32_t en = ent[k];
            const double* src = P + (size_t)(en / NV) * PW + (en % NV) * 4;
#pragma unroll
            for (int d = 0; d < DIM; ++d) num[d] = num[d] + src[d];
            den = den + src[DIM];
        }
        if (den == 0.0) empty++;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            double r = num[d] / den;
            if (den == 0.0 && keep_empty) r = V[(size_t)d * nD + dof];
            V[(size_t)d * nD + dof] = r;
        }
    }
    empty = warp_sum_u64(empty);
    if ((threadIdx.x & 31) == 0 && empty) atomicAdd(&st->nan_dofs, empty);
}

std::mutex na_mutex[NA_MAX_DEVICES];

int grid_for(int64_t n, int threads)
{
    const int64_t g = (n + threads - 1) / threads;
    return (int)(g < 1 ? 1 : g > 148 * 16 ? 148 * 16 : g);
}

}  // namespace
}  // namespace pfem2

using namespace pfem2;

extern "C" int pfem2gpu_project_noalloc(int dim, int32_t n_cells, int32_t n_dofs, const int32_t* d_cell_dofs,
                                        int64_t n_particles, const int32_t* d_cell, const double* d_xi,
                                        const double* d_v, int empty_dof_policy, double* d_V_out,
                                        int64_t* n_empty_dofs, void* stream)
{
    if (dim != 2 && dim != 3) return PFEM2GPU_ERR_ARG;
    const int NV = 1 << dim;
    if (n_cells <= 0 || n_dofs <= 0 || n_particles < 0 || n_particles > INT32_MAX) return PFEM2GPU_ERR_ARG;
    if ((int64_t)n_cells * NV > INT32_MAX) return PFEM2GPU_ERR_ARG;
    if (!d_cell_dofs || !d_V_out || (n_particles > 0 && (!d_cell || !d_xi || !d_v))) return PFEM2GPU_ERR_ARG;
    if (empty_dof_policy != 0 && empty_dof_policy != 1) return PFEM2GPU_ERR_ARG;
    const Layout L = layout(dim, n_cells, n_dofs);
    if (L.total > NA_BYTES) return PFEM2GPU_ERR_SCRATCH;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // an error left pending by earlier work of this host thread is not this call's
    (void)cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PFEM2GPU_ERR_NODEVICE;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return PFEM2GPU_ERR_ARG;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return PFEM2GPU_ERR_CUDA;
    if (cap != cudaStreamCaptureStatusNone) return PFEM2GPU_ERR_STATE;  // the call synchronises its stream

    std::lock_guard<std::mutex> lock(na_mutex[dev]);
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, na_scratch) != cudaSuccess || !p) return PFEM2GPU_ERR_CUDA;
    unsigned char* base = static_cast<unsigned char*>(p);
    DevStats* st = reinterpret_cast<DevStats*>(base + L.stats);
    int32_t* cnt = reinterpret_cast<int32_t*>(base + L.cnt);
    int32_t* off = reinterpret_cast<int32_t*>(base + L.off);
    int32_t* tsum = reinterpret_cast<int32_t*>(base + L.tsum);
    int32_t* ent = reinterpret_cast<int32_t*>(base + L.ent);
    double* partials = reinterpret_cast<double*>(base + L.partials);
    const int64_t nE = (int64_t)n_cells * NV;
    const int ntiles = (int)((n_dofs + NA_TILE - 1) / NA_TILE);
    // once work is queued, every return waits for it, so that the lock covers
    // the work that uses the shared array
    auto fail_after_enqueue = [&](int code) {
        cudaStreamSynchronize(s);
        return code;
    };

    if (cudaMemsetAsync(base, 0, L.off, s) != cudaSuccess) return fail_after_enqueue(PFEM2GPU_ERR_CUDA);
    const int64_t ncount = nE > n_particles ? nE : n_particles;
    k_na_count<<<grid_for(ncount, NA_THREADS), NA_THREADS, 0, s>>>(n_cells, NV, n_dofs, d_cell_dofs, n_particles,
                                                                    d_cell, cnt, st);
    k_na_scan_tiles<<<ntiles, NA_THREADS, 0, s>>>(cnt, n_dofs, tsum);
    k_na_scan_top<<<1, NA_THREADS, 0, s>>>(tsum, ntiles);
    k_na_scan_apply<<<ntiles, NA_THREADS, 0, s>>>(cnt, n_dofs, tsum, off);
    k_na_fill<<<grid_for(nE, NA_THREADS), NA_THREADS, 0, s>>>(n_cells, NV, n_dofs, d_cell_dofs, cnt, off, ent);
    k_na_sort<<<grid_for(n_dofs, NA_THREADS), NA_THREADS, 0, s>>>(n_dofs, off, ent);

    StepArgs a{};  // what partials_of_range reads: the cell count and the partials array
    a.mesh.nC = n_cells;
    a.partials = partials;
    PartState S{};
    S.cell = reinterpret_cast<uint32_t*>(const_cast<int32_t*>(d_cell));
    for (int d = 0; d < dim; ++d) {
        S.xi[d] = const_cast<double*>(d_xi) + (size_t)d * n_particles;
        S.v[d] = const_cast<double*>(d_v) + (size_t)d * n_particles;
    }
    const int cgrid = grid_for((int64_t)n_cells, CELL_WARPS);
    if (dim == 2) {
        k_na_partials<2><<<cgrid, CELL_WARPS * 32, 0, s>>>(a, S, n_particles, st);
        k_na_gather<2><<<grid_for(n_dofs, 256), 256, 0, s>>>(n_dofs, off, ent, partials, empty_dof_policy, d_V_out,
                                                              st);
    } else {
        k_na_partials<3><<<cgrid, CELL_WARPS * 32, 0, s>>>(a, S, n_particles, st);
        k_na_gather<3><<<grid_for(n_dofs, 256), 256, 0, s>>>(n_dofs, off, ent, partials, empty_dof_policy, d_V_out,
                                                              st);
    }
    if (cudaGetLastError() != cudaSuccess) return fail_after_enqueue(PFEM2GPU_ERR_CUDA);
    DevStats h{};
    if (cudaMemcpyAsync(&h, st, sizeof(DevStats), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return fail_after_enqueue(PFEM2GPU_ERR_CUDA);
    if (cudaStreamSynchronize(s) != cudaSuccess) return PFEM2GPU_ERR_CUDA;
    if (h.error_flags) return PFEM2GPU_ERR_ARG;
    if (n_empty_dofs) *n_empty_dofs = (int64_t)h.nan_dofs;
    return PFEM2GPU_OK;
}
