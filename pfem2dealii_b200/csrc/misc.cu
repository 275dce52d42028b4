// Integer kernels of the particle cycle: cell-offset scans, bucketing of the
// advected particles by cell, finalisation of the step's counters, and the
// staging of nodal velocities (component-major doubles, one vector per
// component as the reference's std::array<TrilinosWrappers::MPI::Vector,dim>)
// into the padded per-DoF layout the particle kernels gather from.
#include "launch.h"

namespace pfem2 {

namespace {

constexpr int SB = 256;                 // scan block
constexpr int SI = SCAN_TILE / SB;      // items per thread

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

template <typename T>
__global__ void __launch_bounds__(SB) k_scan_reduce(const T* __restrict__ in, uint32_t n, T* __restrict__ tiles)
{
    const uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x;
    T s = 0;
#pragma unroll
    for (int k = 0; k < SI; ++k) {
        const uint32_t i = base + k * SB;
        if (i < n) s += in[i];
    }
    T total;
    block_excl_scan<T, SB>(s, total);
    if (threadIdx.x == 0) tiles[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(1024) k_scan_top(T* __restrict__ tiles, uint32_t ntiles)
{
    constexpr int PER = SCAN_MAX_TILES / 1024;
    T v[PER], s = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const uint32_t i = threadIdx.x * PER + k;
        v[k] = i < ntiles ? tiles[i] : T(0);
        s += v[k];
    }
    T total;
    T p = block_excl_scan<T, 1024>(s, total);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const uint32_t i = threadIdx.x * PER + k;
        if (i < ntiles) tiles[i] = p;
        p += v[k];
    }
}

// Tile-strided layout: thread t of a tile owns elements t, t+SB, ...; the
// exclusive order inside a tile is therefore (k, t) and is rebuilt by a
// second block scan per item row.
template <typename T>
__global__ void __launch_bounds__(SB) k_scan_down(const T* __restrict__ in, uint32_t n, const T* __restrict__ tiles,
                                                   T* __restrict__ out)
{
    T carry = tiles[blockIdx.x];
#pragma unroll 1
    for (int k = 0; k < SI; ++k) {
        const uint32_t i = blockIdx.x * SCAN_TILE + k * SB + threadIdx.x;
        const T v = i < n ? in[i] : T(0);
        T total;
        const T p = block_excl_scan<T, SB>(v, total);
        if (i < n) out[i] = carry + p;
        if (i == n - 1) out[n] = carry + p + v;
        carry += total;
    }
}

template <typename T>
int scan_impl(const T* in, uint32_t n, T* out, T* tiles, cudaStream_t s)
{
    const uint32_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_reduce<T><<<ntiles, SB, 0, s>>>(in, n, tiles);
    k_scan_top<T><<<1, 1024, 0, s>>>(tiles, ntiles);
    k_scan_down<T><<<ntiles, SB, 0, s>>>(in, n, tiles, out);
    return 3;
}

__global__ void k_bucket(StepArgs a)
{
    const uint32_t n = (uint32_t)a.stats->n_particles;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = a.key[i];
        if (k != LOST) a.idx[a.cell_off[k] + a.slot[i]] = i;
    }
}

// Keys of an uploaded particle set (cells as given, nothing moves).
__global__ void k_rekey(StepArgs a)
{
    const uint32_t n = (uint32_t)a.stats->n_particles;
    uint32_t err = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = a.S0.cell[i];
        if (c < (uint32_t)a.mesh.nC) {
            a.key[i] = c;
            a.slot[i] = atomicAdd(a.cell_count + c, 1u);
        } else {
            a.key[i] = LOST;
            err = ERR_BAD_CELL;
        }
    }
    err = __reduce_or_sync(0xffffffffu, err);
    if ((threadIdx.x & 31) == 0 && err) atomicOr(&a.stats->error_flags, err);
}

__global__ void k_finalize(StepArgs a, uint32_t* cell_start, int count_step)
{
    if (count_step) a.stats->particle_steps += a.stats->n_particles;
    const unsigned long long po = *a.totals;
    uint32_t total = (uint32_t)po;
    const uint32_t seeds = (uint32_t)(po >> 32);
    if (total > a.capacity) {
        a.stats->error_flags |= ERR_CAPACITY;
        total = a.capacity;
    }
    a.stats->n_particles = total;
    a.stats->next_id += seeds;
    a.stats->seeded += seeds;
    cell_start[a.mesh.nC] = total;
}

__global__ void k_set_state(DevStats* st, long long n, long long next_id, long long add_id)
{
    if (n >= 0) st->n_particles = (unsigned long long)n;
    if (next_id >= 0) st->next_id = (unsigned)next_id;
    st->next_id += (unsigned)add_id;
}

template <int DIM, typename Real>
__global__ void k_prep_v(const double* __restrict__ V, const double* __restrict__ Vold, int nD, Real* Vaos,
                         Real* dVaos)
{
    constexpr int VS = Dims<DIM>::VS;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nD; k += gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < VS; ++d) {
            const double v = d < DIM ? V[(size_t)d * nD + k] : 0.0;
            Vaos[(size_t)k * VS + d] = (Real)v;
            if (Vold) {
                // deltaV = V - Vold per DoF (src/pfem2particlehandler.cpp:120-124)
                const double dv = d < DIM ? v - Vold[(size_t)d * nD + k] : 0.0;
                dVaos[(size_t)k * VS + d] = (Real)dv;
            }
        }
    }
}

int grid_for(const void* k, int threads) { return occupancy_grid(k, threads); }

}  // namespace

int launch_scan_u32(const uint32_t* in, uint32_t n, uint32_t* out, uint32_t* tiles, cudaStream_t s)
{
    return scan_impl<uint32_t>(in, n, out, tiles, s);
}

int launch_scan_u64(const unsigned long long* in, uint32_t n, unsigned long long* out, unsigned long long* tiles,
                    cudaStream_t s)
{
    return scan_impl<unsigned long long>(in, n, out, tiles, s);
}

int launch_bucket(const StepArgs& a, cudaStream_t s)
{
    k_bucket<<<grid_for((const void*)k_bucket, 256), 256, 0, s>>>(a);
    return 1;
}

int launch_rekey(const StepArgs& a, cudaStream_t s)
{
    k_rekey<<<grid_for((const void*)k_rekey, 256), 256, 0, s>>>(a);
    return 1;
}

int launch_finalize(const StepArgs& a, uint32_t* cell_start, int count_step, cudaStream_t s)
{
    k_finalize<<<1, 1, 0, s>>>(a, cell_start, count_step);
    return 1;
}

int launch_set_state(DevStats* st, long long n, long long next_id, long long add_id, cudaStream_t s)
{
    k_set_state<<<1, 1, 0, s>>>(st, n, next_id, add_id);
    return 1;
}

int launch_prep_v(int dim, int prec, const double* V, const double* Vold, int nD, void* Vaos, void* dVaos,
                  cudaStream_t s)
{
    const int g = (nD + 255) / 256 < 4096 ? (nD + 255) / 256 : 4096;
    const int grid = g > 0 ? g : 1;
    if (dim == 2 && prec == 0) k_prep_v<2, double><<<grid, 256, 0, s>>>(V, Vold, nD, (double*)Vaos, (double*)dVaos);
    else if (dim == 3 && prec == 0) k_prep_v<3, double><<<grid, 256, 0, s>>>(V, Vold, nD, (double*)Vaos, (double*)dVaos);
    else if (dim == 2) k_prep_v<2, float><<<grid, 256, 0, s>>>(V, Vold, nD, (float*)Vaos, (float*)dVaos);
    else k_prep_v<3, float><<<grid, 256, 0, s>>>(V, Vold, nD, (float*)Vaos, (float*)dVaos);
    return 1;
}

}  // namespace pfem2
