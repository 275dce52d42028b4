// FP64 form (the plain form): compiled with --fmad=false so its arithmetic is
// the reference's own, rounding for rounding.  Also hosts the per-cell
// geometry set-up (vertex coordinates, inverse affine approximation, FP32
// multilinear coefficients) shared by both forms.
#include "advect.cuh"
#include "cellwork.cuh"
#include "launch.h"
#include "shard.cuh"

namespace pfem2 {

namespace {

template <int DIM>
__global__ void k_cell_setup(int nC, const double* __restrict__ verts, const int32_t* __restrict__ cv,
                             double* __restrict__ cellX, double* __restrict__ aff, float* __restrict__ geo32,
                             float* __restrict__ jinv32, uint32_t* __restrict__ twisted)
{
    constexpr int NV = 1 << DIM, GS = Dims<DIM>::GEO, JS = Dims<DIM>::JS;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nC; c += gridDim.x * blockDim.x) {
        double X[NV][DIM];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            const int32_t v = cv[(size_t)c * NV + i];
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                X[i][d] = verts[(size_t)v * DIM + d];
                cellX[((size_t)c * NV + i) * DIM + d] = X[i][d];
            }
        }
        affine_setup64<DIM>(X, aff + (size_t)c * Dims<DIM>::AFF);
        // nested forward differences: Y[k] = Delta^k X (Moebius coefficients)
        double Y[NV][DIM];
#pragma unroll
        for (int i = 0; i < NV; ++i)
#pragma unroll
            for (int d = 0; d < DIM; ++d) Y[i][d] = X[i][d];
#pragma unroll
        for (int b = 0; b < DIM; ++b)
#pragma unroll
            for (int i = NV - 1; i >= 0; --i)
                if ((i >> b) & 1)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) Y[i][d] = Y[i][d] - Y[i ^ (1 << b)][d];
        bool affine = true;
        float* g = geo32 + (size_t)c * GS;
#pragma unroll
        for (int k = 1; k < NV; ++k)
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                g[(k - 1) * DIM + d] = (float)Y[k][d];
                if (__popc(k) >= 2 && Y[k][d] != 0.0) affine = false;
            }
        for (int k = (NV - 1) * DIM; k < GS - 1; ++k) g[k] = 0.0f;
        g[GS - 1] = affine ? 1.0f : 0.0f;
        // inverse Jacobian at the cell centre (exact for affine cells)
        double J[DIM][DIM], Ji[DIM][DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            if (DIM == 2) {
                J[d][0] = Y[1][d] + 0.5 * Y[3][d];
                J[d][1] = Y[2][d] + 0.5 * Y[3][d];
            } else {
                J[d][0] = Y[1][d] + 0.5 * Y[3][d] + 0.5 * Y[5 % NV][d] + 0.25 * Y[7 % NV][d];
                J[d][1] = Y[2][d] + 0.5 * Y[3][d] + 0.5 * Y[6 % NV][d] + 0.25 * Y[7 % NV][d];
                J[d][DIM - 1] = Y[4 % NV][d] + 0.5 * Y[5 % NV][d] + 0.5 * Y[6 % NV][d] + 0.25 * Y[7 % NV][d];
            }
        }
        invert64<DIM>(J, Ji);
        float* jj = jinv32 + (size_t)c * JS;
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int q = 0; q < DIM; ++q) jj[r * DIM + q] = (float)Ji[r][q];
        for (int k = DIM * DIM; k < JS; ++k) jj[k] = 0.0f;
        jj[DIM * DIM] = affine ? 1.0f : 0.0f;
        if (!affine) atomicAdd(twisted, 1u);
    }
}

int grid_of(const void* k, int threads) { return occupancy_grid(k, threads); }

template <int DIM>
int seed_t(const StepArgs& a, uint32_t* cs, cudaStream_t s)
{
    k_seed<DIM, double><<<grid_of((const void*)k_seed<DIM, double>, 256), 256, 0, s>>>(a, cs);
    return 1;
}

}  // namespace

int launch_cell_setup(int dim, int nC, const double* verts, const int32_t* cv, double* cellX, double* aff,
                      float* geo32, float* jinv32, uint32_t* twisted, cudaStream_t s)
{
    const int grid = (nC + 127) / 128;
    if (dim == 2) k_cell_setup<2><<<grid, 128, 0, s>>>(nC, verts, cv, cellX, aff, geo32, jinv32, twisted);
    else k_cell_setup<3><<<grid, 128, 0, s>>>(nC, verts, cv, cellX, aff, geo32, jinv32, twisted);
    return 1;
}

// FP64 launchers (called through the precision-dispatching launchers below)
int launch64_seed(int dim, const StepArgs& a, uint32_t* cs, cudaStream_t s)
{
    return dim == 2 ? seed_t<2>(a, cs, s) : seed_t<3>(a, cs, s);
}

#define PFEM2_GRID(kern, thr) occupancy_grid((const void*)(kern), (thr))

template <typename K>
static int smem_grid(K kernel, int threads, int smem)
{
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
    return sms * (per > 0 ? per : 1);
}

// RK: the midpoint sub-step (params.integrator = PFEM2GPU_RK2), compiled as
// its own kernels so that the Euler ones carry no trace of it.
template <int DIM, bool RK>
static int advect_t(const StepArgs& a, cudaStream_t s)
{
    const int smem = 2 * (int)sizeof(AdvStage<DIM, double, ADV64_CH>);
    static const int grid = smem_grid(k_advect64<DIM, RK>, 256, smem);
    return launch_pdl(k_advect64<DIM, RK>, grid, 256, smem, s, a);
}

template <int DIM, bool RK>
static int search_t(const StepArgs& a, cudaStream_t s)
{
    return launch_pdl(k_search64<DIM, RK>, PFEM2_GRID((k_search64<DIM, RK>), 128), 128, 0, s, a);
}

int launch64_advect(int dim, const StepArgs& a, cudaStream_t s)
{
    if (a.pp.rk2) return dim == 2 ? advect_t<2, true>(a, s) : advect_t<3, true>(a, s);
    return dim == 2 ? advect_t<2, false>(a, s) : advect_t<3, false>(a, s);
}

int launch64_cross(int dim, const StepArgs& a, cudaStream_t s)
{
    if (a.pp.rk2) return dim == 2 ? search_t<2, true>(a, s) : search_t<3, true>(a, s);
    return dim == 2 ? search_t<2, false>(a, s) : search_t<3, false>(a, s);
}

template <int DIM, int CHC>
static int write_c(const StepArgs& a, cudaStream_t s)
{
    const int smem = WR_WARPS * (int)sizeof(WrWarp<DIM, double>);
    // bulk-copy staging where a chunk of cells at the seeding density fits the stage
    if (CHC * a.pp.npart <= WrCfg<DIM, double>::UCAP) {
        static const int grid = smem_grid(k_write<DIM, double, true, CHC>, WR_WARPS * 32, smem);
        return launch_pdl(k_write<DIM, double, true, CHC>, grid, WR_WARPS * 32, smem, s, a);
    }
    static const int grid = smem_grid(k_write<DIM, double, false, CHC>, WR_WARPS * 32, smem);
    return launch_pdl(k_write<DIM, double, false, CHC>, grid, WR_WARPS * 32, smem, s, a);
}

// Chunks of 4 cells on affine meshes; of 2 on the others (graded and
// unstructured meshes, whose cells differ most in particles and arrivals:
// smaller chunks spread the busiest cells over more warps).
template <int DIM>
static int write_t(const StepArgs& a, cudaStream_t s)
{
    if (a.mesh.all_affine) return write_c<DIM, WrCfg<DIM, double>::CHC>(a, s);
    return write_c<DIM, WrCfg<DIM, double>::CHC_UNEVEN>(a, s);
}

int launch64_write(int dim, const StepArgs& a, cudaStream_t s)
{
    return dim == 2 ? write_t<2>(a, s) : write_t<3>(a, s);
}

int launch64_partials(int dim, const StepArgs& a, const uint32_t* cs, cudaStream_t s)
{
    if (dim == 2) k_partials<2, double><<<PFEM2_GRID((k_partials<2, double>), CELL_WARPS * 32), CELL_WARPS * 32, 0, s>>>(a, cs);
    else k_partials<3, double><<<PFEM2_GRID((k_partials<3, double>), CELL_WARPS * 32), CELL_WARPS * 32, 0, s>>>(a, cs);
    return 1;
}

int launch64_correct(int dim, const StepArgs& a, cudaStream_t s)
{
    if (dim == 2) k_correct<2, double><<<PFEM2_GRID((k_correct<2, double>), 256), 256, 0, s>>>(a);
    else k_correct<3, double><<<PFEM2_GRID((k_correct<3, double>), 256), 256, 0, s>>>(a);
    return 1;
}

int launch64_gather(int dim, const StepArgs& a, int keep, cudaStream_t s)
{
    if (dim == 2) return launch_pdl(k_gather<2, double>, PFEM2_GRID((k_gather<2, double>), 256), 256, 0, s, a, keep);
    return launch_pdl(k_gather<3, double>, PFEM2_GRID((k_gather<3, double>), 256), 256, 0, s, a, keep);
    return 1;
}

int launch64_pack_output(int dim, const StepArgs& a, const uint32_t* slot, uint32_t n, float* out, cudaStream_t s)
{
    if (dim == 2) k_pack_output<2, double><<<PFEM2_GRID((k_pack_output<2, double>), 256), 256, 0, s>>>(a, slot, n, out);
    else k_pack_output<3, double><<<PFEM2_GRID((k_pack_output<3, double>), 256), 256, 0, s>>>(a, slot, n, out);
    return 1;
}

// ---------------------------------------------------------------------------
// Vertex -> cell map on the device (initialize_maps,
// src/pfem2particlehandler.cpp:320-324: GridTools::vertex_to_cell_map and
// vertex_to_cell_centers_directions): per vertex the cells around it in
// ascending order, each with the unit direction from the vertex to the cell
// centre, the same FP64 operations as the host builder (this file is
// compiled with --fmad=false).
// ---------------------------------------------------------------------------
namespace {

// A cell's vertex that appears earlier in the same cell is not counted again.
template <int DIM>
__device__ __forceinline__ bool first_in_cell(const int32_t* __restrict__ cv, int c, int i)
{
    constexpr int NV = 1 << DIM;
    const int32_t v = cv[(size_t)c * NV + i];
    for (int j = 0; j < i; ++j)
        if (cv[(size_t)c * NV + j] == v) return false;
    return true;
}

template <int DIM>
__global__ void k_v2c_count(int nC, const int32_t* __restrict__ cv, uint32_t* __restrict__ cnt)
{
    constexpr int NV = 1 << DIM;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nC * NV;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / NV), i = (int)(t % NV);
        if (first_in_cell<DIM>(cv, c, i)) atomicAdd(cnt + cv[t], 1u);
    }
}

template <int DIM>
__global__ void k_v2c_place(int nC, const int32_t* __restrict__ cv, const uint32_t* __restrict__ off,
                            uint32_t* __restrict__ fill, int32_t* __restrict__ cells)
{
    constexpr int NV = 1 << DIM;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nC * NV;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / NV), i = (int)(t % NV);
        if (!first_in_cell<DIM>(cv, c, i)) continue;
        const int32_t v = cv[t];
        cells[off[v] + atomicAdd(fill + v, 1u)] = c;
    }
}

// Per vertex: its cells in ascending order, then the unit directions.
template <int DIM>
__global__ void k_v2c_finish(int nV, const double* __restrict__ verts, const int32_t* __restrict__ cv,
                             const uint32_t* __restrict__ off, int32_t* __restrict__ cells, double* __restrict__ dirs)
{
    constexpr int NV = 1 << DIM;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nV; v += gridDim.x * blockDim.x) {
        const uint32_t b = off[v], e = off[v + 1];
        for (uint32_t k = b + 1; k < e; ++k) {  // insertion sort (a handful of cells)
            const int32_t x = cells[k];
            uint32_t j = k;
            while (j > b && cells[j - 1] > x) {
                cells[j] = cells[j - 1];
                --j;
            }
            cells[j] = x;
        }
        for (uint32_t k = b; k < e; ++k) {
            const int c = cells[k];
            double dir[DIM], s = 0.0;
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                double ctr = 0.0;
#pragma unroll
                for (int i = 0; i < NV; ++i) ctr = ctr + verts[(size_t)cv[(size_t)c * NV + i] * DIM + d];
                ctr = ctr / (double)NV;
                dir[d] = ctr - verts[(size_t)v * DIM + d];
            }
#pragma unroll
            for (int d = 0; d < DIM; ++d) s = s + dir[d] * dir[d];
            s = sqrt(s);
#pragma unroll
            for (int d = 0; d < DIM; ++d) dirs[(size_t)k * DIM + d] = dir[d] / s;
        }
    }
}

// dof -> (cell, local vertex) entries k = cell * NV + i, ascending per dof.
__global__ void k_d2c_count(long long nE, const int32_t* __restrict__ cd, uint32_t* __restrict__ cnt)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nE; k += (long long)gridDim.x * blockDim.x)
        atomicAdd(cnt + cd[k], 1u);
}

__global__ void k_d2c_place(long long nE, const int32_t* __restrict__ cd, const uint32_t* __restrict__ off,
                            uint32_t* __restrict__ fill, int32_t* __restrict__ ent)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nE; k += (long long)gridDim.x * blockDim.x) {
        const int32_t d = cd[k];
        ent[off[d] + atomicAdd(fill + d, 1u)] = (int32_t)k;
    }
}

__global__ void k_d2c_sort(int nD, const uint32_t* __restrict__ off, int32_t* __restrict__ ent)
{
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nD; d += gridDim.x * blockDim.x) {
        const uint32_t b = off[d], e = off[d + 1];
        for (uint32_t k = b + 1; k < e; ++k) {
            const int32_t x = ent[k];
            uint32_t j = k;
            while (j > b && ent[j - 1] > x) {
                ent[j] = ent[j - 1];
                --j;
            }
            ent[j] = x;
        }
    }
}

}  // namespace

int launch_d2c_count(long long nE, const int32_t* cd, uint32_t* cnt, cudaStream_t s)
{
    k_d2c_count<<<PFEM2_GRID(k_d2c_count, 256), 256, 0, s>>>(nE, cd, cnt);
    return 1;
}

int launch_d2c_build(long long nE, int nD, const int32_t* cd, const uint32_t* off, uint32_t* fill, int32_t* ent,
                     cudaStream_t s)
{
    k_d2c_place<<<PFEM2_GRID(k_d2c_place, 256), 256, 0, s>>>(nE, cd, off, fill, ent);
    k_d2c_sort<<<PFEM2_GRID(k_d2c_sort, 128), 128, 0, s>>>(nD, off, ent);
    return 2;
}

// Counts per vertex into cnt (zeroed by the caller), then, once the caller
// has their exclusive scan in off (nV + 1), the ascending lists and the
// directions; fill (nV, zeroed) is the placement counter.
int launch_v2c_count(int dim, int nC, const int32_t* cv, uint32_t* cnt, cudaStream_t s)
{
    if (dim == 2) k_v2c_count<2><<<PFEM2_GRID(k_v2c_count<2>, 256), 256, 0, s>>>(nC, cv, cnt);
    else k_v2c_count<3><<<PFEM2_GRID(k_v2c_count<3>, 256), 256, 0, s>>>(nC, cv, cnt);
    return 1;
}

int launch_v2c_build(int dim, int nC, int nV, const double* verts, const int32_t* cv, const uint32_t* off,
                     uint32_t* fill, int32_t* cells, double* dirs, cudaStream_t s)
{
    if (dim == 2) {
        k_v2c_place<2><<<PFEM2_GRID(k_v2c_place<2>, 256), 256, 0, s>>>(nC, cv, off, fill, cells);
        k_v2c_finish<2><<<PFEM2_GRID(k_v2c_finish<2>, 128), 128, 0, s>>>(nV, verts, cv, off, cells, dirs);
    } else {
        k_v2c_place<3><<<PFEM2_GRID(k_v2c_place<3>, 256), 256, 0, s>>>(nC, cv, off, fill, cells);
        k_v2c_finish<3><<<PFEM2_GRID(k_v2c_finish<3>, 128), 128, 0, s>>>(nV, verts, cv, off, cells, dirs);
    }
    return 2;
}

static int grid_n64(size_t n, int threads)
{
    const size_t g = (n + threads - 1) / threads;
    return (int)(g < 1 ? 1 : g > 148 * 32 ? 148 * 32 : g);
}

int launch64_outbox(const StepArgs& a, uint32_t* out_i, uint32_t* out_c, uint32_t* n_out, uint32_t cap, cudaStream_t s)
{
    k_outbox<double><<<grid_n64((size_t)a.mesh.nC, 256), 256, 0, s>>>(a, out_i, out_c, n_out, cap);
    return 1;
}

int launch64_outbox_pack(int dim, const StepArgs& a, const uint32_t* out_i, const uint32_t* out_c, uint32_t n,
                         uint32_t* id, int32_t* cell, double* x, double* xi, double* v, cudaStream_t s)
{
    if (dim == 2) k_outbox_pack<2, double><<<grid_n64(n, 256), 256, 0, s>>>(a, out_i, out_c, n, id, cell, x, xi, v);
    else k_outbox_pack<3, double><<<grid_n64(n, 256), 256, 0, s>>>(a, out_i, out_c, n, id, cell, x, xi, v);
    return 1;
}

int launch64_inbox(int dim, const StepArgs& a, uint32_t n, uint32_t base, const uint32_t* id, const int32_t* cell,
                   const double* x, const double* xi, const double* v, cudaStream_t s)
{
    if (dim == 2) k_inbox<2, double><<<grid_n64(n, 256), 256, 0, s>>>(a, n, base, id, cell, x, xi, v);
    else k_inbox<3, double><<<grid_n64(n, 256), 256, 0, s>>>(a, n, base, id, cell, x, xi, v);
    return 1;
}

int launch64_partials_io(void* partials, int pw, uint32_t n, const int32_t* cells, double* buf, int to_buf,
                         cudaStream_t s)
{
    k_partials_io<double><<<grid_n64((size_t)n * pw, 256), 256, 0, s>>>(partials, pw, n, cells, buf, to_buf);
    return 1;
}

}  // namespace pfem2
