// FP64 form (the plain form): compiled with --fmad=false so its arithmetic is
// the reference's own, rounding for rounding.  Also hosts the per-cell
// geometry set-up (vertex coordinates, inverse affine approximation, FP32
// multilinear coefficients) shared by both forms.
#include "advect.cuh"
#include "cellwork.cuh"
#include "launch.h"

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

template <int DIM>
static int advect_t(const StepArgs& a, cudaStream_t s)
{
    const int smem = 2 * (int)sizeof(AdvStage<DIM, double, ADV64_CH>);
    static const int grid = smem_grid(k_advect64<DIM>, 256, smem);
    return launch_pdl(k_advect64<DIM>, grid, 256, smem, s, a);
    return 1;
}

int launch64_advect(int dim, const StepArgs& a, cudaStream_t s)
{
    return dim == 2 ? advect_t<2>(a, s) : advect_t<3>(a, s);
}

int launch64_cross(int dim, const StepArgs& a, cudaStream_t s)
{
    if (dim == 2) return launch_pdl(k_search64<2>, PFEM2_GRID(k_search64<2>, 128), 128, 0, s, a);
    return launch_pdl(k_search64<3>, PFEM2_GRID(k_search64<3>, 128), 128, 0, s, a);
    return 1;
}

template <int DIM>
static int write_t(const StepArgs& a, cudaStream_t s)
{
    const int smem = WR_WARPS * (int)sizeof(WrWarp<DIM, double>);
    static const int grid = smem_grid(k_write<DIM, double>, WR_WARPS * 32, smem);
    return launch_pdl(k_write<DIM, double>, grid, WR_WARPS * 32, smem, s, a);
    return 1;
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

}  // namespace pfem2
