// FP32 form: FP32 reference coordinates and velocities, compensated FP32
// projection sums; FP64 only for face-crossing relocation and the final DoF
// division.  Also the precision-dispatching launchers.
#include "advect.cuh"
#include "cellwork.cuh"
#include "launch.h"

namespace pfem2 {

int launch64_seed(int dim, const StepArgs& a, uint32_t* cs, cudaStream_t s);
int launch64_advect(int dim, const StepArgs& a, cudaStream_t s);
int launch64_write(int dim, const StepArgs& a, cudaStream_t s);
int launch64_partials(int dim, const StepArgs& a, const uint32_t* cs, cudaStream_t s);
int launch64_correct(int dim, const StepArgs& a, cudaStream_t s);
int launch64_gather(int dim, const StepArgs& a, int keep, cudaStream_t s);

#define PFEM2_GRID(kern, thr) occupancy_grid((const void*)(kern), (thr))
#define CELL_THREADS (CELL_WARPS * 32)

int launch_seed(int dim, int prec, const StepArgs& a, uint32_t* cs, cudaStream_t s)
{
    if (prec == 0) return launch64_seed(dim, a, cs, s);
    if (dim == 2) k_seed<2, float><<<PFEM2_GRID((k_seed<2, float>), 256), 256, 0, s>>>(a, cs);
    else k_seed<3, float><<<PFEM2_GRID((k_seed<3, float>), 256), 256, 0, s>>>(a, cs);
    return 1;
}

int launch_advect(int dim, int prec, const StepArgs& a, cudaStream_t s)
{
    if (prec == 0) return launch64_advect(dim, a, s);
    if (dim == 2) {
        k_advect32<2><<<PFEM2_GRID(k_advect32<2>, 256), 256, 0, s>>>(a);
        k_cross32<2><<<PFEM2_GRID(k_cross32<2>, 128), 128, 0, s>>>(a);
    } else {
        k_advect32<3><<<PFEM2_GRID(k_advect32<3>, 256), 256, 0, s>>>(a);
        k_cross32<3><<<PFEM2_GRID(k_cross32<3>, 128), 128, 0, s>>>(a);
    }
    return 2;
}

template <int DIM>
static int write32_t_grid()
{
    const int smem = (int)sizeof(WriteSmem<float>);
    static int grid = 0;
    if (!grid) {
        cudaFuncSetAttribute(k_write<DIM, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_write<DIM, float>, WR_WARPS * 32, smem);
        grid = sms * (per > 0 ? per : 1);
    }
    return grid;
}

template <int DIM>
static int write32_t(const StepArgs& a, cudaStream_t s)
{
    const int smem = (int)sizeof(WriteSmem<float>);
    StepArgs args = a;
    void* params[] = {&args};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_write<DIM, float>, dim3(write32_t_grid<DIM>()),
                                                      dim3(WR_WARPS * 32), params, smem, s);
    return e == cudaSuccess ? 1 : -1;
}

int launch_write(int dim, int prec, const StepArgs& a, cudaStream_t s)
{
    if (prec == 0) return launch64_write(dim, a, s);
    return dim == 2 ? write32_t<2>(a, s) : write32_t<3>(a, s);
}

int launch64_write_grid(int dim);

int write_grid(int dim, int prec)
{
    if (prec == 0) return launch64_write_grid(dim);
    return dim == 2 ? write32_t_grid<2>() : write32_t_grid<3>();
}

int launch_partials(int dim, int prec, const StepArgs& a, const uint32_t* cs, cudaStream_t s)
{
    if (prec == 0) return launch64_partials(dim, a, cs, s);
    if (dim == 2) k_partials<2, float><<<PFEM2_GRID((k_partials<2, float>), CELL_THREADS), CELL_THREADS, 0, s>>>(a, cs);
    else k_partials<3, float><<<PFEM2_GRID((k_partials<3, float>), CELL_THREADS), CELL_THREADS, 0, s>>>(a, cs);
    return 1;
}

int launch_correct(int dim, int prec, const StepArgs& a, cudaStream_t s)
{
    if (prec == 0) return launch64_correct(dim, a, s);
    if (dim == 2) k_correct<2, float><<<PFEM2_GRID((k_correct<2, float>), 256), 256, 0, s>>>(a);
    else k_correct<3, float><<<PFEM2_GRID((k_correct<3, float>), 256), 256, 0, s>>>(a);
    return 1;
}

int launch_gather(int dim, int prec, const StepArgs& a, int keep, cudaStream_t s)
{
    if (prec == 0) return launch64_gather(dim, a, keep, s);
    if (dim == 2) k_gather<2, float><<<PFEM2_GRID((k_gather<2, float>), 256), 256, 0, s>>>(a, keep);
    else k_gather<3, float><<<PFEM2_GRID((k_gather<3, float>), 256), 256, 0, s>>>(a, keep);
    return 1;
}

int launch_positions32(int dim, const StepArgs& a, double* xout, cudaStream_t s)
{
    if (dim == 2) k_positions32<2><<<PFEM2_GRID(k_positions32<2>, 256), 256, 0, s>>>(a, xout);
    else k_positions32<3><<<PFEM2_GRID(k_positions32<3>, 256), 256, 0, s>>>(a, xout);
    return 1;
}

}  // namespace pfem2
