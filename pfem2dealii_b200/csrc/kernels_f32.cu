// FP32 form: FP32 reference coordinates and velocities, compensated FP32
// projection sums; FP64 only for face-crossing relocation and the final DoF
// division.  Also the precision-dispatching launchers.
#include "advect.cuh"
#include "cellwork.cuh"
#include "launch.h"
#include "shard.cuh"

namespace pfem2 {

int launch64_seed(int dim, const StepArgs& a, uint32_t* cs, cudaStream_t s);
int launch64_advect(int dim, const StepArgs& a, cudaStream_t s);
int launch64_cross(int dim, const StepArgs& a, cudaStream_t s);
int launch64_write(int dim, const StepArgs& a, cudaStream_t s);
int launch64_partials(int dim, const StepArgs& a, const uint32_t* cs, cudaStream_t s);
int launch64_correct(int dim, const StepArgs& a, cudaStream_t s);
int launch64_gather(int dim, const StepArgs& a, int keep, cudaStream_t s);
int launch64_outbox(const StepArgs& a, uint32_t* out_i, uint32_t* out_c, uint32_t* n_out, uint32_t cap, cudaStream_t s);
int launch64_outbox_pack(int dim, const StepArgs& a, const uint32_t* out_i, const uint32_t* out_c, uint32_t n,
                         uint32_t* id, int32_t* cell, double* x, double* xi, double* v, cudaStream_t s);
int launch64_inbox(int dim, const StepArgs& a, uint32_t n, uint32_t base, const uint32_t* id, const int32_t* cell,
                   const double* x, const double* xi, const double* v, cudaStream_t s);
int launch64_partials_io(void* partials, int pw, uint32_t n, const int32_t* cells, double* buf, int to_buf,
                         cudaStream_t s);

#define PFEM2_GRID(kern, thr) occupancy_grid((const void*)(kern), (thr))
#define CELL_THREADS (CELL_WARPS * 32)

int launch_seed(int dim, int prec, const StepArgs& a, uint32_t* cs, cudaStream_t s)
{
    if (prec == 0) return launch64_seed(dim, a, cs, s);
    if (dim == 2) k_seed<2, float><<<PFEM2_GRID((k_seed<2, float>), 256), 256, 0, s>>>(a, cs);
    else k_seed<3, float><<<PFEM2_GRID((k_seed<3, float>), 256), 256, 0, s>>>(a, cs);
    return 1;
}

template <typename K>
static int smem_grid32(K kernel, int threads, int smem)
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
static int advect32_t(const StepArgs& a, cudaStream_t s)
{
    const int smem = 2 * (int)(sizeof(AdvStage<DIM, float, ADV_CH>) + sizeof(AdvRecStage<DIM>));
    if (a.mesh.all_affine) {
        static const int grid = smem_grid32(k_advect32<DIM, true, RK>, 256, smem);
        return launch_pdl(k_advect32<DIM, true, RK>, grid, 256, smem, s, a);
    } else {
        static const int grid = smem_grid32(k_advect32<DIM, false, RK>, 256, smem);
        return launch_pdl(k_advect32<DIM, false, RK>, grid, 256, smem, s, a);
    }
}

template <int DIM, bool RK>
static int cross32_t(const StepArgs& a, cudaStream_t s)
{
    if (a.mesh.all_affine)
        return launch_pdl(k_cross32<DIM, true, RK>, PFEM2_GRID((k_cross32<DIM, true, RK>), 128), 128, 0, s, a);
    if constexpr (DIM == 2)
        return launch_pdl(k_cross32_occ<DIM, RK>, PFEM2_GRID((k_cross32_occ<DIM, RK>), 128), 128, 0, s, a);
    else
        return launch_pdl(k_cross32<DIM, false, RK>, PFEM2_GRID((k_cross32<DIM, false, RK>), 128), 128, 0, s, a);
}

int launch_advect(int dim, int prec, const StepArgs& a, cudaStream_t s)
{
    if (prec == 0) return launch64_advect(dim, a, s);
    if (a.pp.rk2) return dim == 2 ? advect32_t<2, true>(a, s) : advect32_t<3, true>(a, s);
    return dim == 2 ? advect32_t<2, false>(a, s) : advect32_t<3, false>(a, s);
}

// The queued face crossers of the advect pass (relocation in FP64).
int launch_cross(int dim, int prec, const StepArgs& a, cudaStream_t s)
{
    if (prec == 0) return launch64_cross(dim, a, s);
    if (a.pp.rk2) return dim == 2 ? cross32_t<2, true>(a, s) : cross32_t<3, true>(a, s);
    return dim == 2 ? cross32_t<2, false>(a, s) : cross32_t<3, false>(a, s);
}

template <int DIM, int CHC>
static int write32_c(const StepArgs& a, cudaStream_t s)
{
    const int smem = WR_WARPS * (int)sizeof(WrWarp<DIM, float>);
    // bulk-copy staging where a chunk of cells at the seeding density fits the stage
    if (CHC * a.pp.npart <= WrCfg<DIM, float>::UCAP) {
        static const int grid = smem_grid32(k_write<DIM, float, true, CHC>, WR_WARPS * 32, smem);
        return launch_pdl(k_write<DIM, float, true, CHC>, grid, WR_WARPS * 32, smem, s, a);
    }
    static const int grid = smem_grid32(k_write<DIM, float, false, CHC>, WR_WARPS * 32, smem);
    return launch_pdl(k_write<DIM, float, false, CHC>, grid, WR_WARPS * 32, smem, s, a);
}

// Chunks of 4 cells on affine meshes; of 2 on the others (graded and
// unstructured meshes, whose cells differ most in particles and arrivals:
// smaller chunks spread the busiest cells over more warps).
template <int DIM>
static int write32_t(const StepArgs& a, cudaStream_t s)
{
    if (a.mesh.all_affine) return write32_c<DIM, WrCfg<DIM, float>::CHC>(a, s);
    return write32_c<DIM, WrCfg<DIM, float>::CHC_UNEVEN>(a, s);
}

int launch_write(int dim, int prec, const StepArgs& a, cudaStream_t s)
{
    if (prec == 0) return launch64_write(dim, a, s);
    return dim == 2 ? write32_t<2>(a, s) : write32_t<3>(a, s);
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
    if (dim == 2) return launch_pdl(k_gather<2, float>, PFEM2_GRID((k_gather<2, float>), 256), 256, 0, s, a, keep);
    return launch_pdl(k_gather<3, float>, PFEM2_GRID((k_gather<3, float>), 256), 256, 0, s, a, keep);
    return 1;
}

int launch64_pack_output(int dim, const StepArgs& a, const uint32_t* slot, uint32_t n, float* out, cudaStream_t s);

int launch_pack_output(int dim, int prec, const StepArgs& a, const uint32_t* slot, uint32_t n, float* out,
                       cudaStream_t s)
{
    if (prec == 0) return launch64_pack_output(dim, a, slot, n, out, s);
    if (dim == 2) k_pack_output<2, float><<<PFEM2_GRID((k_pack_output<2, float>), 256), 256, 0, s>>>(a, slot, n, out);
    else k_pack_output<3, float><<<PFEM2_GRID((k_pack_output<3, float>), 256), 256, 0, s>>>(a, slot, n, out);
    return 1;
}

int launch_positions32(int dim, const StepArgs& a, double* xout, cudaStream_t s)
{
    if (dim == 2) k_positions32<2><<<PFEM2_GRID(k_positions32<2>, 256), 256, 0, s>>>(a, xout);
    else k_positions32<3><<<PFEM2_GRID(k_positions32<3>, 256), 256, 0, s>>>(a, xout);
    return 1;
}

static int grid_n(size_t n, int threads)
{
    const size_t g = (n + threads - 1) / threads;
    return (int)(g < 1 ? 1 : g > 148 * 32 ? 148 * 32 : g);
}

int launch_outbox(int prec, const StepArgs& a, uint32_t* out_i, uint32_t* out_c, uint32_t* n_out, uint32_t cap,
                  cudaStream_t s)
{
    if (prec == 0) return launch64_outbox(a, out_i, out_c, n_out, cap, s);
    k_outbox<float><<<grid_n((size_t)a.mesh.nC, 256), 256, 0, s>>>(a, out_i, out_c, n_out, cap);
    return 1;
}

int launch_outbox_pack(int dim, int prec, const StepArgs& a, const uint32_t* out_i, const uint32_t* out_c, uint32_t n,
                       uint32_t* id, int32_t* cell, double* x, double* xi, double* v, cudaStream_t s)
{
    if (prec == 0) return launch64_outbox_pack(dim, a, out_i, out_c, n, id, cell, x, xi, v, s);
    if (dim == 2) k_outbox_pack<2, float><<<grid_n(n, 256), 256, 0, s>>>(a, out_i, out_c, n, id, cell, x, xi, v);
    else k_outbox_pack<3, float><<<grid_n(n, 256), 256, 0, s>>>(a, out_i, out_c, n, id, cell, x, xi, v);
    return 1;
}

int launch_inbox(int dim, int prec, const StepArgs& a, uint32_t n, uint32_t base, const uint32_t* id,
                 const int32_t* cell, const double* x, const double* xi, const double* v, cudaStream_t s)
{
    if (prec == 0) return launch64_inbox(dim, a, n, base, id, cell, x, xi, v, s);
    if (dim == 2) k_inbox<2, float><<<grid_n(n, 256), 256, 0, s>>>(a, n, base, id, cell, x, xi, v);
    else k_inbox<3, float><<<grid_n(n, 256), 256, 0, s>>>(a, n, base, id, cell, x, xi, v);
    return 1;
}

int launch_partials_io(int prec, void* partials, int pw, uint32_t n, const int32_t* cells, double* buf, int to_buf,
                       cudaStream_t s)
{
    if (prec == 0) return launch64_partials_io(partials, pw, n, cells, buf, to_buf, s);
    k_partials_io<float><<<grid_n((size_t)n * pw, 256), 256, 0, s>>>(partials, pw, n, cells, buf, to_buf);
    return 1;
}

}  // namespace pfem2
