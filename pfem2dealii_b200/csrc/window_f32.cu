// Differentiated window, FP32 form: the FP32 form's trajectories (compiled
// like kernels_f32.cu), FP64 projection sums and FP64 adjoint arithmetic.
#include "launch.h"
#include "window.cuh"

namespace pfem2 {

int launch32_win_init(int dim, const WinArgs& w, const double* v0, cudaStream_t s)
{
    if (dim == 2) k_win_init<2, float><<<win_grid(k_win_init<2, float>, 256), 256, 0, s>>>(w, v0);
    else k_win_init<3, float><<<win_grid(k_win_init<3, float>, 256), 256, 0, s>>>(w, v0);
    return 1;
}

int launch32_win_forward(int dim, const WinArgs& w, cudaStream_t s)
{
    return dim == 2 ? win_forward_t<2, float>(w, s) : win_forward_t<3, float>(w, s);
}

int launch32_win_cellsum(int dim, const WinArgs& w, cudaStream_t s)
{
    if (dim == 2) k_win_cellsum<2, float><<<win_grid(k_win_cellsum<2, float>, CELL_WARPS * 32), CELL_WARPS * 32, 0, s>>>(w);
    else k_win_cellsum<3, float><<<win_grid(k_win_cellsum<3, float>, CELL_WARPS * 32), CELL_WARPS * 32, 0, s>>>(w);
    return 1;
}

int launch32_win_bwd(int dim, const WinArgs& w, double* g_v0, int rec_seg, cudaStream_t s)
{
    return dim == 2 ? win_backward_t<2, float>(w, g_v0, rec_seg, s) : win_backward_t<3, float>(w, g_v0, rec_seg, s);
}

}  // namespace pfem2
