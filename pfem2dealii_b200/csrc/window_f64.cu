// Differentiated window, FP64 form (compiled with --fmad=false, like the
// FP64 particle kernels, so its trajectories are the FP64 form's own), plus
// the form-independent window kernels and the precision-dispatching
// launchers.
#define PFEM2_WINDOW_GENERIC
#include "launch.h"
#include "window.cuh"

namespace pfem2 {

// window_f32.cu
int launch32_win_init(int dim, const WinArgs& w, const double* v0, cudaStream_t s);
int launch32_win_forward(int dim, const WinArgs& w, cudaStream_t s);
int launch32_win_cellsum(int dim, const WinArgs& w, cudaStream_t s);
int launch32_win_bwd(int dim, const WinArgs& w, double* g_v0, int rec_seg, cudaStream_t s);

namespace {

uint32_t tiles_of(uint32_t n) { return (n + WIN_TILE - 1) / WIN_TILE; }

}  // namespace

int launch_win_compact(const uint32_t* cells, uint32_t ns, uint32_t nC, uint32_t* tsum, uint32_t* slot,
                       cudaStream_t s)
{
    const uint32_t nt = tiles_of(ns);
    if (nt == 0) return 0;
    k_win_tilesum<<<nt, 256, 0, s>>>(nullptr, cells, ns, nC, tsum);
    k_win_tilescan<<<1, 1024, 0, s>>>(tsum, nt);
    k_win_apply<<<nt, 256, 0, s>>>(nullptr, cells, ns, nC, tsum, slot);
    return 3;
}

int launch_win_scan(const uint32_t* in, uint32_t n, uint32_t* tsum, uint32_t* out, cudaStream_t s)
{
    const uint32_t nt = tiles_of(n);
    k_win_tilesum<<<nt, 256, 0, s>>>(in, nullptr, n, 0, tsum);
    k_win_tilescan<<<1, 1024, 0, s>>>(tsum, nt);
    k_win_apply<<<nt, 256, 0, s>>>(in, nullptr, n, 0, tsum, out);
    return 3;
}

int launch_win_init(int dim, int prec, const WinArgs& w, const double* v0, cudaStream_t s)
{
    if (prec != 0) return launch32_win_init(dim, w, v0, s);
    if (dim == 2) k_win_init<2, double><<<win_grid(k_win_init<2, double>, 256), 256, 0, s>>>(w, v0);
    else k_win_init<3, double><<<win_grid(k_win_init<3, double>, 256), 256, 0, s>>>(w, v0);
    return 1;
}

int launch_win_forward(int dim, int prec, const WinArgs& w, cudaStream_t s)
{
    if (prec != 0) return launch32_win_forward(dim, w, s);
    return dim == 2 ? win_forward_t<2, double>(w, s) : win_forward_t<3, double>(w, s);
}

// Projection of the final state: count, scan, place, per-cell sums, gather.
// ccnt and nempty must be zero on entry.
int launch_win_project(int dim, int prec, const WinArgs& w, cudaStream_t s)
{
    const int nC = w.a.mesh.nC;
    int n = 0;
    k_win_count<<<win_grid(k_win_count, 256), 256, 0, s>>>(w);
    n += 1 + launch_win_scan(w.ccnt, (uint32_t)nC, w.tsum, w.cstart, s);
    cudaMemsetAsync(w.ccnt, 0, (size_t)nC * sizeof(uint32_t), s);
    k_win_place<<<win_grid(k_win_place, 256), 256, 0, s>>>(w);
    n += 1;
    if (prec == 0) {
        if (dim == 2) k_win_cellsum<2, double><<<win_grid(k_win_cellsum<2, double>, CELL_WARPS * 32), CELL_WARPS * 32, 0, s>>>(w);
        else k_win_cellsum<3, double><<<win_grid(k_win_cellsum<3, double>, CELL_WARPS * 32), CELL_WARPS * 32, 0, s>>>(w);
        n += 1;
    } else {
        n += launch32_win_cellsum(dim, w, s);
    }
    if (dim == 2) k_win_gather<2><<<win_grid(k_win_gather<2>, 256), 256, 0, s>>>(w);
    else k_win_gather<3><<<win_grid(k_win_gather<3>, 256), 256, 0, s>>>(w);
    return n + 1;
}

// The FP64 vertices W_i = X_i + h V_i of every cell's sub-step map.
int launch_win_wcell(int dim, const WinArgs& w, const double* Vcell, double* Wout, cudaStream_t s)
{
    if (dim == 2) k_win_wcell<2><<<win_grid(k_win_wcell<2>, 256), 256, 0, s>>>(w, Vcell, Wout);
    else k_win_wcell<3><<<win_grid(k_win_wcell<3>, 256), 256, 0, s>>>(w, Vcell, Wout);
    return 1;
}

// Backward: projection seeds, the segments in reverse, DoF gathers.  gadv,
// gdv and err must be zero on entry.
int launch_win_backward(int dim, int prec, const WinArgs& w, const double* gU, double* g_v0, double* gV,
                        double* gVold, int rec_seg, cudaStream_t s)
{
    int n = 0;
    if (dim == 2) k_win_gseed<2><<<win_grid(k_win_gseed<2>, 256), 256, 0, s>>>(w, gU);
    else k_win_gseed<3><<<win_grid(k_win_gseed<3>, 256), 256, 0, s>>>(w, gU);
    n += 1;
    if (prec == 0)
        n += dim == 2 ? win_backward_t<2, double>(w, g_v0, rec_seg, s) : win_backward_t<3, double>(w, g_v0, rec_seg, s);
    else n += launch32_win_bwd(dim, w, g_v0, rec_seg, s);
    if (dim == 2) k_win_gV<2><<<win_grid(k_win_gV<2>, 256), 256, 0, s>>>(w, gU, gV, gVold);
    else k_win_gV<3><<<win_grid(k_win_gV<3>, 256), 256, 0, s>>>(w, gU, gV, gVold);
    return n + 1;
}

}  // namespace pfem2
