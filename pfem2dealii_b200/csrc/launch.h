// Host-side launchers of the particle kernels (one translation unit per
// precision form plus the integer kernels).  Each launcher returns the number
// of kernels it enqueued on the stream.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <unordered_map>

#include "common.cuh"

namespace pfem2 {

// Grid of a grid-stride kernel: every SM filled to its occupancy limit.
inline int occupancy_grid(const void* kernel, int threads, size_t smem = 0)
{
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(kernel);
    if (it != cache.end()) return it->second;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
    const int g = sms * (per > 0 ? per : 1);
    cache[kernel] = g;
    return g;
}

// Launch with programmatic dependent launch (the kernel calls pdl_entry()
// first): it may be scheduled while the previous kernel drains, which hides
// the launch gap between the dependent kernels of a step.  Returns 1 (one
// kernel) or -1 when the launch was refused.
template <typename... KArgs, typename... Args>
inline int launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, ((KArgs)args)...) == cudaSuccess ? 1 : -1;
}

// kernels_f64.cu / kernels_f32.cu (prec: 0 = FP64 form, 1 = FP32 form)
int launch_cell_setup(int dim, int nC, const double* verts, const int32_t* cv, double* cellX, double* aff,
                      float* geo32, float* jinv32, uint32_t* twisted, cudaStream_t s);
int launch_seed(int dim, int prec, const StepArgs& a, uint32_t* cell_start, cudaStream_t s);
int launch_advect(int dim, int prec, const StepArgs& a, cudaStream_t s);
int launch_cross(int dim, int prec, const StepArgs& a, cudaStream_t s);
int launch_write(int dim, int prec, const StepArgs& a, cudaStream_t s);
int launch_partials(int dim, int prec, const StepArgs& a, const uint32_t* cell_start, cudaStream_t s);
int launch_correct(int dim, int prec, const StepArgs& a, cudaStream_t s);
int launch_gather(int dim, int prec, const StepArgs& a, int keep_empty, cudaStream_t s);
int launch_positions32(int dim, const StepArgs& a, double* xout, cudaStream_t s);
// shard.cuh: the exchange of a partitioned move, and partial sums to and from doubles
int launch_outbox(int prec, const StepArgs& a, uint32_t* out_i, uint32_t* out_c, uint32_t* n_out, uint32_t cap,
                  cudaStream_t s);
int launch_outbox_pack(int dim, int prec, const StepArgs& a, const uint32_t* out_i, const uint32_t* out_c, uint32_t n,
                       uint32_t* id, int32_t* cell, double* x, double* xi, double* v, cudaStream_t s);
int launch_inbox(int dim, int prec, const StepArgs& a, uint32_t n, uint32_t base, const uint32_t* id,
                 const int32_t* cell, const double* x, const double* xi, const double* v, cudaStream_t s);
int launch_partials_io(int prec, void* partials, int pw, uint32_t n, const int32_t* cells, double* buf, int to_buf,
                       cudaStream_t s);
int launch_pack_output(int dim, int prec, const StepArgs& a, const uint32_t* slot, uint32_t n, float* out,
                       cudaStream_t s);

// kernels_f64.cu: vertex -> cell and dof -> cell maps built on the device
int launch_v2c_count(int dim, int nC, const int32_t* cv, uint32_t* cnt, cudaStream_t s);
int launch_v2c_build(int dim, int nC, int nV, const double* verts, const int32_t* cv, const uint32_t* off,
                     uint32_t* fill, int32_t* cells, double* dirs, cudaStream_t s);
int launch_d2c_count(long long nE, const int32_t* cd, uint32_t* cnt, cudaStream_t s);
int launch_d2c_build(long long nE, int nD, const int32_t* cd, const uint32_t* off, uint32_t* fill, int32_t* ent,
                     cudaStream_t s);

// fem.cu: the Q1 FEM systems' volume terms
int launch_fem_pattern(int dim, const FemArgs& f, bool fill, uint32_t* count, unsigned* err, cudaStream_t s);
int launch_fem_assemble(int dim, int sys, const FemArgs& f, cudaStream_t s);
int launch_fem_contrib(int dim, const FemArgs& f, bool fill, uint32_t* count, cudaStream_t s);
int launch_fem_velocity_bc(int dim, const FemArgs& f, const uint8_t* dmask, const int32_t* face_id, const double* P,
                           double* local, int32_t* last_id, int n_ids, const int32_t* ids, const double* id_vel,
                           double coeff, double* value, int32_t* flag, cudaStream_t s);
int launch_fem_constrain(int nD, long long nnz, int nm, int ns, const int32_t* row_ptr, const int32_t* cols,
                         const int32_t* con_idx, int n_con, const double* g, double* A, double* rhs, cudaStream_t s);

// misc.cu
constexpr int SCAN_TILE = 512;        // cells per tile of the slot-offset scan
constexpr int SCAN_MAX_TILES = 16384; // tile sums the scan buffer holds
// Slots per cell (count + new particles) into cub, their exclusive scan into
// coff (coff[nC] = totals); two kernels.
int launch_slots_scan(const StepArgs& a, unsigned long long* tiles, cudaStream_t s);
int launch_rekey(int dim, int prec, const StepArgs& a, cudaStream_t s);
int launch_fill_u32(uint32_t* p, uint32_t n, uint32_t v, cudaStream_t s);
int launch_set_state(DevStats* st, long long n, long long next_id, long long add_id, cudaStream_t s);
int launch_cell_v(int dim, int prec, const double* V, const double* Vold, const int32_t* cd, int nC, int nD, void* Vc,
                  void* dVc, double* Vcopy, cudaStream_t s);
int launch_nonfinite(const double* v, size_t n, unsigned* flag, cudaStream_t s);
int launch_cell_rec32(int dim, const double* V, const double* Vold, const int32_t* cd, const double* aff,
                      const float* jinv32, int nC, int nD, float* vrec, float* dvrec, double* Vcopy,
                      cudaStream_t s);

// window_f64.cu / window_f32.cu: the differentiated window (window.cuh)
struct WinArgs;
int launch_win_compact(const uint32_t* cells, uint32_t ns, uint32_t nC, uint32_t* tsum, uint32_t* slot,
                       cudaStream_t s);
int launch_win_scan(const uint32_t* in, uint32_t n, uint32_t* tsum, uint32_t* out, cudaStream_t s);
int launch_win_init(int dim, int prec, const WinArgs& w, const double* v0, cudaStream_t s);
int launch_win_forward(int dim, int prec, const WinArgs& w, cudaStream_t s);
int launch_win_project(int dim, int prec, const WinArgs& w, cudaStream_t s);
int launch_win_backward(int dim, int prec, const WinArgs& w, const double* gU, double* g_v0, double* gV,
                        double* gVold, int rec_seg, cudaStream_t s);
int launch_win_wcell(int dim, const WinArgs& w, const double* Vcell, double* Wout, cudaStream_t s);

}  // namespace pfem2
