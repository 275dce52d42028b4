// Small kernels of the particle cycle: arrival-list set-up for an uploaded
// particle set, finalisation of the step's counters, and the staging of nodal
// velocities (component-major doubles, one vector per component as the
// reference's std::array<TrilinosWrappers::MPI::Vector,dim>) into per-cell
// vertex records the particle kernels read.
#include "launch.h"

namespace pfem2 {

namespace {

// Links every particle of an uploaded set into the arrival list of its cell
// (the old ranges are empty, so the write pass sorts them all).
__global__ void k_rekey(StepArgs a)
{
    const uint32_t n = (uint32_t)a.stats->n_particles;
    uint32_t err = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t nloop = (n + stride - 1) / stride * stride;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nloop; i += stride) {
        if (i >= n) continue;
        const uint32_t c = a.S0.cell[i];
        if (c < (uint32_t)a.mesh.nC) {
            a.key[i] = c;
            a.next[i] = atomicExch(a.head + c, i);
        } else {
            a.key[i] = LOST;
            err = ERR_BAD_CELL;
        }
    }
    err = __reduce_or_sync(0xffffffffu, err);
    if ((threadIdx.x & 31) == 0 && err) atomicOr(&a.stats->error_flags, err);
}

__global__ void k_fill_u32(uint32_t* p, uint32_t n, uint32_t v)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_finalize(StepArgs a, int count_step)
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
    a.cs_new[a.mesh.nC] = total;
}

__global__ void k_set_state(DevStats* st, long long n, long long next_id, long long add_id)
{
    if (n >= 0) st->n_particles = (unsigned long long)n;
    if (next_id >= 0) st->next_id = (unsigned)next_id;
    st->next_id += (unsigned)add_id;
}

// Per-cell copy of the nodal velocity (and V - Vold, deltaV of
// src/pfem2particlehandler.cpp:120-124) for every cell vertex, padded to
// VS components, in the form's precision.
template <int DIM, typename Real>
__global__ void k_cell_v(const double* __restrict__ V, const double* __restrict__ Vold, const int32_t* __restrict__ cd,
                         int nC, int nD, Real* __restrict__ Vc, Real* __restrict__ dVc)
{
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

// FP32 form: per-cell polynomial of the velocity field, b_k = nested
// differences of the vertex values (bit d of k selects xi_d).  On affine
// cells the coefficients are mapped to reference space, w_k = J^-1 b_k, with
// the cell's exact FP64 inverse Jacobian, so that d xi = dt w(xi).
template <int DIM>
__global__ void k_cell_rec32(const double* __restrict__ V, const double* __restrict__ Vold,
                             const int32_t* __restrict__ cd, const double* __restrict__ aff,
                             const float* __restrict__ jinv32, int nC, int nD, float* __restrict__ vrec,
                             float* __restrict__ dvrec)
{
    constexpr int NV = 1 << DIM, F = Dims<DIM>::REC4 * 4, AFF = Dims<DIM>::AFF;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nC; c += gridDim.x * blockDim.x) {
        double f[NV][DIM], g[NV][DIM];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            const int dof = __ldg(cd + (size_t)c * NV + i);
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                f[i][d] = V[(size_t)d * nD + dof];
                g[i][d] = Vold ? f[i][d] - Vold[(size_t)d * nD + dof] : 0.0;
            }
        }
#pragma unroll
        for (int b = 0; b < DIM; ++b)
#pragma unroll
            for (int i = NV - 1; i >= 0; --i)
                if ((i >> b) & 1)
#pragma unroll
                    for (int d = 0; d < DIM; ++d) {
                        f[i][d] -= f[i ^ (1 << b)][d];
                        g[i][d] -= g[i ^ (1 << b)][d];
                    }
        const bool affine = jinv32[(size_t)c * Dims<DIM>::JS + DIM * DIM] != 0.0f;
        float* r = vrec + (size_t)c * F;
#pragma unroll
        for (int k = 0; k < NV; ++k)
#pragma unroll
            for (int d = 0; d < DIM; ++d) {
                double w = f[k][d];
                if (affine) {
                    w = 0.0;
#pragma unroll
                    for (int e = 0; e < DIM; ++e) w += aff[(size_t)c * AFF + d * DIM + e] * f[k][e];
                }
                r[k * DIM + d] = (float)w;
            }
        for (int k = NV * DIM; k < F; ++k) r[k] = 0.0f;
        r[NV * DIM] = affine ? 1.0f : 0.0f;
        if (Vold) {
            float* q = dvrec + (size_t)c * F;
#pragma unroll
            for (int k = 0; k < NV; ++k)
#pragma unroll
                for (int d = 0; d < DIM; ++d) q[k * DIM + d] = (float)g[k][d];
            for (int k = NV * DIM; k < F; ++k) q[k] = 0.0f;
        }
    }
}

int grid_for(const void* k, int threads) { return occupancy_grid(k, threads); }

}  // namespace

int launch_cell_rec32(int dim, const double* V, const double* Vold, const int32_t* cd, const double* aff,
                      const float* jinv32, int nC, int nD, float* vrec, float* dvrec, cudaStream_t s)
{
    const int g = (nC + 127) / 128 < 8192 ? (nC + 127) / 128 : 8192;
    const int grid = g > 0 ? g : 1;
    if (dim == 2) k_cell_rec32<2><<<grid, 128, 0, s>>>(V, Vold, cd, aff, jinv32, nC, nD, vrec, dvrec);
    else k_cell_rec32<3><<<grid, 128, 0, s>>>(V, Vold, cd, aff, jinv32, nC, nD, vrec, dvrec);
    return 1;
}

int launch_rekey(const StepArgs& a, cudaStream_t s)
{
    k_rekey<<<grid_for((const void*)k_rekey, 256), 256, 0, s>>>(a);
    return 1;
}

int launch_fill_u32(uint32_t* p, uint32_t n, uint32_t v, cudaStream_t s)
{
    k_fill_u32<<<grid_for((const void*)k_fill_u32, 256), 256, 0, s>>>(p, n, v);
    return 1;
}

int launch_finalize(const StepArgs& a, int count_step, cudaStream_t s)
{
    k_finalize<<<1, 1, 0, s>>>(a, count_step);
    return 1;
}

int launch_set_state(DevStats* st, long long n, long long next_id, long long add_id, cudaStream_t s)
{
    k_set_state<<<1, 1, 0, s>>>(st, n, next_id, add_id);
    return 1;
}

int launch_cell_v(int dim, int prec, const double* V, const double* Vold, const int32_t* cd, int nC, int nD, void* Vc,
                  void* dVc, cudaStream_t s)
{
    const int total = nC * (1 << dim);
    const int g = (total + 255) / 256 < 8192 ? (total + 255) / 256 : 8192;
    const int grid = g > 0 ? g : 1;
    if (dim == 2 && prec == 0) k_cell_v<2, double><<<grid, 256, 0, s>>>(V, Vold, cd, nC, nD, (double*)Vc, (double*)dVc);
    else if (dim == 3 && prec == 0) k_cell_v<3, double><<<grid, 256, 0, s>>>(V, Vold, cd, nC, nD, (double*)Vc, (double*)dVc);
    else if (dim == 2) k_cell_v<2, float><<<grid, 256, 0, s>>>(V, Vold, cd, nC, nD, (float*)Vc, (float*)dVc);
    else k_cell_v<3, float><<<grid, 256, 0, s>>>(V, Vold, cd, nC, nD, (float*)Vc, (float*)dVc);
    return 1;
}

}  // namespace pfem2
