// Cell-range partitions of one mesh over several handles (one per GPU): the
// kernels around the exchange of particles that cross into another
// partition during a move.
//
// The reference distributes cells over MPI ranks (p4est) and sends the
// particles found in another rank's cells after each relocation
// (send_recv_particles, src/pfem2particlehandler.cpp:480-502,507-618).  Here
// every handle holds the whole mesh and the whole FEM velocity, so a particle
// finishes all its sub-steps on the handle it started on; the particles that
// end the move in another partition's cells are taken out once, before count
// correction, and enter the owner's count correction as arrivals.  Each
// cell's particles and their order (stayers, arrivals by key, seeds by part)
// are then those of an unpartitioned run.
#pragma once

#include "advect.cuh"
#include "cellwork.cuh"

namespace pfem2 {

// The particles whose move ended in a cell outside [cbeg, cend): every such
// cell's arrivals (its slots, then its overflow list) go to the outbox as
// (particle index, cell); the cell's counters are reset, so the write pass
// finds it empty.  One thread per cell; outbox order is not defined (the
// receiver orders arrivals by key).
template <typename Real>  // one instance per form's translation unit
__global__ void k_outbox(StepArgs a, uint32_t* out_i, uint32_t* out_c, uint32_t* n_out, uint32_t out_cap)
{
    const uint32_t nC = (uint32_t)a.mesh.nC;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nC; c += gridDim.x * blockDim.x) {
        if (c >= (uint32_t)a.cbeg && c < (uint32_t)a.cend) continue;
        const uint32_t na = a.carr[c];
        if (na == 0) continue;
        const uint32_t base = atomicAdd(n_out, na);
        uint32_t p = a.head[c];
        for (uint32_t k = 0; k < na; ++k) {
            uint32_t i;
            if (k < (uint32_t)ARRCAP) {
                i = a.carrs[(size_t)c * ARRCAP + k];
            } else {
                if (p == LOST) break;
                i = p;
                p = a.next[p];
            }
            if (base + k < out_cap) {
                out_i[base + k] = i;
                out_c[base + k] = c;
            } else {
                atomicOr(&a.stats->error_flags, ERR_CAPACITY);
            }
        }
        a.carr[c] = 0;
        a.ccount[c] = 0;
        a.head[c] = LOST;
        for (int w = 0; w < a.pp.occw; ++w) a.cocc[(size_t)c * a.pp.occw + w] = 0ull;
    }
}

// Outbox particles as doubles for the host: id, cell, and row-major x (FP64
// form), xi, v (dim per particle), from the move's output state.
template <int DIM, typename Real>
__global__ void k_outbox_pack(StepArgs a, const uint32_t* out_i, const uint32_t* out_c, uint32_t n, uint32_t* id,
                              int32_t* cell, double* x, double* xi, double* v)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t i = out_i[j];
        id[j] = a.S0.id[i];
        cell[j] = (int32_t)out_c[j];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            xi[(size_t)j * DIM + d] = (double)ldr<Real>(a.T.xi[d], i);
            v[(size_t)j * DIM + d] = (double)ldr<Real>(a.T.v[d], i);
            if constexpr (std::is_same<Real, double>::value) x[(size_t)j * DIM + d] = ldr<double>(a.T.x[d], i);
        }
    }
}

// Particles that arrived from other partitions, appended to the move's
// output state at slots base.. (beyond every cell's old range, so the write
// pass meets them as arrivals only) and entered among their cells' arrivals
// and counts, as the advect pass enters its own.
template <int DIM, typename Real>
__global__ void k_inbox(StepArgs a, uint32_t n, uint32_t base, const uint32_t* id, const int32_t* cell,
                        const double* x, const double* xi, const double* v)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t i = base + j;
        const uint32_t c = (uint32_t)cell[j];
        Real r[DIM];
        a.S0.id[i] = id[j];
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            r[d] = (Real)xi[(size_t)j * DIM + d];
            str<Real>(a.T.xi[d], i, r[d]);
            str<Real>(a.T.v[d], i, (Real)v[(size_t)j * DIM + d]);
            if constexpr (std::is_same<Real, double>::value) str<double>(a.T.x[d], i, x[(size_t)j * DIM + d]);
        }
        arrive(a, i, c, LOST, true);
        count_one(a, c, ext_part<DIM, Real>(r, a.pp));
    }
}

// Projection partial sums of listed cells, to and from doubles (PW per cell).
template <typename Real>
__global__ void k_partials_io(void* partials, int pw, uint32_t n, const int32_t* cells, double* buf, int to_buf)
{
    Real* P = reinterpret_cast<Real*>(partials);
    const size_t tot = (size_t)n * pw;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < tot; t += (size_t)gridDim.x * blockDim.x) {
        const size_t c = (size_t)cells[t / pw], e = t % pw;
        if (to_buf) buf[t] = (double)P[c * pw + e];
        else P[c * pw + e] = (Real)buf[t];
    }
}

}  // namespace pfem2
