// Shared device-side definitions of the PFEM-2 particle kernels.
//
// Particles live on the device as structure-of-arrays, sorted by (cell,
// cell part, key(id)) after every step:
//   cell u32 | id u32 | x[dim] f64 (FP64 form only) | xi[dim] | v[dim]
// with xi and v in f64 (FP64 form) or f32 (FP32 form).  The reference keeps an
// std::vector of 88/136-byte AoS records (src/pfem2particle.h:63-72); the
// per-particle cell_dofs copy and velocity_ext are not stored: DoFs come from
// the per-cell table and velocity_ext only lives inside one sub-step.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pfem2 {

constexpr uint32_t LOST = 0xFFFFFFFFu;  // no cell / end of a list
constexpr uint32_t HOLE = 0xFFFFFFFEu;  // cell of an empty slot (where a removed particle would have gone)
constexpr int MAX_CAND = 64;   // cells around one vertex tried by the relocation search
constexpr int REG_CAND = 12;   // FP32 form on affine meshes: candidates kept in registers
constexpr int NPE_MAX = 256;   // extended cell parts (q0+1)(q1+1)(q2+1)
constexpr int OCCW_MAX = 4;    // 64-bit part-occupancy words per cell
constexpr int ARRCAP = 32;     // arrival slots per cell before the overflow list
constexpr int CELL_WARPS = 4;  // warps per block of the warp-per-cell helper kernels
constexpr int KEY_CACHE = 128; // (part, key) pairs cached per warp on the general path
constexpr int ADV_CH = 512;    // particles per staged chunk of the FP32 advect pass
// cells whose velocity records an FP32 advect chunk stages with its particles
// (a chunk spans about ADV_CH / particles-per-cell + 1 cells; beyond this
// many, the chunk's particles read their records from global memory)
template <int DIM> struct AdvRec {
    static constexpr int MAXC = DIM == 3 ? 32 : 48;
};
constexpr int WR_WARPS = 4;    // write pass: warps per block
constexpr int WR_CHC = 4;      // write pass: cells per warp chunk

// error_flags bits
constexpr uint32_t ERR_CAPACITY = 1u;        // more particles than the arrays hold
constexpr uint32_t ERR_CAND_OVERFLOW = 2u;   // a vertex touches more than MAX_CAND cells
constexpr uint32_t ERR_BAD_CELL = 4u;        // a particle carries an out-of-range cell
constexpr uint32_t ERR_TIMEOUT = 8u;         // a bounded wait gave up
constexpr uint32_t ERR_COUNT = 16u;          // write pass: other new-particle count than the move's occupancy gave
constexpr uint32_t ERR_COUNT_UB = 32u;       // write pass: more particles than the cell's slots
constexpr uint32_t ERR_ARRIVAL = 64u;        // write pass: an arrival list shorter than its count

struct DevStats {
    unsigned long long n_particles;
    unsigned long long lost;
    unsigned long long removed;
    unsigned long long seeded;
    unsigned long long map_failures;
    unsigned long long near_face;
    unsigned long long searched;
    unsigned long long nan_dofs;
    unsigned long long fallback64;   // FP32 form: sub-steps relocated by the FP64 search
    unsigned long long particle_steps; // particles advanced, summed over moves
    unsigned long long n_slots;      // length of the particle arrays (particles + empty slots)
    unsigned long long step_holes;   // empty slots left by the last write pass
    unsigned int next_id;
    unsigned int error_flags;
    unsigned int write_done;         // write pass: warps finished (the last one finalises the step)
    unsigned int write_next;         // write pass: next chunk of cells to hand out
    unsigned int adv_next;           // advect pass: next chunk of particles to hand out
};

struct MeshDev {
    int nC, nV, nD;
    int all_affine;           // 1 if every cell's multilinear map is affine (no twist terms)
    const int32_t* cv;        // nC x NV vertex ids
    const int32_t* cd;        // nC x NV DoF ids
    const double* cellX;      // nC x NV x DIM vertex coordinates, cell-major
    const double* aff;        // nC x (DIM*DIM + DIM): inverse affine approximation A^-1 and b
    const float* geo32;       // nC x GEO: FP32 multilinear coefficients relative to vertex 0
    const float* jinv32;      // nC x JS: FP32 inverse Jacobian at the centre, then the affine flag
    const int32_t* v2c_off;   // nV + 1
    const int32_t* v2c_cells; // cells around each vertex, ascending
    const double* v2c_dirs;   // DIM per entry: unit vertex -> cell-centre direction
    const int32_t* d2c_off;   // nD + 1
    const int32_t* d2c_ent;   // cell * NV + local vertex, cells ascending
};

struct PartParams {
    int q[3];
    int npart;     // q0*q1*q2 real cell parts
    int npe;       // (q0+1)(q1+1)(q2+1) extended parts
    int maxpp;     // maximum particles per cell part (max+1 survive)
    int S;         // sub-steps
    double dtp;    // dt / S
    int rk2;       // sub-steps by the midpoint rule (PFEM2GPU_RK2) instead of Euler
    double h[3];   // 1.0 / q
    uint32_t seed; // removal key seed
    unsigned long long realmask[OCCW_MAX];  // real parts among the extended parts, 64 per word
    int occw;                               // occupancy words in use
};

// SoA particle arrays; x is null in the FP32 form.
struct PartState {
    uint32_t* cell;
    uint32_t* id;
    void* x[3];
    void* xi[3];
    void* v[3];
};

struct StepArgs {
    MeshDev mesh;
    PartParams pp;
    PartState S0;   // current, sorted
    PartState S1;   // next, sorted
    PartState T;    // advect output, in S0 order (cell/id unused)
    const void* Vc;     // FP64 form: nC x NV x VS nodal velocity per cell vertex, VS = 4 (3D) or 2 (2D)
    const void* dVc;    // FP64 form: nC x NV x VS velocity increment V - Vold per cell vertex
    const float* vrec32;  // FP32 form: nC x REC4 float4, velocity polynomial of each cell (+ affine flag)
    const float* dvrec32; // FP32 form: nC x REC4 float4, polynomial of V - Vold
    const double* Vd;     // staged nodal velocity, component-major (nD per component)
    int do_correct;
    int apply_counts;   // write kernel: 1 = count correction, 0 = keep all (re-sort only)
    int count_step;     // write kernel: add the step's particles to particle_steps
    int reset_nan;      // write kernel: zero nan_dofs for the projection that follows
    uint32_t* key;      // cell after the move, or LOST
    uint32_t* head;     // nC: overflow list of particles that moved into the cell (LOST = none)
    uint32_t* next;     // next particle on the same overflow list
    uint32_t* carr;     // nC: particles that moved into the cell
    uint32_t* carrs;    // nC x ARRCAP: the first ARRCAP of them
    uint32_t* ccount;   // nC: particles in the cell after the move
    unsigned long long* cocc;  // nC x occw: parts occupied after the move
    unsigned long long* cub;   // nC: new particles << 32 | slots needed
    unsigned long long* coff;  // nC + 1: exclusive scan of cub
    uint32_t* chunk_first;     // per ADV_CH-slot chunk of the layout the step writes: the cell its first slot
                               // belongs to (the seed and write passes fill it; null: not kept)
    const uint32_t* cs_old;    // nC + 1: cell ranges of S0
    uint32_t* cs_new;          // nC + 1: cell ranges of S1
    uint2* xq;                 // particles (index, sub-step) queued for FP64 relocation
    uint32_t* nxq;             // queue length
    uint4* gscr;               // write pass, general path: per-particle scratch in the cell's output range
    void* partials;                // nC x PW projection partial sums
    double* Vout;                  // nD x DIM component-major projected velocity
    double* Vout2;                 // a second copy of it (the handle's last projection), or null
    const double* Vkeep;           // empty_dof_policy 1: value kept where no particle contributes
    DevStats* stats;
    uint32_t capacity;
    int cbeg, cend;     // the cells this handle owns (the whole mesh unless partitioned)
};

// Differentiated window (window.cuh): device arrays of one window.
constexpr int WIN_BT = 128;             // threads per block of the per-particle window kernels
constexpr int WIN_TILE = 1024;          // elements per tile of the window scans
constexpr uint32_t ERR_REPLAY = 128u;   // backward: a recomputed segment ended elsewhere than its checkpoint

struct WinArgs {
    StepArgs a;                // mesh, parameters, staged velocities (Vc/dVc or vrec32/dvrec32, Vd = V)
    uint32_t n;                // particles in the window
    int K, C, nseg;            // steps, steps per segment, segments
    int do_correct;            // 1: correction with V - Vold every step
    int keep_empty;            // empty_dof_policy 1: U = V where no particle weighs
    const double* V;           // dim x nD component-major
    const double* Vold;        // dim x nD or null
    const uint32_t* slot;      // window particle -> slot of the handle's current state
    uint32_t* ck_cell;         // nseg x n: state at the start of each segment
    void* ck_xi[3];            // nseg x n (Real)
    double* ck_x[3];           // nseg x n (FP64 form)
    uint32_t* fin_cell;        // n: the forward's running state, after K steps its end (LOST: deleted)
    void* fin_xi[3];           // n (Real)
    double* fin_x[3];          // n (FP64 form)
    double* fin_v[3];          // n: particle velocities in FP64 (both forms)
    uint32_t* r_cell;          // n: running state of a segment replay
    void* r_xi[3];             // n (Real)
    double* r_x[3];            // n (FP64 form)
    uint32_t* rec_cell;        // (C*S + 1) x n: states before every sub-step of one segment, then its end
    void* rec_xi[3];           // (C*S + 1) x n (Real)
    uint2* q;                  // n: (particle, sub-step) of the step's face crossers
    uint32_t* nq;              // queue length
    uint32_t* ccnt;            // nC: particles per final cell, then placement counters
    uint32_t* cstart;          // nC + 1: exclusive scan of ccnt
    uint32_t* tsum;            // scan tile sums
    uint32_t* order;           // n: particles by final cell
    uint32_t* order2;          // n: the same, ascending particle index inside each cell
    double* part;              // nC x NV x 4: sum N_i v_d and sum N_i per (cell, vertex)
    double* U;                 // dim x nD
    double* den;               // nD
    double* gnum;              // dim x nD
    double* gden;              // nD
    double* gxi;               // dim x n: adjoint of xi between segments
    double* gv;                // dim x n: adjoint of the particle velocity
    double* gadv;              // nC x NV x DIM: dJ/dV through the sub-steps
    double* gdv;               // nC x NV x DIM: dJ/d(V - Vold) through the corrections
    const double* Wcell;       // nC x NV x VS: X_i + h V_i per cell vertex (the sub-step map's vertices)
    const double* dVcell;      // nC x NV x VS: V - Vold per cell vertex (FP64)
    unsigned long long* nempty;
    unsigned int* err;
};

// Q1 FEM systems assembled on the device (fem.cu).
constexpr int FEM_PREDICTION = 0, FEM_PRESSURE = 1, FEM_CORRECTION = 2;
constexpr int FEM_ROWMAX = 64;  // matrix entries per row the pattern pass can hold

struct FemArgs {
    int nC, nD;
    long long nnz;
    const double* cellX;
    const int32_t* cd;
    const int32_t* d2c_off;
    const int32_t* d2c_ent;
    int32_t* row_ptr;
    int32_t* cols;
    int32_t* con_off;   // per matrix entry: its contributions, in ascending cell order
    int32_t* con;       // (cell * NV + local row) * NV + local column
    double rho, mu, dt;
    const double* U;
    const double* U2;
    const double* P;
    double* local;      // per (cell, local row): matrices x 2^dim local entries
    double* local_rhs;  // per (cell, local row): right-hand sides
    double* A;          // matrices x nnz
    double* rhs;        // right-hand sides x nD
    const uint16_t* fmask;  // per cell: bit f = boundary face f with prediction face terms,
                            // bit 8 + f = with pressure face terms (null: none)
};

template <int DIM> struct Dims {
    static constexpr int NV = 1 << DIM;
    static constexpr int VS = DIM == 3 ? 4 : 2;        // padded velocity stride
    static constexpr int PW = DIM == 3 ? 32 : 16;      // projection partials per cell (NV x 4)
    static constexpr int AFF = DIM * DIM + DIM;
    static constexpr int GEO = DIM == 3 ? 24 : 8;      // FP32 geometry floats per cell
    static constexpr int JS = DIM == 3 ? 12 : 8;       // FP32 inverse Jacobian + flag, padded
    static constexpr int REC4 = DIM == 3 ? 7 : 3;      // float4 per FP32 velocity record (coefficients + flag)
};

// End of a move, run by one thread after the write pass: the new slot count
// and particle count, the ids handed out, the cell ranges' end.
__device__ __forceinline__ void finalize_step(const StepArgs& a)
{
    DevStats* st = a.stats;
    if (a.count_step) st->particle_steps += st->n_particles;
    const unsigned long long po = a.coff[a.mesh.nC];
    uint32_t slots = (uint32_t)po;
    const uint32_t seeds = (uint32_t)(po >> 32);
    if (slots > a.capacity) {
        st->error_flags |= ERR_CAPACITY;
        slots = a.capacity;
    }
    st->adv_next = 0;  // the advect pass of this step has finished
    *a.nxq = 0;        // and the crossing queue has been drained
    if (a.reset_nan) st->nan_dofs = 0;
    st->n_slots = slots;
    st->n_particles = slots - (st->step_holes < slots ? st->step_holes : slots);
    st->step_holes = 0;
    st->next_id += seeds;
    st->seeded += seeds;
    a.cs_new[a.mesh.nC] = slots;
}

// Entry of a kernel of the step sequence, launched with programmatic
// dependent launch: wait until the previous kernel on the stream has
// completed and its writes are visible, then let the next kernel be
// scheduled (its blocks wait in the same place).  Without the launch
// attribute both instructions return at once.
__device__ __forceinline__ void pdl_entry()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__host__ __device__ inline uint32_t key_of(uint32_t id, uint32_t seed)
{
    if (!seed) return id;
    uint32_t x = id ^ seed;  // bijective 32-bit mixer (lowbias32, C. Wellons)
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Extended cell-part index of reference coordinates: (int)(xi_d / h_d) per
// direction (src/pfem2particlehandler.cpp:369-370), which reaches q_d on the
// upper face; digits combined x-major, base q_d + 1.
// xi_d * q_d and xi_d / h_d round to within 3 ulp of each other, so their
// truncations can only differ within 1e-12 (xi_d * q_d <= 64) of an integer;
// only there is the division evaluated.
template <int DIM, typename Real>
__device__ __forceinline__ int ext_part(const Real* xi, const PartParams& pp)
{
    if constexpr (sizeof(Real) == 4) {
        // FP32 form: (int)(xi * q) in FP32, at most q - 1.  A stored FP32
        // xi_d of exactly 1 stands for every inside point within 3e-8 of the
        // upper face, where the FP64 form (and the reference) has xi_d < 1
        // and so part q - 1; only an xi_d of exactly 1 in FP64 reaches the
        // extra part q.  Particles pile up there at no-slip walls that the
        // flow runs into (the stagnation side of an obstacle): without the
        // cap they fall out of part q - 1 in the FP32 form, which then seeds
        // and removes differently from the FP64 form.
        int e = 0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            int k = (int)(xi[d] * (float)pp.q[d]);
            k = k < 0 ? 0 : (k > pp.q[d] - 1 ? pp.q[d] - 1 : k);
            e = e * (pp.q[d] + 1) + k;
        }
        return e;
    }
    int e = 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const double x = (double)xi[d];
        const double t = x * (double)pp.q[d];
        const double f = t - floor(t);
        int k = (f > 1e-12 && f < 1.0 - 1e-12) ? (int)t : (int)(x / pp.h[d]);
        k = k < 0 ? 0 : (k > pp.q[d] ? pp.q[d] : k);
        e = e * (pp.q[d] + 1) + k;
    }
    return e;
}

// Is extended part e one of the q0*q1*q2 real parts?  Writes its digits.
template <int DIM>
__device__ __forceinline__ bool real_part(int e, const PartParams& pp, int* idx)
{
    bool real = true;
#pragma unroll
    for (int d = DIM - 1; d >= 0; --d) {
        const int b = pp.q[d] + 1;
        idx[d] = e % b;
        e /= b;
        real = real && idx[d] < pp.q[d];
    }
    return real;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One atomic per warp for a per-thread counter (all 32 lanes must call it).
__device__ __forceinline__ void warp_count(unsigned long long* dst, unsigned long long v)
{
    v = warp_sum_u64(v);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

}  // namespace pfem2
