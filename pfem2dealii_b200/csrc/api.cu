// C ABI of the particle path: handle, device memory, and the per-call kernel
// sequences.  One time step of the reference loop (src/pfem2solver.cpp:162-164)
// maps to
//   correct(V, Vold)  -> stage V, V - Vold per cell vertex (the correction is fused into move)
//   move(V)           -> advect (staged) | FP64 relocation queue | slots per cell | scan | write (its last block finalises the step)
//   project(V_out)    -> gather (per-cell partials were summed by write) | D2H
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/pfem2gpu.h"
#include "launch.h"

using namespace pfem2;

struct pfem2gpu_handle {
    int dim = 2, prec = 0, dev = 0;
    pfem2gpu_params prm{};
    PartParams pp{};
    cudaStream_t stream = nullptr;
    // mesh
    int nC = 0, nV = 0, nD = 0;
    bool has_mesh = false;
    int32_t *cv = nullptr, *cd = nullptr, *v2c_off = nullptr, *v2c_cells = nullptr, *d2c_off = nullptr,
            *d2c_ent = nullptr;
    double *verts = nullptr, *cellX = nullptr, *aff = nullptr, *v2c_dirs = nullptr;
    float* geo32 = nullptr;
    uint32_t* twisted = nullptr;  // cells whose map is not affine (set by cell_setup)
    bool all_affine = false;
    // velocities
    double *Vstage = nullptr, *Vstage2 = nullptr, *Vout = nullptr;
    double* Vin = nullptr;  // host V of the current call, uploaded before its check (see stage_v)
    unsigned* nf_h = nullptr;  // mapped host word: the uploaded V holds a non-finite value
    unsigned* nf_d = nullptr;  // its device address
    void *Vc = nullptr, *dVc = nullptr;
    bool vaos_valid = false;
    // particles
    uint32_t cap = 0;
    PartState S0{}, S1{}, T{};
    uint32_t *key = nullptr, *next = nullptr;
    double* xtmp = nullptr;
    uint32_t *head = nullptr, *cs0 = nullptr, *cs1 = nullptr;  // cs0: cell ranges of S0
    uint2* xq = nullptr;
    uint32_t* nxq = nullptr;
    uint32_t *carr = nullptr, *carrs = nullptr, *ccount = nullptr;
    unsigned long long *cocc = nullptr, *cub = nullptr, *coff = nullptr, *tiles64 = nullptr;
    uint4* gscr = nullptr;
    uint32_t* chunk_first = nullptr;  // FP32 form: first cell of each advect chunk of the current layout
    float *jinv32 = nullptr, *vrec32 = nullptr, *dvrec32 = nullptr;
    bool launch_failed = false;
    // CUDA graphs of the per-step sequences (one per buffer parity and
    // variant), rebuilt whenever device buffers are reallocated
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        uint64_t gen = 0;
        uint64_t kernels = 0;
        int seen = 0;
        const void* key[3] = {nullptr, nullptr, nullptr};
    };
    Graph move_graph[2][2];  // [parity][do_correct]
    Graph step_graph[2];     // [parity] fused correct+move+project (device vectors)
    int parity = 0;
    uint64_t gen = 1;
    bool use_graphs = true;
    void* partials = nullptr;
    DevStats* stats = nullptr;
    DevStats* stats_h = nullptr;
    bool has_particles = false, pending_correct = false, partials_valid = false;
    bool has_projection = false;  // Vout holds the last projection of this mesh
    // cell-range partition (pfem2gpu_set_partition): the handle owns cells
    // [pbeg, pend); pend < 0 is the whole mesh.  A partitioned move runs in
    // phases (move_phase 1: outbox ready, 2: inbox entered and slots scanned).
    int64_t pbeg = 0, pend = -1;
    int move_phase = 0;
    uint32_t *ob_i = nullptr, *ob_c = nullptr, *ob_n = nullptr;
    uint32_t ob_cap = 0, ob_count = 0;
    void* xbuf = nullptr;  // staging of exchanged particles and partial sums
    size_t xbuf_bytes = 0;
    // accounting
    uint64_t launches = 0;
    bool profiling = false;
    struct Ev {
        std::string name;
        cudaEvent_t a, b;
    };
    std::vector<Ev> open_ev;
    std::vector<cudaEvent_t> ev_pool;
    std::map<std::string, std::pair<double, long long>> prof;
    std::string err;
    // output packing: live-slot list, its scan tiles, the packed floats
    uint32_t *out_slot = nullptr, *out_tsum = nullptr;
    float *out_dev = nullptr, *out_host = nullptr;
    uint32_t out_cap = 0, out_tcap = 0, out_dcap = 0;
    // FEM systems: the CSR pattern (built once per mesh), per-(cell, row)
    // local values, and device copies of host inputs/outputs
    struct Fem {
        int32_t *row_ptr = nullptr, *cols = nullptr, *con_off = nullptr, *con = nullptr;
        long long nnz = -1;
        double *local = nullptr, *local_rhs = nullptr, *io = nullptr;
        size_t local_n = 0, rhs_n = 0, io_n = 0;
        uint16_t* fmask = nullptr;  // per cell: faces with prediction / pressure face terms
        uint8_t* dmask = nullptr;    // per cell: boundary faces in the velocity Dirichlet set
        int32_t* face_id = nullptr;  // per cell and face: boundary id, -1 interior
        double *bc_P = nullptr, *bc_loc = nullptr, *bc_val = nullptr, *bc_vel = nullptr;  // velocity_bc buffers
        int32_t *bc_lid = nullptr, *bc_flag = nullptr, *bc_ids = nullptr;
        int32_t bc_ncap = 0;                // ids the bc_ids / bc_vel buffers hold
        int32_t* con_idx = nullptr;  // per DoF: index among the constrained rows, or -1
        double* con_val = nullptr;
        size_t con_val_n = 0;
    } fem;
    // differentiated window: checkpoints, final state, projection and adjoint
    // buffers (per-particle arrays sized ncap x segcap, the rest per mesh)
    struct Win {
        uint32_t ncap = 0, tsumcap = 0, n = 0;
        int segcap = 0, tcap = -1, K = 0, C = 1, nseg = 0, rec_seg = -1;
        bool do_correct = false, ready = false, mesh_ready = false;
        uint32_t *slot = nullptr, *ck_cell = nullptr, *fin_cell = nullptr, *r_cell = nullptr, *rec_cell = nullptr,
                 *order = nullptr, *order2 = nullptr, *tsum = nullptr, *ccnt = nullptr, *cstart = nullptr,
                 *nq = nullptr;
        uint2* q = nullptr;
        void *ck_xi = nullptr, *fin_xi = nullptr, *r_xi = nullptr, *rec_xi = nullptr;
        double *fin_v = nullptr, *ck_x = nullptr, *fin_x = nullptr, *r_x = nullptr, *gxi = nullptr, *gv = nullptr, *hv0 = nullptr;
        double *part = nullptr, *U = nullptr, *den = nullptr, *gnum = nullptr, *gden = nullptr, *gadv = nullptr,
               *gdv = nullptr, *V = nullptr, *Vold = nullptr, *gU = nullptr, *gV = nullptr, *gVold = nullptr,
               *Vcell = nullptr, *dVcell = nullptr, *Wcell = nullptr;
        unsigned long long* nempty = nullptr;
        unsigned int* err = nullptr;
    } win;
};

namespace {

size_t esize(const pfem2gpu_handle* h) { return h->prec == PFEM2GPU_FP64 ? 8 : 4; }

int fail(pfem2gpu_handle* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    return code;
}

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(h, e_ == cudaErrorMemoryAllocation ? PFEM2GPU_ERR_NOMEM : PFEM2GPU_ERR_CUDA,  \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t n)
{
    *p = nullptr;
    return cudaMalloc((void**)p, n ? n * sizeof(T) : sizeof(T));
}

void dfree(void* p)
{
    if (p) cudaFree(p);
}

cudaEvent_t take_event(pfem2gpu_handle* h)
{
    if (!h->ev_pool.empty()) {
        cudaEvent_t e = h->ev_pool.back();
        h->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

// Run one launcher, counting its kernels and, when profiling, timing it with
// events on the handle's stream.
template <typename F>
void run(pfem2gpu_handle* h, const char* name, F&& f)
{
    int n = 0;
    if (h->profiling) {
        cudaEvent_t a = take_event(h), b = take_event(h);
        cudaEventRecord(a, h->stream);
        n = f();
        cudaEventRecord(b, h->stream);
        h->open_ev.push_back({name, a, b});
    } else {
        n = f();
    }
    if (n < 0) h->launch_failed = true;
    else h->launches += n;
}

void collect_profile(pfem2gpu_handle* h)
{
    if (h->open_ev.empty()) return;
    cudaStreamSynchronize(h->stream);
    for (auto& e : h->open_ev) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e.a, e.b);
        auto& slot = h->prof[e.name];
        slot.first += ms;
        slot.second += 1;
        h->ev_pool.push_back(e.a);
        h->ev_pool.push_back(e.b);
    }
    h->open_ev.clear();
}

StepArgs args(pfem2gpu_handle* h)
{
    StepArgs a{};
    a.mesh.nC = h->nC;
    a.mesh.all_affine = h->all_affine ? 1 : 0;
    a.mesh.nV = h->nV;
    a.mesh.nD = h->nD;
    a.mesh.cv = h->cv;
    a.mesh.cd = h->cd;
    a.mesh.cellX = h->cellX;
    a.mesh.aff = h->aff;
    a.mesh.geo32 = h->geo32;
    a.mesh.jinv32 = h->jinv32;
    a.mesh.v2c_off = h->v2c_off;
    a.mesh.v2c_cells = h->v2c_cells;
    a.mesh.v2c_dirs = h->v2c_dirs;
    a.mesh.d2c_off = h->d2c_off;
    a.mesh.d2c_ent = h->d2c_ent;
    a.pp = h->pp;
    a.S0 = h->S0;
    a.S1 = h->S1;
    a.T = h->T;
    a.Vc = h->Vc;
    a.dVc = h->dVc;
    a.vrec32 = h->vrec32;
    a.dvrec32 = h->dvrec32;
    a.Vd = h->Vstage;
    a.do_correct = 0;
    a.apply_counts = 1;
    a.key = h->key;
    a.head = h->head;
    a.next = h->next;
    a.cs_old = h->cs0;
    a.cs_new = h->cs1;
    a.xq = h->xq;
    a.nxq = h->nxq;
    a.carr = h->carr;
    a.carrs = h->carrs;
    a.ccount = h->ccount;
    a.cocc = h->cocc;
    a.cub = h->cub;
    a.coff = h->coff;
    a.chunk_first = h->chunk_first;
    a.gscr = h->gscr;
    a.partials = h->partials;
    a.Vout = h->Vout;
    a.Vkeep = h->Vstage;
    a.stats = h->stats;
    a.capacity = h->cap;
    a.cbeg = (int)h->pbeg;
    a.cend = h->pend < 0 ? h->nC : (int)h->pend;
    return a;
}

void free_state(PartState& s)
{
    dfree(s.cell);
    dfree(s.id);
    for (int d = 0; d < 3; ++d) {
        dfree(s.x[d]);
        dfree(s.xi[d]);
        dfree(s.v[d]);
    }
    s = PartState{};
}

void free_win_particles(pfem2gpu_handle::Win& W)
{
    for (void* p : {(void*)W.slot, (void*)W.ck_cell, (void*)W.fin_cell, (void*)W.r_cell, (void*)W.rec_cell,
                    (void*)W.order, (void*)W.order2, (void*)W.q, W.ck_xi, W.fin_xi, (void*)W.fin_v, W.r_xi, W.rec_xi,
                    (void*)W.ck_x, (void*)W.fin_x, (void*)W.r_x, (void*)W.gxi, (void*)W.gv, (void*)W.hv0})
        dfree(p);
    W.slot = W.ck_cell = W.fin_cell = W.r_cell = W.rec_cell = W.order = W.order2 = nullptr;
    W.q = nullptr;
    W.ck_xi = W.fin_xi = W.r_xi = W.rec_xi = nullptr;
    W.fin_v = nullptr;
    W.ck_x = W.fin_x = W.r_x = W.gxi = W.gv = W.hv0 = nullptr;
    W.ncap = 0;
    W.segcap = 0;
    W.tcap = -1;
    W.ready = false;
}

void free_fem(pfem2gpu_handle::Fem& F)
{
    for (void* p : {(void*)F.row_ptr, (void*)F.cols, (void*)F.con_off, (void*)F.con, (void*)F.local,
                    (void*)F.local_rhs, (void*)F.io, (void*)F.fmask, (void*)F.con_idx, (void*)F.con_val,
                    (void*)F.dmask, (void*)F.face_id, (void*)F.bc_P, (void*)F.bc_loc, (void*)F.bc_val,
                    (void*)F.bc_vel, (void*)F.bc_lid, (void*)F.bc_flag, (void*)F.bc_ids})
        dfree(p);
    F = pfem2gpu_handle::Fem{};
}

// Device scratch of one call, released on every return path.
struct Scratch {
    std::vector<void*> p;
    template <typename T>
    cudaError_t get(T** ptr, size_t n)
    {
        cudaError_t e = dalloc(ptr, n);
        if (e == cudaSuccess) p.push_back(*ptr);
        return e;
    }
    ~Scratch()
    {
        for (void* q : p) dfree(q);
    }
};

void free_win_mesh(pfem2gpu_handle::Win& W)
{
    for (void* p : {(void*)W.tsum, (void*)W.ccnt, (void*)W.cstart, (void*)W.part, (void*)W.U, (void*)W.den,
                    (void*)W.gnum, (void*)W.gden, (void*)W.gadv, (void*)W.gdv, (void*)W.V, (void*)W.Vold, (void*)W.gU,
                    (void*)W.gV, (void*)W.gVold, (void*)W.nempty, (void*)W.err, (void*)W.Vcell, (void*)W.dVcell,
                    (void*)W.Wcell, (void*)W.nq})
        dfree(p);
    W.tsum = W.ccnt = W.cstart = W.nq = nullptr;
    W.part = W.U = W.den = W.gnum = W.gden = W.gadv = W.gdv = W.V = W.Vold = W.gU = W.gV = W.gVold = nullptr;
    W.Vcell = W.dVcell = W.Wcell = nullptr;
    W.nempty = nullptr;
    W.err = nullptr;
    W.tsumcap = 0;
    W.mesh_ready = false;
    W.ready = false;
}

cudaError_t alloc_state(pfem2gpu_handle* h, PartState& s, uint32_t cap, bool with_ids)
{
    cudaError_t e = cudaSuccess;
    const size_t es = esize(h);
    if (with_ids) {
        if ((e = dalloc(&s.cell, cap)) != cudaSuccess) return e;
        if ((e = dalloc(&s.id, cap)) != cudaSuccess) return e;
    }
    for (int d = 0; d < h->dim; ++d) {
        if (h->prec == PFEM2GPU_FP64 && (e = cudaMalloc(&s.x[d], cap * 8ull)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&s.xi[d], cap * es)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&s.v[d], cap * es)) != cudaSuccess) return e;
    }
    return e;
}

// The particle slots params.capacity allows (0: no limit), in whole
// 16-byte chunks of 4-byte slots.
uint64_t capacity_limit(const pfem2gpu_handle* h)
{
    return h->prm.capacity > 0 ? ((uint64_t)h->prm.capacity + 3) & ~3ull : 0x7FFFFFF0ull;
}

// Particle arrays sized for `need` particles (grown by 1.5x, S0 kept), up to
// `want` when that is more, never beyond params.capacity: a `need` above it
// is PFEM2GPU_ERR_CAPACITY before any allocation.
int ensure_capacity(pfem2gpu_handle* h, uint64_t need, uint64_t want = 0)
{
    const uint64_t limit = capacity_limit(h);
    if (need > limit)
        return fail(h, PFEM2GPU_ERR_CAPACITY, "particle capacity " + std::to_string(limit) + " below the " +
                                                  std::to_string(need) + " particles needed");
    if (need <= h->cap && h->S0.cell && want <= h->cap) return PFEM2GPU_OK;
    if (h->cap >= limit && h->S0.cell) return PFEM2GPU_OK;  // at the limit: need fits already
    uint64_t cap = std::max<uint64_t>(std::max(need, want), (uint64_t)h->cap * 3 / 2);
    cap = (std::max<uint64_t>(cap, 1024) + 3) & ~3ull;  // whole 16-byte chunks for the bulk copies
    cap = std::min(cap, limit);
    PartState n0{}, n1{}, nt{};
    CK(alloc_state(h, n0, (uint32_t)cap, true));
    CK(alloc_state(h, n1, (uint32_t)cap, true));
    CK(alloc_state(h, nt, (uint32_t)cap, false));
    uint32_t* cf_new = nullptr;
    const size_t ncf = (cap + ADV_CH - 1) / ADV_CH + 1;
    if (h->prec == PFEM2GPU_FP32) {
        CK(dalloc(&cf_new, ncf));
        if (h->chunk_first)
            CK(cudaMemcpyAsync(cf_new, h->chunk_first, ((size_t)h->cap + ADV_CH - 1) / ADV_CH * 4 + 4,
                               cudaMemcpyDeviceToDevice, h->stream));
    }
    if (h->S0.cell && h->has_particles) {
        const size_t n = h->cap, es = esize(h);
        CK(cudaMemcpyAsync(n0.cell, h->S0.cell, n * 4, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(n0.id, h->S0.id, n * 4, cudaMemcpyDeviceToDevice, h->stream));
        for (int d = 0; d < h->dim; ++d) {
            if (h->S0.x[d]) CK(cudaMemcpyAsync(n0.x[d], h->S0.x[d], n * 8, cudaMemcpyDeviceToDevice, h->stream));
            CK(cudaMemcpyAsync(n0.xi[d], h->S0.xi[d], n * es, cudaMemcpyDeviceToDevice, h->stream));
            CK(cudaMemcpyAsync(n0.v[d], h->S0.v[d], n * es, cudaMemcpyDeviceToDevice, h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    free_state(h->S0);
    free_state(h->S1);
    free_state(h->T);
    dfree(h->chunk_first);
    h->chunk_first = cf_new;
    dfree(h->key);
    dfree(h->next);
    dfree(h->xtmp);
    dfree(h->xq);
    dfree(h->gscr);
    h->gscr = nullptr;
    h->key = h->next = nullptr;
    h->xtmp = nullptr;
    h->xq = nullptr;
    h->S0 = n0;
    h->S1 = n1;
    h->T = nt;
    CK(dalloc(&h->key, cap));
    CK(dalloc(&h->next, cap));
    CK(dalloc(&h->xq, cap));
    CK(dalloc(&h->gscr, cap));
    if (!h->nxq) {
        CK(dalloc(&h->nxq, 1));
        CK(cudaMemsetAsync(h->nxq, 0, sizeof(uint32_t), h->stream));
    }
    if (h->prec == PFEM2GPU_FP32) CK(dalloc(&h->xtmp, cap * h->dim));
    h->cap = (uint32_t)cap;
    h->gen++;
    return PFEM2GPU_OK;
}

// A host nodal velocity (the FEM solution) must be finite everywhere.
// Device vectors are not inspected.  Vold is not checked either: it may be a
// projection, which is NaN where no particle reaches (the reference's 0/0).
bool all_finite(const double* V, size_t n)
{
    const uint64_t* b = reinterpret_cast<const uint64_t*>(V);
    uint64_t bad = 0;
    for (size_t i = 0; i < n; ++i) bad |= (uint64_t)((b[i] & 0x7FF0000000000000ull) == 0x7FF0000000000000ull);
    return bad == 0;
}

int check_async(pfem2gpu_handle* h);

// Nodal velocity staging: host or device component-major V (and Vold) ->
// padded per-DoF V (and V - Vold) in the form's precision.  Vold is on the
// device when `device` is set or when it is the handle's last projection.
// A host V is uploaded into a buffer of its own and checked there by one
// device pass that reports to a mapped host word; the call waits for the
// copy and the check (the staging could not start before the copy anyway),
// and a non-finite value returns PFEM2GPU_ERR_ARG before any kernel that
// reads V runs, so the staged velocity and the particles stay as they were.
// (A host scan of the 3 x 135 k values of the duct took 157 us, more than
// the copy it overlapped.)
int stage_v(pfem2gpu_handle* h, const double* V, const double* Vold, bool device)
{
    const size_t bytes = (size_t)h->dim * h->nD * sizeof(double);
    const double* v = V;
    const double* vo = Vold;
    if (!device) {
        CK(cudaMemcpyAsync(h->Vin, V, bytes, cudaMemcpyHostToDevice, h->stream));
        v = h->Vin;
        if (Vold && Vold != h->Vout) {
            CK(cudaMemcpyAsync(h->Vstage2, Vold, bytes, cudaMemcpyHostToDevice, h->stream));
            vo = h->Vstage2;
        }
        *reinterpret_cast<volatile unsigned*>(h->nf_h) = 0u;  // no kernel is writing it: every check is waited for
        run(h, "check_velocity",
            [&] { return launch_nonfinite(h->Vin, (size_t)h->dim * h->nD, h->nf_d, h->stream); });
        int rc = check_async(h);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->stream));
        if (*reinterpret_cast<volatile unsigned*>(h->nf_h)) return fail(h, PFEM2GPU_ERR_ARG, "non-finite nodal velocity");
    }
    // the staging kernel also writes the kept copy of V
    double* vcopy = v != h->Vstage ? h->Vstage : nullptr;
    if (h->prec == PFEM2GPU_FP64) {
        run(h, "stage_velocity", [&] {
            return launch_cell_v(h->dim, h->prec, v, vo, h->cd, h->nC, h->nD, h->Vc, Vold ? h->dVc : nullptr, vcopy,
                                 h->stream);
        });
    } else {
        run(h, "stage_velocity", [&] {
            return launch_cell_rec32(h->dim, v, vo, h->cd, h->aff, h->jinv32, h->nC, h->nD, h->vrec32,
                                     Vold ? h->dvrec32 : nullptr, vcopy, h->stream);
        });
    }
    h->vaos_valid = true;
    return PFEM2GPU_OK;
}

int check_async(pfem2gpu_handle* h)
{
    if (h->launch_failed) {
        h->launch_failed = false;
        return fail(h, PFEM2GPU_ERR_CUDA, "kernel launch failed");
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, PFEM2GPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return PFEM2GPU_OK;
}

int apply_pending_correction(pfem2gpu_handle* h)
{
    if (!h->pending_correct) return PFEM2GPU_OK;
    StepArgs a = args(h);
    run(h, "correct", [&] { return launch_correct(h->dim, h->prec, a, h->stream); });
    h->pending_correct = false;
    h->partials_valid = false;
    return check_async(h);
}

// The write pass (count correction, sorted layout, projection partials) and
// the counters of the step; S1 becomes the current state.  Shared by move and
// set_particles.
void swap_state(pfem2gpu_handle* h)
{
    std::swap(h->S0, h->S1);
    std::swap(h->cs0, h->cs1);
    h->parity ^= 1;
    h->partials_valid = true;
}

// The write pass (count correction, new layout, projection partials) and
// the counters of the step.
int enqueue_write(pfem2gpu_handle* h, StepArgs& a, int count_step, int reset_nan = 0)
{
    a.reset_nan = reset_nan;
    run(h, "slots_scan", [&] { return launch_slots_scan(a, h->tiles64, h->stream); });
    a.count_step = count_step;  // the write pass's last block finalises the step
    run(h, "write", [&] { return launch_write(h->dim, h->prec, a, h->stream); });
    return PFEM2GPU_OK;
}

int write_and_swap(pfem2gpu_handle* h, StepArgs& a, int count_step)
{
    enqueue_write(h, a, count_step);
    swap_state(h);
    return check_async(h);
}

// The crossing queue's counter is zero here: set at allocation, and reset by
// the write pass that ends every move.
int enqueue_move(pfem2gpu_handle* h, int do_correct, int reset_nan = 0)
{
    StepArgs a = args(h);
    a.do_correct = do_correct;
    run(h, "advect", [&] { return launch_advect(h->dim, h->prec, a, h->stream); });
    run(h, "cross", [&] { return launch_cross(h->dim, h->prec, a, h->stream); });
    return enqueue_write(h, a, 1, reset_nan);
}

// Run `enqueue` through a cached CUDA graph: eager on the first use of a
// variant (which also settles every one-time kernel attribute), captured on
// the second, replayed afterwards.  Profiling runs stay eager so that every
// launch is timed.
template <typename F>
int graphed(pfem2gpu_handle* h, pfem2gpu_handle::Graph& g, const void* k0, const void* k1, const void* k2, F&& enqueue)
{
    const bool same = g.key[0] == k0 && g.key[1] == k1 && g.key[2] == k2;
    if (h->profiling || !h->use_graphs) return enqueue();
    if (g.exec && g.gen == h->gen && same) {
        CK(cudaGraphLaunch(g.exec, h->stream));
        h->launches += g.kernels;
        return PFEM2GPU_OK;
    }
    if (!same || g.gen != h->gen) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
        g.seen = 0;
        g.key[0] = k0;
        g.key[1] = k1;
        g.key[2] = k2;
    }
    if (g.seen++ == 0) return enqueue();
    const uint64_t l0 = h->launches;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue();
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(h->stream, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ec != cudaSuccess) return fail(h, PFEM2GPU_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(h, PFEM2GPU_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    g.gen = h->gen;
    g.kernels = h->launches - l0;
    h->launches = l0;
    CK(cudaGraphLaunch(g.exec, h->stream));
    h->launches += g.kernels;
    return PFEM2GPU_OK;
}

int do_move(pfem2gpu_handle* h)
{
    if (!h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "move before seed");
    if (!h->vaos_valid) return fail(h, PFEM2GPU_ERR_STATE, "move without a velocity");
    const int dc = h->pending_correct ? 1 : 0;
    h->pending_correct = false;
    const int rc = graphed(h, h->move_graph[h->parity][dc], nullptr, nullptr, nullptr, [&] { return enqueue_move(h, dc); });
    if (rc) return rc;
    swap_state(h);
    return check_async(h);
}

int sync_stats(pfem2gpu_handle* h)
{
    CK(cudaMemcpyAsync(h->stats_h, h->stats, sizeof(DevStats), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->profiling) collect_profile(h);
    const uint32_t f = h->stats_h->error_flags;
    if (f & ERR_CAPACITY) return fail(h, PFEM2GPU_ERR_CAPACITY, "particle capacity exceeded");
    if (f) return fail(h, PFEM2GPU_ERR_DEVICE, "kernel error flags " + std::to_string(f));
    return PFEM2GPU_OK;
}

// Grow the particle arrays ahead of need (the next step may add up to one
// particle per empty part); only at points that already synchronize.
int maybe_grow(pfem2gpu_handle* h)
{
    const uint64_t n = h->stats_h->n_slots;
    const uint64_t own = (uint64_t)((h->pend < 0 ? h->nC : h->pend) - h->pbeg) * h->pp.npart;
    if (n + own / 2 > h->cap && h->cap < capacity_limit(h)) return ensure_capacity(h, n, n + own);
    return PFEM2GPU_OK;
}


// ---------------------------------------------------------------------------
// Differentiated window (window.cuh).
// ---------------------------------------------------------------------------
int win_reserve(pfem2gpu_handle* h, uint32_t n, uint32_t ns, int nseg, int tseg)
{
    auto& W = h->win;
    const int dim = h->dim, NV = 1 << dim;
    const size_t nc = h->nC, nd = h->nD, es = esize(h), VS = dim == 3 ? 4 : 2;
    const bool fp64 = h->prec == PFEM2GPU_FP64;
    if (!W.mesh_ready) {
        CK(dalloc(&W.ccnt, nc));
        CK(dalloc(&W.cstart, nc + 1));
        CK(dalloc(&W.part, nc * NV * 4));
        CK(dalloc(&W.U, nd * dim));
        CK(dalloc(&W.den, nd));
        CK(dalloc(&W.gnum, nd * dim));
        CK(dalloc(&W.gden, nd));
        CK(dalloc(&W.gadv, nc * NV * dim));
        CK(dalloc(&W.gdv, nc * NV * dim));
        CK(dalloc(&W.V, nd * dim));
        CK(dalloc(&W.Vold, nd * dim));
        CK(dalloc(&W.gU, nd * dim));
        CK(dalloc(&W.gV, nd * dim));
        CK(dalloc(&W.gVold, nd * dim));
        CK(dalloc(&W.nempty, 1));
        CK(dalloc(&W.err, 1));
        CK(dalloc(&W.nq, 1));
        CK(dalloc(&W.Vcell, nc * NV * VS));
        CK(dalloc(&W.dVcell, nc * NV * VS));
        CK(dalloc(&W.Wcell, nc * NV * VS));
        W.mesh_ready = true;
    }
    const uint32_t tneed = (std::max<uint32_t>(ns, (uint32_t)nc) + WIN_TILE - 1) / WIN_TILE + 1;
    if (tneed > W.tsumcap) {
        dfree(W.tsum);
        W.tsum = nullptr;
        W.tsumcap = 0;
        CK(dalloc(&W.tsum, tneed));
        W.tsumcap = tneed;
    }
    if (n > W.ncap || nseg > W.segcap || tseg > W.tcap) {
        CK(cudaStreamSynchronize(h->stream));
        const uint32_t ncap = std::max<uint32_t>(std::max<uint32_t>(n, 1024), W.ncap);
        const int segcap = std::max(nseg, W.segcap), tcap = std::max(tseg, W.tcap);
        free_win_particles(W);
        const size_t nck = (size_t)segcap * ncap, nrec = (size_t)(tcap + 1) * ncap;
        CK(dalloc(&W.slot, ncap));
        CK(dalloc(&W.ck_cell, nck));
        CK(cudaMalloc(&W.ck_xi, nck * dim * es));
        CK(dalloc(&W.fin_cell, ncap));
        CK(cudaMalloc(&W.fin_xi, (size_t)ncap * dim * es));
        CK(dalloc(&W.fin_v, (size_t)ncap * dim));
        CK(dalloc(&W.r_cell, ncap));
        CK(cudaMalloc(&W.r_xi, (size_t)ncap * dim * es));
        CK(dalloc(&W.rec_cell, nrec));
        CK(cudaMalloc(&W.rec_xi, nrec * dim * es));
        if (fp64) {
            CK(dalloc(&W.ck_x, nck * dim));
            CK(dalloc(&W.fin_x, (size_t)ncap * dim));
            CK(dalloc(&W.r_x, (size_t)ncap * dim));
        }
        CK(dalloc(&W.q, ncap));
        CK(dalloc(&W.order, ncap));
        CK(dalloc(&W.order2, ncap));
        CK(dalloc(&W.gxi, (size_t)ncap * dim));
        CK(dalloc(&W.gv, (size_t)ncap * dim));
        CK(dalloc(&W.hv0, (size_t)ncap * dim));
        W.ncap = ncap;
        W.segcap = segcap;
        W.tcap = tcap;
    }
    return PFEM2GPU_OK;
}

WinArgs winargs(pfem2gpu_handle* h)
{
    auto& W = h->win;
    WinArgs w{};
    w.a = args(h);
    w.n = W.n;
    w.K = W.K;
    w.C = W.C;
    w.nseg = W.nseg;
    w.do_correct = W.do_correct ? 1 : 0;
    w.keep_empty = h->prm.empty_dof_policy == 1 ? 1 : 0;
    w.V = W.V;
    w.Vold = W.do_correct ? W.Vold : nullptr;
    w.slot = W.slot;
    const size_t es = esize(h), nck = (size_t)W.segcap * W.ncap, nrec = (size_t)(W.tcap + 1) * W.ncap;
    w.ck_cell = W.ck_cell;
    w.fin_cell = W.fin_cell;
    w.r_cell = W.r_cell;
    w.rec_cell = W.rec_cell;
    for (int d = 0; d < h->dim; ++d) {
        w.ck_xi[d] = (char*)W.ck_xi + d * nck * es;
        w.ck_x[d] = W.ck_x ? W.ck_x + d * nck : nullptr;
        w.fin_xi[d] = (char*)W.fin_xi + (size_t)d * W.ncap * es;
        w.fin_x[d] = W.fin_x ? W.fin_x + (size_t)d * W.ncap : nullptr;
        w.fin_v[d] = W.fin_v + (size_t)d * W.ncap;
        w.r_xi[d] = (char*)W.r_xi + (size_t)d * W.ncap * es;
        w.r_x[d] = W.r_x ? W.r_x + (size_t)d * W.ncap : nullptr;
        w.rec_xi[d] = (char*)W.rec_xi + d * nrec * es;
    }
    w.q = W.q;
    w.nq = W.nq;
    w.ccnt = W.ccnt;
    w.cstart = W.cstart;
    w.tsum = W.tsum;
    w.order = W.order;
    w.order2 = W.order2;
    w.part = W.part;
    w.U = W.U;
    w.den = W.den;
    w.gnum = W.gnum;
    w.gden = W.gden;
    w.gxi = W.gxi;
    w.gv = W.gv;
    w.gadv = W.gadv;
    w.gdv = W.gdv;
    w.Wcell = W.Wcell;
    w.dVcell = W.dVcell;
    w.nempty = W.nempty;
    w.err = W.err;
    return w;
}

// Does the handle own only part of the mesh's cells (pfem2gpu_set_partition)?
static bool split(const pfem2gpu_handle* h) { return h->pend >= 0 && (h->pbeg > 0 || h->pend < h->nC); }

int window_forward_impl(pfem2gpu_handle* h, int K, int C, const double* V, const double* Vold, const double* v0,
                        double* U_out, bool host)
{
    if (!h || !V || K < 0 || C < 1) return PFEM2GPU_ERR_ARG;
    if (h->pp.rk2) return fail(h, PFEM2GPU_ERR_ARG, "the differentiated window supports Euler sub-steps only");
    if (h->move_phase || split(h)) return fail(h, PFEM2GPU_ERR_STATE, "the differentiated window needs an unpartitioned handle");
    if (!h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "window before seed");
    if ((int64_t)C * h->pp.S > 100000) return fail(h, PFEM2GPU_ERR_ARG, "checkpoint_every x sub-steps too large");
    int rc = apply_pending_correction(h);
    if (rc) return rc;
    if ((rc = sync_stats(h))) return rc;
    auto& W = h->win;
    const uint32_t n = (uint32_t)h->stats_h->n_particles, ns = (uint32_t)h->stats_h->n_slots;
    const int nseg = K > 0 ? (K + C - 1) / C : 1;
    const int tseg = std::min(C, std::max(K, 1)) * h->pp.S;
    if ((rc = win_reserve(h, n, ns, nseg, tseg))) return rc;
    W.ready = false;
    W.n = n;
    W.K = K;
    W.C = C;
    W.nseg = nseg;
    W.do_correct = Vold != nullptr;
    const size_t vbytes = (size_t)h->dim * h->nD * sizeof(double);
    const cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    CK(cudaMemcpyAsync(W.V, V, vbytes, kind, h->stream));
    if (Vold) CK(cudaMemcpyAsync(W.Vold, Vold, vbytes, kind, h->stream));
    const double* v0d = v0;
    if (v0 && host) {
        CK(cudaMemcpyAsync(W.hv0, v0, (size_t)n * h->dim * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        v0d = W.hv0;
    }
    if ((rc = stage_v(h, W.V, Vold ? W.Vold : nullptr, true))) return rc;
    // FP64 per-cell vertex velocities for the backward pass
    WinArgs w = winargs(h);
    run(h, "window_cells", [&] {
        return launch_cell_v(h->dim, 0, W.V, Vold ? W.Vold : nullptr, h->cd, h->nC, h->nD, W.Vcell, W.dVcell,
                             nullptr, h->stream) +
               launch_win_wcell(h->dim, w, W.Vcell, W.Wcell, h->stream);
    });
    run(h, "window_compact", [&] { return launch_win_compact(h->S0.cell, ns, (uint32_t)h->nC, W.tsum, W.slot, h->stream); });
    run(h, "window_init", [&] { return launch_win_init(h->dim, h->prec, w, v0d, h->stream); });
    run(h, "window_forward", [&] { return launch_win_forward(h->dim, h->prec, w, h->stream); });
    W.rec_seg = K > 0 ? nseg - 1 : -1;
    CK(cudaMemsetAsync(W.ccnt, 0, (size_t)h->nC * sizeof(uint32_t), h->stream));
    CK(cudaMemsetAsync(W.nempty, 0, sizeof(unsigned long long), h->stream));
    run(h, "window_project", [&] { return launch_win_project(h->dim, h->prec, w, h->stream); });
    if ((rc = check_async(h))) return rc;
    if (U_out) CK(cudaMemcpyAsync(U_out, W.U, vbytes, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, h->stream));
    if (host) CK(cudaStreamSynchronize(h->stream));
    W.ready = true;
    return PFEM2GPU_OK;
}

int window_backward_impl(pfem2gpu_handle* h, const double* gU, double* g_v0, double* gV, double* gVold, bool host)
{
    if (!h || !gU) return PFEM2GPU_ERR_ARG;
    auto& W = h->win;
    if (!W.ready) return fail(h, PFEM2GPU_ERR_STATE, "window backward without a window forward");
    int rc;
    // the window's velocities again (other calls may have staged others since)
    if ((rc = stage_v(h, W.V, W.do_correct ? W.Vold : nullptr, true))) return rc;
    const size_t vbytes = (size_t)h->dim * h->nD * sizeof(double);
    const double* gUd = gU;
    if (host) {
        CK(cudaMemcpyAsync(W.gU, gU, vbytes, cudaMemcpyHostToDevice, h->stream));
        gUd = W.gU;
    }
    double* gv0d = host ? (g_v0 ? W.hv0 : nullptr) : g_v0;
    double* gVd = host ? W.gV : gV;
    double* gVoldd = host ? W.gVold : gVold;
    const size_t nacc = (size_t)h->nC * (1 << h->dim) * h->dim * sizeof(double);
    CK(cudaMemsetAsync(W.gadv, 0, nacc, h->stream));
    CK(cudaMemsetAsync(W.gdv, 0, nacc, h->stream));
    CK(cudaMemsetAsync(W.err, 0, sizeof(unsigned int), h->stream));
    WinArgs w = winargs(h);
    run(h, "window_backward",
        [&] { return launch_win_backward(h->dim, h->prec, w, gUd, gv0d, gVd, gVoldd, W.rec_seg, h->stream); });
    W.rec_seg = W.K > 0 ? 0 : -1;
    if ((rc = check_async(h))) return rc;
    if (host) {
        if (g_v0) CK(cudaMemcpyAsync(g_v0, W.hv0, (size_t)W.n * h->dim * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        if (gV) CK(cudaMemcpyAsync(gV, W.gV, vbytes, cudaMemcpyDeviceToHost, h->stream));
        if (gVold) CK(cudaMemcpyAsync(gVold, W.gVold, vbytes, cudaMemcpyDeviceToHost, h->stream));
    }
    unsigned int err = 0;
    CK(cudaMemcpyAsync(&err, W.err, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->profiling) collect_profile(h);
    if (err) return fail(h, PFEM2GPU_ERR_DEVICE, "window backward: a recomputed segment left the forward trajectory");
    return PFEM2GPU_OK;
}

// Packed Float32 positions and velocities of the live particles (slot
// order) into dst (device, >= 6 n floats); n = the particle count.
int pack_output(pfem2gpu_handle* h, float* dst, int64_t capacity, int64_t* n)
{
    *n = 0;
    if (!h->has_particles) return PFEM2GPU_OK;
    int rc = apply_pending_correction(h);
    if (rc) return rc;
    if ((rc = sync_stats(h))) return rc;
    const uint32_t np = (uint32_t)h->stats_h->n_particles, ns = (uint32_t)h->stats_h->n_slots;
    *n = np;
    if (capacity < (int64_t)np) return fail(h, PFEM2GPU_ERR_ARG, "output buffer too small");
    if (np > h->out_cap) {
        dfree(h->out_slot);
        h->out_slot = nullptr;
        h->out_cap = 0;
        CK(dalloc(&h->out_slot, np));
        h->out_cap = np;
    }
    const uint32_t tneed = (ns + WIN_TILE - 1) / WIN_TILE + 1;
    if (tneed > h->out_tcap) {
        dfree(h->out_tsum);
        h->out_tsum = nullptr;
        h->out_tcap = 0;
        CK(dalloc(&h->out_tsum, tneed));
        h->out_tcap = tneed;
    }
    StepArgs a = args(h);
    run(h, "output_compact", [&] { return launch_win_compact(h->S0.cell, ns, (uint32_t)h->nC, h->out_tsum, h->out_slot, h->stream); });
    run(h, "output_pack", [&] { return launch_pack_output(h->dim, h->prec, a, h->out_slot, np, dst, h->stream); });
    return check_async(h);
}

}  // namespace

extern "C" {

const char* pfem2gpu_error_string(int code)
{
    switch (code) {
    case PFEM2GPU_OK: return "ok";
    case PFEM2GPU_ERR_ARG: return "invalid argument";
    case PFEM2GPU_ERR_CUDA: return "CUDA error";
    case PFEM2GPU_ERR_STATE: return "call out of order";
    case PFEM2GPU_ERR_CAPACITY: return "particle capacity exceeded";
    case PFEM2GPU_ERR_NOMEM: return "device out of memory";
    case PFEM2GPU_ERR_NODEVICE: return "no CUDA device";
    case PFEM2GPU_ERR_DEVICE: return "kernel reported invalid data";
    case PFEM2GPU_ERR_SCRATCH: return "mesh larger than the static scratch of pfem2gpu_project_noalloc";
    default: return "unknown error";
    }
}

int pfem2gpu_last_error(pfem2gpu_handle* h, char* buf, int64_t len)
{
    if (!h || !buf || len <= 0) return PFEM2GPU_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", h->err.c_str());
    return PFEM2GPU_OK;
}

int pfem2gpu_create(int dim, int precision, const pfem2gpu_params* prm, pfem2gpu_handle** out)
{
    if (!out || !prm) return PFEM2GPU_ERR_ARG;
    *out = nullptr;
    if (dim != 2 && dim != 3) return PFEM2GPU_ERR_ARG;
    if (precision != PFEM2GPU_FP64 && precision != PFEM2GPU_FP32) return PFEM2GPU_ERR_ARG;
    int npart = 1, npe = 1;
    for (int d = 0; d < dim; ++d) {
        if (prm->particles_per_cell[d] < 1 || prm->particles_per_cell[d] > 64) return PFEM2GPU_ERR_ARG;
        npart *= prm->particles_per_cell[d];
        npe *= prm->particles_per_cell[d] + 1;
    }
    if (npe > NPE_MAX) return PFEM2GPU_ERR_ARG;
    if (!(std::isfinite(prm->time_step)) || prm->particle_integration_steps < 0) return PFEM2GPU_ERR_ARG;
    if (prm->integrator != PFEM2GPU_EULER && prm->integrator != PFEM2GPU_RK2) return PFEM2GPU_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PFEM2GPU_ERR_NODEVICE;
    }
    pfem2gpu_handle* h = new pfem2gpu_handle();
    h->dim = dim;
    h->prec = precision;
    h->prm = *prm;
    cudaGetDevice(&h->dev);
    PartParams& pp = h->pp;
    for (int d = 0; d < 3; ++d) {
        pp.q[d] = d < dim ? prm->particles_per_cell[d] : 1;
        pp.h[d] = 1.0 / pp.q[d];
    }
    pp.npart = npart;
    pp.npe = npe;
    pp.maxpp = prm->max_particles_per_cell_part;
    pp.S = prm->particle_integration_steps == 0 ? 1 : prm->particle_integration_steps;  // :34-36
    pp.dtp = prm->time_step / (double)pp.S;                                               // :38
    pp.seed = prm->removal_seed;
    pp.rk2 = prm->integrator == PFEM2GPU_RK2 ? 1 : 0;
    pp.occw = (npe + 63) / 64;
    for (int w = 0; w < OCCW_MAX; ++w) pp.realmask[w] = 0;
    for (int e = 0; e < npe; ++e) {  // extended-part digits, x-major, base q_d + 1
        int r = e;
        bool real = true;
        for (int d = dim - 1; d >= 0; --d) {
            real = real && (r % (pp.q[d] + 1)) < pp.q[d];
            r /= pp.q[d] + 1;
        }
        if (real) pp.realmask[e >> 6] |= 1ull << (e & 63);
    }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->stats, sizeof(DevStats)) != cudaSuccess ||
        cudaMallocHost(&h->stats_h, sizeof(DevStats)) != cudaSuccess ||
        cudaHostAlloc(&h->nf_h, sizeof(unsigned), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&h->nf_d, h->nf_h, 0) != cudaSuccess ||
        cudaMemsetAsync(h->stats, 0, sizeof(DevStats), h->stream) != cudaSuccess) {
        pfem2gpu_destroy(h);
        return PFEM2GPU_ERR_CUDA;
    }
    std::memset(h->stats_h, 0, sizeof(DevStats));
    *out = h;
    return PFEM2GPU_OK;
}

int pfem2gpu_destroy(pfem2gpu_handle* h)
{
    if (!h) return PFEM2GPU_ERR_ARG;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* p : {(void*)h->cv, (void*)h->cd, (void*)h->v2c_off, (void*)h->v2c_cells, (void*)h->d2c_off,
                    (void*)h->d2c_ent, (void*)h->verts, (void*)h->cellX, (void*)h->aff, (void*)h->v2c_dirs,
                    (void*)h->geo32, (void*)h->Vstage, (void*)h->Vstage2, (void*)h->Vout, (void*)h->Vin, h->Vc, h->dVc,
                    (void*)h->key, (void*)h->next, (void*)h->xtmp, (void*)h->head, (void*)h->cs0, (void*)h->cs1,
                    (void*)h->carr, (void*)h->carrs, (void*)h->ccount, (void*)h->cocc, (void*)h->cub, (void*)h->coff,
                    (void*)h->tiles64, (void*)h->gscr, (void*)h->jinv32, (void*)h->xq, (void*)h->nxq,
                    (void*)h->vrec32, (void*)h->dvrec32, h->partials, (void*)h->stats, (void*)h->twisted})
        dfree(p);
    dfree(h->chunk_first);
    for (void* p : {(void*)h->ob_i, (void*)h->ob_c, (void*)h->ob_n, h->xbuf}) dfree(p);
    free_state(h->S0);
    free_state(h->S1);
    free_state(h->T);
    free_win_particles(h->win);
    free_win_mesh(h->win);
    free_fem(h->fem);
    dfree(h->out_slot);
    dfree(h->out_tsum);
    dfree(h->out_dev);
    if (h->out_host) cudaFreeHost(h->out_host);
    if (h->stats_h) cudaFreeHost(h->stats_h);
    if (h->nf_h) cudaFreeHost(h->nf_h);
    for (auto& row : h->move_graph)
        for (auto& g : row)
            if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& g : h->step_graph)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& e : h->open_ev) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    for (auto e : h->ev_pool) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return PFEM2GPU_OK;
}

// Counting sorts on the device (cv, cd and verts already resident): dof ->
// entries k = cell * NV + i ascending per dof, and, unless the caller gave
// them, vertex -> cells ascending with the unit vertex -> centre directions.
// One host read of the vertex map's length sizes its arrays.
static cudaError_t build_maps(pfem2gpu_handle* h, size_t nc, size_t nvx, size_t nd, bool given,
                              const int32_t* v2c_offsets, const int32_t* v2c_cells, const double* v2c_dirs)
{
    const int dim = h->dim, NV = 1 << dim;
    const size_t nmax = std::max(nvx, nd), ntiles = (nmax + WIN_TILE - 1) / WIN_TILE + 1;
    uint32_t *cnt = nullptr, *fill = nullptr, *tsum = nullptr;
    cudaError_t e = cudaSuccess;
    auto done = [&](cudaError_t r) {
        dfree(cnt);
        dfree(fill);
        dfree(tsum);
        return r;
    };
#define BM(x)                                      \
    do {                                           \
        if ((e = (x)) != cudaSuccess) return done(e); \
    } while (0)
    BM(dalloc(&cnt, nmax));
    BM(dalloc(&fill, nmax));
    BM(dalloc(&tsum, ntiles));
    cudaStream_t s = h->stream;
    // dof -> (cell, local vertex)
    BM(cudaMemsetAsync(cnt, 0, nd * 4, s));
    BM(cudaMemsetAsync(fill, 0, nd * 4, s));
    launch_d2c_count((long long)(nc * NV), h->cd, cnt, s);
    launch_win_scan(cnt, (uint32_t)nd, tsum, (uint32_t*)h->d2c_off, s);
    launch_d2c_build((long long)(nc * NV), (int)nd, h->cd, (const uint32_t*)h->d2c_off, fill, h->d2c_ent, s);
    BM(cudaGetLastError());
    // vertex -> cells
    int32_t total = 0;
    if (given) {
        total = v2c_offsets[nvx];
        BM(dalloc(&h->v2c_cells, std::max<size_t>(total, 1)));
        BM(dalloc(&h->v2c_dirs, std::max<size_t>((size_t)total * dim, 1)));
        BM(cudaMemcpyAsync(h->v2c_off, v2c_offsets, (nvx + 1) * 4, cudaMemcpyHostToDevice, s));
        BM(cudaMemcpyAsync(h->v2c_cells, v2c_cells, (size_t)total * 4, cudaMemcpyHostToDevice, s));
        BM(cudaMemcpyAsync(h->v2c_dirs, v2c_dirs, (size_t)total * dim * 8, cudaMemcpyHostToDevice, s));
        BM(cudaStreamSynchronize(s));
        return done(cudaSuccess);
    }
    BM(cudaMemsetAsync(cnt, 0, nvx * 4, s));
    BM(cudaMemsetAsync(fill, 0, nvx * 4, s));
    launch_v2c_count(dim, (int)nc, h->cv, cnt, s);
    launch_win_scan(cnt, (uint32_t)nvx, tsum, (uint32_t*)h->v2c_off, s);
    BM(cudaGetLastError());
    BM(cudaMemcpyAsync(&total, h->v2c_off + nvx, 4, cudaMemcpyDeviceToHost, s));
    BM(cudaStreamSynchronize(s));
    BM(dalloc(&h->v2c_cells, std::max<size_t>(total, 1)));
    BM(dalloc(&h->v2c_dirs, std::max<size_t>((size_t)total * dim, 1)));
    launch_v2c_build(dim, (int)nc, (int)nvx, h->verts, h->cv, (const uint32_t*)h->v2c_off, fill, h->v2c_cells,
                     h->v2c_dirs, s);
    BM(cudaGetLastError());
    BM(cudaStreamSynchronize(s));
#undef BM
    return done(cudaSuccess);
}

int pfem2gpu_set_mesh(pfem2gpu_handle* h, int64_t n_cells, int64_t n_verts, int64_t n_dofs, const double* vertices,
                      const int32_t* cell_vertices, const int32_t* cell_dofs, const int32_t* v2c_offsets,
                      const int32_t* v2c_cells, const double* v2c_dirs)
{
    if (!h || !vertices || !cell_vertices || !cell_dofs) return PFEM2GPU_ERR_ARG;
    if (n_cells < 1 || n_verts < 1 || n_dofs < 1 || n_cells > (1ll << 30) || n_verts > (1ll << 30) ||
        n_dofs > (1ll << 30))
        return fail(h, PFEM2GPU_ERR_ARG, "mesh sizes out of range");
    if ((n_cells + SCAN_TILE - 1) / SCAN_TILE > SCAN_MAX_TILES) return fail(h, PFEM2GPU_ERR_ARG, "too many cells");
    if (h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "mesh change with live particles");
    const int dim = h->dim, NV = 1 << dim;
    for (int64_t k = 0; k < n_cells * NV; ++k) {
        if (cell_vertices[k] < 0 || cell_vertices[k] >= n_verts) return fail(h, PFEM2GPU_ERR_ARG, "bad cell vertex");
        if (cell_dofs[k] < 0 || cell_dofs[k] >= n_dofs) return fail(h, PFEM2GPU_ERR_ARG, "bad cell dof");
    }
    if (n_cells * NV > (int64_t)INT32_MAX) return fail(h, PFEM2GPU_ERR_ARG, "mesh too large");
    // vertex -> cells (ascending) and unit vertex -> centre directions: the
    // caller's maps, checked here, or built on the device further down
    const bool given_maps = v2c_offsets && v2c_cells && v2c_dirs;
    if (given_maps) {
        if (v2c_offsets[0] != 0) return fail(h, PFEM2GPU_ERR_ARG, "v2c offsets must start at 0");
        for (int64_t v = 0; v < n_verts; ++v)
            if (v2c_offsets[v + 1] < v2c_offsets[v]) return fail(h, PFEM2GPU_ERR_ARG, "v2c offsets not monotone");
        for (int64_t k = 0; k < v2c_offsets[n_verts]; ++k)
            if (v2c_cells[k] < 0 || v2c_cells[k] >= n_cells) return fail(h, PFEM2GPU_ERR_ARG, "bad v2c cell");
    }
    // release an older mesh (a failure further down leaves no dangling pointer)
    for (void** p : {(void**)&h->cv, (void**)&h->cd, (void**)&h->v2c_off, (void**)&h->v2c_cells, (void**)&h->d2c_off,
                     (void**)&h->d2c_ent, (void**)&h->verts, (void**)&h->cellX, (void**)&h->aff,
                     (void**)&h->v2c_dirs, (void**)&h->geo32, (void**)&h->Vstage, (void**)&h->Vstage2,
                     (void**)&h->Vout, (void**)&h->Vin, (void**)&h->Vc, (void**)&h->dVc, (void**)&h->head, (void**)&h->cs0,
                     (void**)&h->cs1, (void**)&h->carr, (void**)&h->carrs, (void**)&h->ccount, (void**)&h->cocc,
                     (void**)&h->cub, (void**)&h->coff, (void**)&h->tiles64, (void**)&h->jinv32, (void**)&h->vrec32,
                     (void**)&h->dvrec32, (void**)&h->partials, (void**)&h->twisted}) {
        dfree(*p);
        *p = nullptr;
    }
    free_win_mesh(h->win);
    free_fem(h->fem);
    h->has_mesh = false;
    h->has_projection = false;
    h->nC = (int)n_cells;
    h->nV = (int)n_verts;
    h->nD = (int)n_dofs;
    const size_t nc = n_cells, nvx = n_verts, nd = n_dofs;
    const int VS = dim == 3 ? 4 : 2, PW = dim == 3 ? 32 : 16, GS = dim == 3 ? 24 : 8, AFF = dim * dim + dim;
    CK(dalloc(&h->cv, nc * NV));
    CK(dalloc(&h->cd, nc * NV));
    CK(dalloc(&h->verts, nvx * dim));
    CK(dalloc(&h->v2c_off, nvx + 1));
    CK(dalloc(&h->d2c_off, nd + 1));
    CK(dalloc(&h->d2c_ent, nc * NV));
    CK(dalloc(&h->cellX, nc * NV * dim));
    CK(dalloc(&h->aff, nc * AFF));
    CK(dalloc(&h->geo32, nc * GS));
    CK(dalloc(&h->Vstage, nd * dim));
    CK(dalloc(&h->Vstage2, nd * dim));
    CK(dalloc(&h->Vin, nd * dim));
    CK(dalloc(&h->Vout, nd * dim));
    const size_t vcn = h->prec == PFEM2GPU_FP64 ? nc * NV * VS : 1;
    CK(cudaMalloc(&h->Vc, vcn * esize(h)));
    CK(cudaMalloc(&h->dVc, vcn * esize(h)));
    CK(dalloc(&h->head, nc));
    CK(dalloc(&h->cs0, nc + 1));
    CK(dalloc(&h->cs1, nc + 1));
    const int occw = h->pp.occw;
    CK(dalloc(&h->carr, nc));
    CK(dalloc(&h->carrs, nc * ARRCAP));
    CK(dalloc(&h->ccount, nc));
    CK(dalloc(&h->cocc, nc * occw));
    CK(dalloc(&h->cub, nc));
    CK(dalloc(&h->coff, nc + 1));
    CK(dalloc(&h->tiles64, SCAN_MAX_TILES));
    CK(cudaMemsetAsync(h->carr, 0, nc * 4, h->stream));
    CK(cudaMemsetAsync(h->ccount, 0, nc * 4, h->stream));
    CK(cudaMemsetAsync(h->cocc, 0, nc * occw * 8, h->stream));
    if (h->prec == PFEM2GPU_FP32) {
        const size_t rec = (size_t)(dim == 3 ? 7 : 3) * 4;
        CK(dalloc(&h->vrec32, nc * rec));
        CK(dalloc(&h->dvrec32, nc * rec));
        CK(cudaMemsetAsync(h->vrec32, 0, nc * rec * 4, h->stream));
        CK(cudaMemsetAsync(h->dvrec32, 0, nc * rec * 4, h->stream));
    }
    CK(dalloc(&h->jinv32, nc * (dim == 3 ? 12 : 8)));
    CK(dalloc(&h->twisted, 1));
    CK(cudaMemsetAsync(h->twisted, 0, 4, h->stream));
    CK(cudaMalloc(&h->partials, nc * PW * esize(h)));
    CK(cudaMemcpyAsync(h->cv, cell_vertices, nc * NV * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->cd, cell_dofs, nc * NV * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->verts, vertices, nvx * dim * 8, cudaMemcpyHostToDevice, h->stream));
    CK(build_maps(h, nc, nvx, nd, given_maps, v2c_offsets, v2c_cells, v2c_dirs));
    CK(cudaMemsetAsync(h->Vc, 0, vcn * esize(h), h->stream));
    CK(cudaMemsetAsync(h->dVc, 0, vcn * esize(h), h->stream));
    run(h, "fill", [&] { return launch_fill_u32(h->head, (uint32_t)nc, LOST, h->stream); });
    CK(cudaMemsetAsync(h->Vstage, 0, nd * dim * 8, h->stream));
    run(h, "cell_setup",
        [&] {
            return launch_cell_setup(dim, h->nC, h->verts, h->cv, h->cellX, h->aff, h->geo32, h->jinv32, h->twisted,
                                     h->stream);
        });
    uint32_t twisted = 0;
    CK(cudaMemcpyAsync(&twisted, h->twisted, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));  // host vectors above go out of scope
    h->all_affine = twisted == 0;
    h->has_mesh = true;
    h->vaos_valid = false;
    h->gen++;
    return check_async(h);
}

// Seeding checks its host V before it allocates anything (stage_v checks the
// V of the other calls while it is uploaded).
static int host_velocity_ok(pfem2gpu_handle* h, const double* V, bool device)
{
    if (device || all_finite(V, (size_t)h->dim * h->nD)) return PFEM2GPU_OK;
    return fail(h, PFEM2GPU_ERR_ARG, "non-finite nodal velocity");
}

static int seed_impl(pfem2gpu_handle* h, const double* V, bool device)
{
    if (!h || !V) return PFEM2GPU_ERR_ARG;
    if (h->move_phase) return fail(h, PFEM2GPU_ERR_STATE, "inside a partitioned move");
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "seed before set_mesh");
    if (h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "seed called twice");
    // a partitioned handle seeds its own cells; ids count every cell's parts
    const int64_t own = (h->pend < 0 ? h->nC : h->pend) - h->pbeg;
    const uint64_t n = (uint64_t)own * h->pp.npart, n_all = (uint64_t)h->nC * h->pp.npart;
    int rc = host_velocity_ok(h, V, device);
    if (rc) return rc;
    if ((rc = ensure_capacity(h, n, h->prm.capacity > 0 ? (uint64_t)h->prm.capacity : 2 * n))) return rc;
    if ((rc = stage_v(h, V, nullptr, device))) return rc;
    StepArgs a = args(h);
    run(h, "seed", [&] { return launch_seed(h->dim, h->prec, a, h->cs0, h->stream); });
    run(h, "finalize", [&] { return launch_set_state(h->stats, (long long)n, -1, (long long)n_all, h->stream); });
    h->has_particles = true;
    h->partials_valid = false;
    h->pending_correct = false;
    return check_async(h);
}

int pfem2gpu_seed(pfem2gpu_handle* h, const double* V) { return seed_impl(h, V, false); }
int pfem2gpu_seed_device(pfem2gpu_handle* h, const double* dV) { return seed_impl(h, dV, true); }

static int correct_impl(pfem2gpu_handle* h, const double* V, const double* Vold, bool device)
{
    if (!h || !V || !Vold) return PFEM2GPU_ERR_ARG;
    if (h->move_phase) return fail(h, PFEM2GPU_ERR_STATE, "inside a partitioned move");
    if (!h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "correct before seed");
    int rc = apply_pending_correction(h);
    if (rc) return rc;
    if ((rc = stage_v(h, V, Vold, device))) return rc;
    h->pending_correct = true;
    h->partials_valid = false;
    return PFEM2GPU_OK;
}

int pfem2gpu_correct(pfem2gpu_handle* h, const double* V, const double* Vold) { return correct_impl(h, V, Vold, false); }
int pfem2gpu_correct_device(pfem2gpu_handle* h, const double* dV, const double* dVold)
{
    return correct_impl(h, dV, dVold, true);
}

// Vold = the handle's last projection, which stays on the device.
static int correct_from_projection(pfem2gpu_handle* h, const double* V, bool device)
{
    if (!h || !V) return PFEM2GPU_ERR_ARG;
    if (!h->has_projection) return fail(h, PFEM2GPU_ERR_STATE, "correct from projection before any projection");
    return correct_impl(h, V, h->Vout, device);
}

int pfem2gpu_correct_from_projection(pfem2gpu_handle* h, const double* V)
{
    return correct_from_projection(h, V, false);
}
int pfem2gpu_correct_from_projection_device(pfem2gpu_handle* h, const double* dV)
{
    return correct_from_projection(h, dV, true);
}

static int move_impl(pfem2gpu_handle* h, const double* V, bool device)
{
    if (!h) return PFEM2GPU_ERR_ARG;
    if (h->move_phase) return fail(h, PFEM2GPU_ERR_STATE, "inside a partitioned move");
    if (!h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "move before seed");
    if (split(h)) return fail(h, PFEM2GPU_ERR_STATE, "a partitioned handle moves with pfem2gpu_move_exchange_*");
    if (V) {
        // keep a staged correction: only V is re-staged
        int rc = stage_v(h, V, nullptr, device);
        if (rc) return rc;
    }
    return do_move(h);
}

int pfem2gpu_move(pfem2gpu_handle* h, const double* V) { return move_impl(h, V, false); }
int pfem2gpu_move_device(pfem2gpu_handle* h, const double* dV) { return move_impl(h, dV, true); }

static int project_impl(pfem2gpu_handle* h, double* out, bool device)
{
    if (!h || !out) return PFEM2GPU_ERR_ARG;
    if (h->move_phase) return fail(h, PFEM2GPU_ERR_STATE, "inside a partitioned move");
    if (!h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "project before seed");
    int rc = apply_pending_correction(h);
    if (rc) return rc;
    StepArgs a = args(h);
    if (!h->partials_valid) {
        run(h, "partials", [&] { return launch_partials(h->dim, h->prec, a, h->cs0, h->stream); });
        h->partials_valid = true;
    }
    CK(cudaMemsetAsync(&h->stats->nan_dofs, 0, sizeof(unsigned long long), h->stream));
    run(h, "gather", [&] { return launch_gather(h->dim, h->prec, a, h->prm.empty_dof_policy == 1, h->stream); });
    if ((rc = check_async(h))) return rc;
    h->has_projection = true;
    const size_t bytes = (size_t)h->dim * h->nD * sizeof(double);
    if (device) {
        if (out != h->Vout) CK(cudaMemcpyAsync(out, h->Vout, bytes, cudaMemcpyDeviceToDevice, h->stream));
        return PFEM2GPU_OK;
    }
    CK(cudaMemcpyAsync(out, h->Vout, bytes, cudaMemcpyDeviceToHost, h->stream));
    if ((rc = sync_stats(h))) return rc;
    return maybe_grow(h);
}

int pfem2gpu_project(pfem2gpu_handle* h, double* V_out) { return project_impl(h, V_out, false); }
int pfem2gpu_project_device(pfem2gpu_handle* h, double* dV_out) { return project_impl(h, dV_out, true); }

int pfem2gpu_step_device(pfem2gpu_handle* h, const double* dV, const double* dVold, double* dV_out)
{
    if (!h || !dV || !dV_out) return PFEM2GPU_ERR_ARG;
    if (h->move_phase) return fail(h, PFEM2GPU_ERR_STATE, "inside a partitioned move");
    if (!h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "step before seed");
    if (split(h)) return fail(h, PFEM2GPU_ERR_STATE, "a partitioned handle moves with pfem2gpu_move_exchange_*");
    if (!dVold) {  // the reference's data flow: Vold = the last projection
        if (!h->has_projection) return fail(h, PFEM2GPU_ERR_STATE, "step from projection before any projection");
        dVold = h->Vout;
    }
    int rc = apply_pending_correction(h);
    if (rc) return rc;
    rc = graphed(h, h->step_graph[h->parity], dV, dVold, dV_out, [&]() -> int {
        // kernels only: the staging kernel keeps the copy of V, the write
        // pass resets the counters, the gather writes the caller's vector
        int r = stage_v(h, dV, dVold, true);
        if (r) return r;
        if ((r = enqueue_move(h, 1, 1))) return r;
        StepArgs a = args(h);
        a.Vout = dV_out;
        a.Vout2 = dV_out != h->Vout ? h->Vout : nullptr;  // the handle keeps its last projection
        run(h, "gather", [&] { return launch_gather(h->dim, h->prec, a, h->prm.empty_dof_policy == 1, h->stream); });
        return PFEM2GPU_OK;
    });
    if (rc) return rc;
    h->has_projection = true;
    h->vaos_valid = true;
    h->pending_correct = false;
    swap_state(h);
    return check_async(h);
}

int pfem2gpu_get_particles(pfem2gpu_handle* h, uint32_t* id, int32_t* cell, double* x, double* xi, double* v,
                           int64_t capacity, int64_t* n)
{
    if (!h || !n) return PFEM2GPU_ERR_ARG;
    if (h->move_phase) return fail(h, PFEM2GPU_ERR_STATE, "inside a partitioned move");
    *n = 0;
    if (!h->has_particles) return PFEM2GPU_OK;
    int rc = apply_pending_correction(h);
    if (rc) return rc;
    if ((rc = sync_stats(h))) return rc;
    const int64_t np = (int64_t)h->stats_h->n_particles;
    const int64_t ns = (int64_t)h->stats_h->n_slots;
    *n = np;
    if (capacity < np) return fail(h, PFEM2GPU_ERR_ARG, "output arrays too small");
    const int dim = h->dim;
    // slots of the current state; empty slots (cell HOLE) are skipped
    std::vector<uint32_t> cells(ns), ids;
    CK(cudaMemcpyAsync(cells.data(), h->S0.cell, ns * 4, cudaMemcpyDeviceToHost, h->stream));
    if (id) {
        ids.resize(ns);
        CK(cudaMemcpyAsync(ids.data(), h->S0.id, ns * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    std::vector<int64_t> live;
    live.reserve(np);
    for (int64_t i = 0; i < ns; ++i)
        if (cells[i] != HOLE) live.push_back(i);
    if ((int64_t)live.size() != np) return fail(h, PFEM2GPU_ERR_DEVICE, "slot count mismatch");
    for (int64_t k = 0; k < np; ++k) {
        if (id) id[k] = ids[live[k]];
        if (cell) cell[k] = (int32_t)cells[live[k]];
    }
    std::vector<double> tmp(ns);
    std::vector<float> tmpf(ns);
    auto fetch = [&](void* const* src, double* dst) -> int {
        for (int d = 0; d < dim; ++d) {
            if (h->prec == PFEM2GPU_FP64) {
                CK(cudaMemcpyAsync(tmp.data(), src[d], ns * 8, cudaMemcpyDeviceToHost, h->stream));
                CK(cudaStreamSynchronize(h->stream));
                for (int64_t k = 0; k < np; ++k) dst[k * dim + d] = tmp[live[k]];
            } else {
                CK(cudaMemcpyAsync(tmpf.data(), src[d], ns * 4, cudaMemcpyDeviceToHost, h->stream));
                CK(cudaStreamSynchronize(h->stream));
                for (int64_t k = 0; k < np; ++k) dst[k * dim + d] = (double)tmpf[live[k]];
            }
        }
        return PFEM2GPU_OK;
    };
    if (xi && (rc = fetch(h->S0.xi, xi))) return rc;
    if (v && (rc = fetch(h->S0.v, v))) return rc;
    if (x) {
        if (h->prec == PFEM2GPU_FP64) {
            if ((rc = fetch(h->S0.x, x))) return rc;
        } else {
            StepArgs a = args(h);
            run(h, "positions", [&] { return launch_positions32(dim, a, h->xtmp, h->stream); });
            std::vector<double> xs((size_t)ns * dim);
            CK(cudaMemcpyAsync(xs.data(), h->xtmp, ns * dim * 8, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            for (int64_t k = 0; k < np; ++k)
                for (int d = 0; d < dim; ++d) x[k * dim + d] = xs[(size_t)live[k] * dim + d];
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    return check_async(h);
}

int pfem2gpu_set_particles(pfem2gpu_handle* h, int64_t n, const uint32_t* id, const int32_t* cell, const double* x,
                           const double* xi, const double* v, uint32_t next_id)
{
    if (!h || n < 0 || (n > 0 && (!id || !cell || !xi || !v))) return PFEM2GPU_ERR_ARG;
    if (h->prec == PFEM2GPU_FP64 && n > 0 && !x) return PFEM2GPU_ERR_ARG;
    if (h->move_phase) return fail(h, PFEM2GPU_ERR_STATE, "inside a partitioned move");
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "set_particles before set_mesh");
    const int64_t cb = h->pbeg, ce = h->pend < 0 ? h->nC : h->pend;
    for (int64_t i = 0; i < n; ++i)
        if (cell[i] < cb || cell[i] >= ce) return fail(h, PFEM2GPU_ERR_ARG, "particle cell outside the handle's cells");
    // reference coordinates inside the unit cell (GeometryInfo::is_inside_unit_cell, the test every
    // particle of the reference passed), finite velocities and positions
    for (int64_t i = 0; i < n * h->dim; ++i) {
        if (!(xi[i] >= 0.0 && xi[i] <= 1.0)) return fail(h, PFEM2GPU_ERR_ARG, "particle reference coordinate outside [0, 1]");
        if (!std::isfinite(v[i])) return fail(h, PFEM2GPU_ERR_ARG, "non-finite particle velocity");
        if (x && h->prec == PFEM2GPU_FP64 && !std::isfinite(x[i])) return fail(h, PFEM2GPU_ERR_ARG, "non-finite particle position");
    }
    int rc = ensure_capacity(h, (uint64_t)n, std::max<uint64_t>((uint64_t)n + (uint64_t)h->nC * h->pp.npart, h->cap));
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    const int dim = h->dim;
    CK(cudaMemcpyAsync(h->S0.id, id, n * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->S0.cell, cell, n * 4, cudaMemcpyHostToDevice, h->stream));
    std::vector<double> tmp(n);
    std::vector<float> tmpf(n);
    auto put = [&](const double* src, void* const* dst) -> int {
        for (int d = 0; d < dim; ++d) {
            if (h->prec == PFEM2GPU_FP64 || dst == h->T.x) {
                for (int64_t i = 0; i < n; ++i) tmp[i] = src[i * dim + d];
                CK(cudaMemcpyAsync(dst[d], tmp.data(), n * 8, cudaMemcpyHostToDevice, h->stream));
            } else {
                for (int64_t i = 0; i < n; ++i) tmpf[i] = (float)src[i * dim + d];
                CK(cudaMemcpyAsync(dst[d], tmpf.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
            }
            CK(cudaStreamSynchronize(h->stream));
        }
        return PFEM2GPU_OK;
    };
    if ((rc = put(xi, h->T.xi))) return rc;
    if ((rc = put(v, h->T.v))) return rc;
    if (h->prec == PFEM2GPU_FP64 && (rc = put(x, h->T.x))) return rc;
    CK(cudaMemsetAsync(h->stats, 0, sizeof(DevStats), h->stream));
    run(h, "finalize", [&] { return launch_set_state(h->stats, n, next_id, 0, h->stream); });
    CK(cudaMemsetAsync(h->cs0, 0, (h->nC + 1) * sizeof(uint32_t), h->stream));
    StepArgs a = args(h);
    a.apply_counts = 0;
    run(h, "rekey", [&] { return launch_rekey(h->dim, h->prec, a, h->stream); });
    h->has_particles = true;
    h->pending_correct = false;
    if ((rc = write_and_swap(h, a, 0))) return rc;
    return sync_stats(h);
}

// ---------------------------------------------------------------------------
// Cell-range partitions (shard.cuh): one handle per GPU, each owning a
// contiguous range of cells of the same mesh.
// ---------------------------------------------------------------------------

int pfem2gpu_set_partition(pfem2gpu_handle* h, int64_t cell_begin, int64_t cell_end)
{
    if (!h) return PFEM2GPU_ERR_ARG;
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "set_partition before set_mesh");
    if (h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "set_partition after particles exist");
    if (cell_begin < 0 || cell_begin > cell_end || cell_end > h->nC) return fail(h, PFEM2GPU_ERR_ARG, "bad cell range");
    h->pbeg = cell_begin;
    h->pend = cell_end;
    h->gen++;
    return PFEM2GPU_OK;
}

// Device staging of `bytes` for an exchange.
static int xbuf_reserve(pfem2gpu_handle* h, size_t bytes)
{
    if (bytes <= h->xbuf_bytes) return PFEM2GPU_OK;
    CK(cudaStreamSynchronize(h->stream));
    dfree(h->xbuf);
    h->xbuf = nullptr;
    h->xbuf_bytes = 0;
    CK(cudaMalloc(&h->xbuf, bytes));
    h->xbuf_bytes = bytes;
    return PFEM2GPU_OK;
}

// Offsets of id, cell, x, xi, v for n particles in the staging buffer.
struct XLayout {
    size_t id, cell, x, xi, v, total;
};
static XLayout xlayout(int dim, size_t n)
{
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    XLayout L;
    L.id = 0;
    L.cell = al(4 * n);
    L.x = L.cell + al(4 * n);
    L.xi = L.x + al(8 * n * dim);
    L.v = L.xi + al(8 * n * dim);
    L.total = L.v + al(8 * n * dim) + 256;
    return L;
}

int pfem2gpu_move_exchange_begin(pfem2gpu_handle* h, const double* V, int64_t* n_out)
{
    if (!h || !n_out) return PFEM2GPU_ERR_ARG;
    if (!h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "move before seed");
    if (h->move_phase != 0) return fail(h, PFEM2GPU_ERR_STATE, "a partitioned move is in progress");
    int rc;
    if (V && (rc = stage_v(h, V, nullptr, false))) return rc;
    if (!h->vaos_valid) return fail(h, PFEM2GPU_ERR_STATE, "move without a velocity");
    if (h->ob_cap < h->cap) {
        CK(cudaStreamSynchronize(h->stream));
        for (void* p : {(void*)h->ob_i, (void*)h->ob_c}) dfree(p);
        h->ob_i = h->ob_c = nullptr;
        h->ob_cap = 0;
        CK(dalloc(&h->ob_i, h->cap));
        CK(dalloc(&h->ob_c, h->cap));
        h->ob_cap = h->cap;
    }
    if (!h->ob_n) CK(dalloc(&h->ob_n, 1));
    StepArgs a = args(h);
    a.do_correct = h->pending_correct ? 1 : 0;
    h->pending_correct = false;
    h->partials_valid = false;
    CK(cudaMemsetAsync(h->ob_n, 0, sizeof(uint32_t), h->stream));
    run(h, "advect", [&] { return launch_advect(h->dim, h->prec, a, h->stream); });
    run(h, "cross", [&] { return launch_cross(h->dim, h->prec, a, h->stream); });
    run(h, "outbox", [&] { return launch_outbox(h->prec, a, h->ob_i, h->ob_c, h->ob_n, h->ob_cap, h->stream); });
    if ((rc = check_async(h))) return rc;
    uint32_t n = 0;
    CK(cudaMemcpyAsync(&n, h->ob_n, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    if ((rc = sync_stats(h))) return rc;  // also the current slot count, for the inbox
    h->ob_count = n < h->ob_cap ? n : h->ob_cap;
    h->move_phase = 1;
    *n_out = h->ob_count;
    return PFEM2GPU_OK;
}

int pfem2gpu_move_outbox(pfem2gpu_handle* h, uint32_t* id, int32_t* cell, double* x, double* xi, double* v,
                         int64_t capacity, int64_t* n)
{
    if (!h || !n) return PFEM2GPU_ERR_ARG;
    if (h->move_phase != 1) return fail(h, PFEM2GPU_ERR_STATE, "outbox outside a partitioned move");
    const size_t m = h->ob_count, dim = (size_t)h->dim;
    *n = (int64_t)m;
    if (capacity < (int64_t)m) return fail(h, PFEM2GPU_ERR_ARG, "outbox arrays too small");
    if (m == 0) return PFEM2GPU_OK;
    if (!id || !cell || !xi || !v || (h->prec == PFEM2GPU_FP64 && !x)) return PFEM2GPU_ERR_ARG;
    const XLayout L = xlayout(h->dim, m);
    int rc = xbuf_reserve(h, L.total);
    if (rc) return rc;
    char* b = static_cast<char*>(h->xbuf);
    StepArgs a = args(h);
    run(h, "outbox_pack", [&] {
        return launch_outbox_pack(h->dim, h->prec, a, h->ob_i, h->ob_c, (uint32_t)m, (uint32_t*)(b + L.id),
                                  (int32_t*)(b + L.cell), (double*)(b + L.x), (double*)(b + L.xi), (double*)(b + L.v),
                                  h->stream);
    });
    if ((rc = check_async(h))) return rc;
    CK(cudaMemcpyAsync(id, b + L.id, 4 * m, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(cell, b + L.cell, 4 * m, cudaMemcpyDeviceToHost, h->stream));
    if (h->prec == PFEM2GPU_FP64) CK(cudaMemcpyAsync(x, b + L.x, 8 * m * dim, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(xi, b + L.xi, 8 * m * dim, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(v, b + L.v, 8 * m * dim, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PFEM2GPU_OK;
}

int pfem2gpu_move_inbox(pfem2gpu_handle* h, int64_t n, const uint32_t* id, const int32_t* cell, const double* x,
                        const double* xi, const double* v, int64_t* n_seeds)
{
    if (!h || !n_seeds || n < 0 || (n > 0 && (!id || !cell || !xi || !v))) return PFEM2GPU_ERR_ARG;
    if (h->prec == PFEM2GPU_FP64 && n > 0 && !x) return PFEM2GPU_ERR_ARG;
    if (h->move_phase != 1) return fail(h, PFEM2GPU_ERR_STATE, "inbox outside a partitioned move");
    const int64_t cb = h->pbeg, ce = h->pend < 0 ? h->nC : h->pend;
    for (int64_t i = 0; i < n; ++i)
        if (cell[i] < cb || cell[i] >= ce) return fail(h, PFEM2GPU_ERR_ARG, "inbox particle outside the handle's cells");
    for (int64_t i = 0; i < n * h->dim; ++i)
        if (!(xi[i] >= 0.0 && xi[i] <= 1.0) || !std::isfinite(v[i]))
            return fail(h, PFEM2GPU_ERR_ARG, "inbox particle with a bad reference coordinate or velocity");
    const uint64_t base = h->stats_h->n_slots;  // read when the move began
    if (base + (uint64_t)n > h->cap) return fail(h, PFEM2GPU_ERR_CAPACITY, "inbox beyond the particle capacity");
    StepArgs a = args(h);
    int rc;
    if (n > 0) {
        const size_t m = (size_t)n, dim = (size_t)h->dim;
        const XLayout L = xlayout(h->dim, m);
        if ((rc = xbuf_reserve(h, L.total))) return rc;
        char* b = static_cast<char*>(h->xbuf);
        CK(cudaMemcpyAsync(b + L.id, id, 4 * m, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(b + L.cell, cell, 4 * m, cudaMemcpyHostToDevice, h->stream));
        if (h->prec == PFEM2GPU_FP64)
            CK(cudaMemcpyAsync(b + L.x, x, 8 * m * dim, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(b + L.xi, xi, 8 * m * dim, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(b + L.v, v, 8 * m * dim, cudaMemcpyHostToDevice, h->stream));
        run(h, "inbox", [&] {
            return launch_inbox(h->dim, h->prec, a, (uint32_t)m, (uint32_t)base, (const uint32_t*)(b + L.id),
                                (const int32_t*)(b + L.cell), (const double*)(b + L.x), (const double*)(b + L.xi),
                                (const double*)(b + L.v), h->stream);
        });
    }
    run(h, "slots_scan", [&] { return launch_slots_scan(a, h->tiles64, h->stream); });
    if ((rc = check_async(h))) return rc;
    unsigned long long po = 0;
    CK(cudaMemcpyAsync(&po, h->coff + h->nC, sizeof(po), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *n_seeds = (int64_t)(po >> 32);
    h->move_phase = 2;
    return PFEM2GPU_OK;
}

int pfem2gpu_move_exchange_end(pfem2gpu_handle* h, uint32_t first_id, uint32_t next_id)
{
    if (!h) return PFEM2GPU_ERR_ARG;
    if (h->move_phase != 2) return fail(h, PFEM2GPU_ERR_STATE, "exchange_end before the inbox");
    StepArgs a = args(h);
    a.count_step = 1;
    a.reset_nan = 0;
    run(h, "finalize", [&] { return launch_set_state(h->stats, -1, first_id, 0, h->stream); });
    run(h, "write", [&] { return launch_write(h->dim, h->prec, a, h->stream); });
    swap_state(h);
    run(h, "finalize", [&] { return launch_set_state(h->stats, -1, next_id, 0, h->stream); });
    h->move_phase = 0;
    int rc = check_async(h);
    if (rc || (rc = sync_stats(h))) return rc;
    return maybe_grow(h);
}

static int partials_io(pfem2gpu_handle* h, int64_t n, const int32_t* cells, double* out, const double* in)
{
    if (!h || n < 0 || (n > 0 && !cells)) return PFEM2GPU_ERR_ARG;
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "partials before set_mesh");
    for (int64_t i = 0; i < n; ++i)
        if (cells[i] < 0 || cells[i] >= h->nC) return fail(h, PFEM2GPU_ERR_ARG, "bad cell");
    if (!h->has_particles) return fail(h, PFEM2GPU_ERR_STATE, "partials before seed");
    if (h->move_phase != 0) return fail(h, PFEM2GPU_ERR_STATE, "partials inside a partitioned move");
    int rc = apply_pending_correction(h);
    if (rc) return rc;
    if (!h->partials_valid) {
        StepArgs a = args(h);
        run(h, "partials", [&] { return launch_partials(h->dim, h->prec, a, h->cs0, h->stream); });
        h->partials_valid = true;
    }
    if (n == 0) return check_async(h);
    const int pw = h->dim == 3 ? 32 : 16;
    const size_t cb = ((size_t)4 * n + 255) & ~(size_t)255, vb = (size_t)8 * n * pw;
    if ((rc = xbuf_reserve(h, cb + vb))) return rc;
    char* b = static_cast<char*>(h->xbuf);
    CK(cudaMemcpyAsync(b, cells, 4 * n, cudaMemcpyHostToDevice, h->stream));
    if (in) CK(cudaMemcpyAsync(b + cb, in, vb, cudaMemcpyHostToDevice, h->stream));
    run(h, "partials_io", [&] {
        return launch_partials_io(h->prec, h->partials, pw, (uint32_t)n, (const int32_t*)b, (double*)(b + cb),
                                  in ? 0 : 1, h->stream);
    });
    if ((rc = check_async(h))) return rc;
    if (out) CK(cudaMemcpyAsync(out, b + cb, vb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PFEM2GPU_OK;
}

int pfem2gpu_get_partials(pfem2gpu_handle* h, int64_t n, const int32_t* cells, double* out)
{
    if (!out && n > 0) return PFEM2GPU_ERR_ARG;
    return partials_io(h, n, cells, out, nullptr);
}

int pfem2gpu_set_partials(pfem2gpu_handle* h, int64_t n, const int32_t* cells, const double* in)
{
    if (!in && n > 0) return PFEM2GPU_ERR_ARG;
    return partials_io(h, n, cells, nullptr, in);
}

int pfem2gpu_get_stats(pfem2gpu_handle* h, pfem2gpu_stats* out)
{
    if (!h || !out) return PFEM2GPU_ERR_ARG;
    int rc = sync_stats(h);
    const DevStats& s = *h->stats_h;
    out->n_particles = (int64_t)s.n_particles;
    out->lost = (int64_t)s.lost;
    out->removed = (int64_t)s.removed;
    out->seeded = (int64_t)s.seeded;
    out->map_failures = (int64_t)s.map_failures;
    out->near_face = (int64_t)s.near_face;
    out->searched = (int64_t)s.searched;
    out->nan_dofs = (int64_t)s.nan_dofs;
    out->fallback64 = (int64_t)s.fallback64;
    out->particle_steps = (int64_t)s.particle_steps;
    out->next_id = s.next_id;
    out->error_flags = s.error_flags;
    if (rc == PFEM2GPU_OK && h->has_particles) return maybe_grow(h);
    return rc == PFEM2GPU_ERR_CAPACITY || rc == PFEM2GPU_ERR_DEVICE ? PFEM2GPU_OK : rc;
}

int pfem2gpu_reset_stats(pfem2gpu_handle* h)
{
    if (!h) return PFEM2GPU_ERR_ARG;
    CK(cudaMemcpyAsync(h->stats_h, h->stats, sizeof(DevStats), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    DevStats s{};
    s.n_particles = h->stats_h->n_particles;
    s.next_id = h->stats_h->next_id;
    s.nan_dofs = h->stats_h->nan_dofs;
    s.particle_steps = h->stats_h->particle_steps;
    s.n_slots = h->stats_h->n_slots;
    *h->stats_h = s;
    CK(cudaMemcpyAsync(h->stats, h->stats_h, sizeof(DevStats), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PFEM2GPU_OK;
}

int pfem2gpu_synchronize(pfem2gpu_handle* h)
{
    if (!h) return PFEM2GPU_ERR_ARG;
    CK(cudaStreamSynchronize(h->stream));
    if (h->profiling) collect_profile(h);
    return check_async(h);
}

int pfem2gpu_get_stream(pfem2gpu_handle* h, void** stream)
{
    if (!h || !stream) return PFEM2GPU_ERR_ARG;
    *stream = (void*)h->stream;
    return PFEM2GPU_OK;
}

int pfem2gpu_host_register(void* ptr, size_t bytes)
{
    if (!ptr || !bytes) return PFEM2GPU_ERR_ARG;
    return cudaHostRegister(ptr, bytes, cudaHostRegisterDefault) == cudaSuccess ? PFEM2GPU_OK : PFEM2GPU_ERR_CUDA;
}

int pfem2gpu_host_unregister(void* ptr)
{
    if (!ptr) return PFEM2GPU_ERR_ARG;
    return cudaHostUnregister(ptr) == cudaSuccess ? PFEM2GPU_OK : PFEM2GPU_ERR_CUDA;
}

int pfem2gpu_profile(pfem2gpu_handle* h, int enable)
{
    if (!h) return PFEM2GPU_ERR_ARG;
    collect_profile(h);
    if (enable) h->prof.clear();
    h->profiling = enable != 0;
    return PFEM2GPU_OK;
}

int pfem2gpu_profile_report(pfem2gpu_handle* h, char* buf, int64_t len)
{
    if (!h || !buf || len <= 0) return PFEM2GPU_ERR_ARG;
    collect_profile(h);
    std::string s = "{";
    bool first = true;
    for (auto& kv : h->prof) {
        char tmp[256];
        std::snprintf(tmp, sizeof tmp, "%s\"%s\": [%.6f, %lld]", first ? "" : ", ", kv.first.c_str(),
                      kv.second.first, kv.second.second);
        s += tmp;
        first = false;
    }
    s += "}";
    if ((int64_t)s.size() + 1 > len) return PFEM2GPU_ERR_ARG;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return PFEM2GPU_OK;
}

int pfem2gpu_launch_count(pfem2gpu_handle* h, uint64_t* count)
{
    if (!h || !count) return PFEM2GPU_ERR_ARG;
    *count = h->launches;
    return PFEM2GPU_OK;
}

int pfem2gpu_pack_output_device(pfem2gpu_handle* h, float* d_out, int64_t capacity, int64_t* n)
{
    if (!h || !n || (capacity > 0 && !d_out)) return PFEM2GPU_ERR_ARG;
    if (h->move_phase) return fail(h, PFEM2GPU_ERR_STATE, "inside a partitioned move");
    return pack_output(h, d_out, capacity, n);
}

int pfem2gpu_write_vtu(pfem2gpu_handle* h, const char* path)
{
    if (!h || !path) return PFEM2GPU_ERR_ARG;
    // the live particles' positions and velocities packed on the device as
    // the Float32 values the file holds, one device-to-host copy
    int rc = apply_pending_correction(h);
    if (rc) return rc;
    if (h->has_particles && (rc = sync_stats(h))) return rc;
    const int64_t want = h->has_particles ? (int64_t)h->stats_h->n_particles : 0;
    if (want > 0 && (uint64_t)want > h->out_dcap) {
        dfree(h->out_dev);
        if (h->out_host) cudaFreeHost(h->out_host);
        h->out_dev = nullptr;
        h->out_host = nullptr;
        h->out_dcap = 0;
        CK(dalloc(&h->out_dev, (size_t)want * 6));
        CK(cudaMallocHost(&h->out_host, (size_t)want * 6 * sizeof(float)));
        h->out_dcap = (uint32_t)want;
    }
    int64_t n = 0;
    if ((rc = pack_output(h, h->out_dev, want, &n))) return rc;
    if (n > 0) CK(cudaMemcpyAsync(h->out_host, h->out_dev, (size_t)n * 6 * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const float* xp = h->out_host;
    const float* vp = h->out_host ? h->out_host + (size_t)n * 3 : nullptr;
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(h, PFEM2GPU_ERR_ARG, std::string("cannot open ") + path);
    // layout of output_particle_solution, src/pfem2particlehandler.cpp:223-291
    std::fprintf(f, "<?xml version=\"1.0\" ?> \n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" "
                    "byte_order=\"LittleEndian\">\n  <UnstructuredGrid>\n");
    std::fprintf(f, "    <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\">\n", (long long)n, (long long)n);
    std::fprintf(f, "      <Points>\n        <DataArray type=\"Float32\" NumberOfComponents=\"3\" Format=\"ascii\">\n");
    for (int64_t i = 0; i < n; ++i)
        std::fprintf(f, "          %g %.6f %.6f\n", (double)xp[3 * i], (double)xp[3 * i + 1], (double)xp[3 * i + 2]);
    std::fprintf(f, "        </DataArray>\n      </Points>\n      <Cells>\n");
    std::fprintf(f, "        <DataArray type=\"Int32\" Name=\"connectivity\" Format=\"ascii\">\n");
    for (int64_t i = 0; i < n; ++i) std::fprintf(f, "          %lld\n", (long long)i);
    std::fprintf(f, "        </DataArray>\n        <DataArray type=\"Int32\" Name=\"offsets\" Format=\"ascii\">\n        ");
    for (int64_t i = 0; i < n; ++i) std::fprintf(f, "  %lld", (long long)i + 1);
    std::fprintf(f, "\n        </DataArray>\n        <DataArray type=\"Int32\" Name=\"types\" Format=\"ascii\">\n        ");
    for (int64_t i = 0; i < n; ++i) std::fprintf(f, "  1");
    std::fprintf(f, "\n        </DataArray>\n      </Cells>\n      <PointData Scalars=\"scalars\">\n");
    std::fprintf(f, "        <DataArray type=\"Float32\" Name=\"velocity\" NumberOfComponents=\"3\" Format=\"ascii\">\n");
    for (int64_t i = 0; i < n; ++i)
        std::fprintf(f, "          %g %.6f %.6f\n", (double)vp[3 * i], (double)vp[3 * i + 1], (double)vp[3 * i + 2]);
    std::fprintf(f, "        </DataArray>\n        <DataArray type=\"Float32\" Name=\"subdomain\" Format=\"ascii\">\n        ");
    for (int64_t i = 0; i < n; ++i) std::fprintf(f, "  0");
    std::fprintf(f, "\n        </DataArray>\n      </PointData>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n");
    std::fclose(f);
    return PFEM2GPU_OK;
}

int pfem2gpu_window_forward_device(pfem2gpu_handle* h, int32_t steps, int32_t checkpoint_every, const double* dV,
                                   const double* dVold, const double* dv0, double* dU_out)
{
    return window_forward_impl(h, steps, checkpoint_every, dV, dVold, dv0, dU_out, false);
}

int pfem2gpu_window_backward_device(pfem2gpu_handle* h, const double* dgU, double* dg_v0, double* dg_V,
                                    double* dg_Vold)
{
    return window_backward_impl(h, dgU, dg_v0, dg_V, dg_Vold, false);
}

int pfem2gpu_adjoint(pfem2gpu_handle* h, int32_t steps, int32_t checkpoint_every, const double* V, const double* Vold,
                     const double* v0, const double* gU, double* U, double* g_v0, double* g_V, double* g_Vold)
{
    int rc = window_forward_impl(h, steps, checkpoint_every, V, Vold, v0, U, true);
    if (rc) return rc;
    return window_backward_impl(h, gU, g_v0, g_V, g_Vold, true);
}

// The CSR pattern of the FEM matrices: per DoF row the DoFs sharing a cell
// with it (from the DoF -> cell map), ascending.
static int fem_pattern_build(pfem2gpu_handle* h)
{
    auto& F = h->fem;
    const size_t NV = (size_t)1 << h->dim;
    if ((size_t)h->nC * NV * NV > (size_t)INT32_MAX) return fail(h, PFEM2GPU_ERR_ARG, "mesh too large for the FEM lists");
    const size_t nd = h->nD, ntiles = (nd + WIN_TILE - 1) / WIN_TILE + 1;
    Scratch sc;
    uint32_t *cnt = nullptr, *tsum = nullptr;
    unsigned* err = nullptr;
    CK(dalloc(&F.row_ptr, nd + 1));
    CK(sc.get(&cnt, nd));
    CK(sc.get(&tsum, ntiles));
    CK(sc.get(&err, 1));
    CK(cudaMemsetAsync(err, 0, sizeof(unsigned), h->stream));
    FemArgs f{};
    f.nC = h->nC;
    f.nD = h->nD;
    f.cd = h->cd;
    f.d2c_off = h->d2c_off;
    f.d2c_ent = h->d2c_ent;
    f.row_ptr = F.row_ptr;
    run(h, "fem_pattern", [&] {
        int n = launch_fem_pattern(h->dim, f, false, cnt, err, h->stream);
        return n + launch_win_scan(cnt, (uint32_t)nd, tsum, (uint32_t*)F.row_ptr, h->stream);
    });
    int32_t nnz = 0;
    unsigned e = 0;
    CK(cudaMemcpyAsync(&nnz, F.row_ptr + nd, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (e) return fail(h, PFEM2GPU_ERR_ARG, "a DoF couples to more than 64 DoFs");
    CK(dalloc(&F.cols, std::max<size_t>(nnz, 1)));
    f.cols = F.cols;
    run(h, "fem_pattern", [&] { return launch_fem_pattern(h->dim, f, true, cnt, err, h->stream); });
    // contribution lists of the entries (count, scan, fill)
    const size_t nz = (size_t)nnz, ztiles = (nz + WIN_TILE - 1) / WIN_TILE + 1;
    uint32_t *zcnt = nullptr, *ztsum = nullptr;
    CK(sc.get(&zcnt, std::max<size_t>(nz, 1)));
    CK(sc.get(&ztsum, ztiles));
    CK(dalloc(&F.con_off, nz + 1));
    f.con_off = F.con_off;
    run(h, "fem_pattern", [&] {
        int n = launch_fem_contrib(h->dim, f, false, zcnt, h->stream);
        return n + launch_win_scan(zcnt, (uint32_t)nz, ztsum, (uint32_t*)F.con_off, h->stream);
    });
    int32_t ncon = 0;
    CK(cudaMemcpyAsync(&ncon, F.con_off + nz, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    CK(dalloc(&F.con, std::max<size_t>(ncon, 1)));
    f.con = F.con;
    run(h, "fem_pattern", [&] { return launch_fem_contrib(h->dim, f, true, zcnt, h->stream); });
    CK(cudaStreamSynchronize(h->stream));
    int rc = check_async(h);
    if (rc == PFEM2GPU_OK) F.nnz = nnz;
    return rc;
}

// The CSR pattern of the FEM matrices and the entries' contribution lists,
// built on the device once per mesh (a failure leaves nothing half built).
static int fem_pattern(pfem2gpu_handle* h)
{
    if (h->fem.nnz >= 0) return PFEM2GPU_OK;
    auto& F = h->fem;  // the boundary ids survive a failed build
    uint16_t* keep = F.fmask;
    uint8_t* keep_d = F.dmask;
    int32_t* keep_f = F.face_id;
    F.fmask = nullptr;
    F.dmask = nullptr;
    F.face_id = nullptr;
    const int rc = fem_pattern_build(h);
    if (rc != PFEM2GPU_OK) free_fem(F);
    F.fmask = keep;
    F.dmask = keep_d;
    F.face_id = keep_f;
    return rc;
}

int pfem2gpu_fem_pattern(pfem2gpu_handle* h, int32_t* row_ptr, int32_t* cols, int64_t capacity, int64_t* nnz)
{
    if (!h || !nnz) return PFEM2GPU_ERR_ARG;
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "no mesh");
    int rc = fem_pattern(h);
    if (rc) return rc;
    *nnz = h->fem.nnz;
    if (row_ptr) CK(cudaMemcpyAsync(row_ptr, h->fem.row_ptr, ((size_t)h->nD + 1) * 4, cudaMemcpyDeviceToHost, h->stream));
    if (cols) {
        if (capacity < h->fem.nnz) return fail(h, PFEM2GPU_ERR_ARG, "output arrays too small");
        CK(cudaMemcpyAsync(cols, h->fem.cols, (size_t)h->fem.nnz * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return PFEM2GPU_OK;
}

static int fem_sizes(int dim, int system, int* nm, int* ns)
{
    if (system < PFEM2GPU_FEM_PREDICTION || system > PFEM2GPU_FEM_CORRECTION) return 1;
    *nm = system == PFEM2GPU_FEM_PREDICTION ? dim : 1;
    *ns = system == PFEM2GPU_FEM_PRESSURE ? 1 : dim;
    return 0;
}

static int fem_run(pfem2gpu_handle* h, int system, double rho, double mu, double dt, const double* dU,
                   const double* dU2, const double* dP, double* dA, double* drhs)
{
    int nm, ns;
    fem_sizes(h->dim, system, &nm, &ns);
    auto& F = h->fem;
    const int NV = 1 << h->dim;
    const size_t nloc = (size_t)h->nC * NV * nm * NV, nr = (size_t)h->nC * NV * ns;
    if (nloc > F.local_n) {
        dfree(F.local);
        F.local = nullptr;
        F.local_n = 0;
        CK(dalloc(&F.local, nloc));
        F.local_n = nloc;
    }
    if (nr > F.rhs_n) {
        dfree(F.local_rhs);
        F.local_rhs = nullptr;
        F.rhs_n = 0;
        CK(dalloc(&F.local_rhs, nr));
        F.rhs_n = nr;
    }
    FemArgs f{};
    f.nC = h->nC;
    f.nD = h->nD;
    f.nnz = F.nnz;
    f.cellX = h->cellX;
    f.cd = h->cd;
    f.d2c_off = h->d2c_off;
    f.d2c_ent = h->d2c_ent;
    f.row_ptr = F.row_ptr;
    f.cols = F.cols;
    f.con_off = F.con_off;
    f.con = F.con;
    f.rho = rho;
    f.mu = mu;
    f.dt = dt;
    f.U = dU;
    f.U2 = dU2;
    f.P = dP;
    f.local = F.local;
    f.local_rhs = F.local_rhs;
    f.A = dA;
    f.rhs = drhs;
    f.fmask = F.fmask;
    run(h, "fem_assemble", [&] { return launch_fem_assemble(h->dim, system, f, h->stream); });
    return check_async(h);
}

static int fem_check(pfem2gpu_handle* h, int system, const double* U, const double* U2, const double* P,
                     const double* A, const double* rhs)
{
    int nm, ns;
    if (!h) return PFEM2GPU_ERR_ARG;
    if (fem_sizes(h->dim, system, &nm, &ns)) return fail(h, PFEM2GPU_ERR_ARG, "unknown FEM system");
    if (!A || !rhs || !U) return fail(h, PFEM2GPU_ERR_ARG, "missing vector");
    if (system == PFEM2GPU_FEM_PREDICTION && !U2) return fail(h, PFEM2GPU_ERR_ARG, "missing old velocity");
    if (system == PFEM2GPU_FEM_CORRECTION && !P) return fail(h, PFEM2GPU_ERR_ARG, "missing pressure");
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "no mesh");
    return fem_pattern(h);
}

int pfem2gpu_fem_set_boundary(pfem2gpu_handle* h, const int32_t* face_ids, int32_t n_velocity_dirichlet,
                              const int32_t* velocity_dirichlet, int32_t n_pressure_dirichlet,
                              const int32_t* pressure_dirichlet)
{
    if (!h) return PFEM2GPU_ERR_ARG;
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "no mesh");
    auto& F = h->fem;
    dfree(F.fmask);
    dfree(F.dmask);
    dfree(F.face_id);
    F.fmask = nullptr;
    F.dmask = nullptr;
    F.face_id = nullptr;
    if (!face_ids) return PFEM2GPU_OK;
    if ((n_velocity_dirichlet > 0 && !velocity_dirichlet) || (n_pressure_dirichlet > 0 && !pressure_dirichlet) ||
        n_velocity_dirichlet < 0 || n_pressure_dirichlet < 0)
        return fail(h, PFEM2GPU_ERR_ARG, "bad Dirichlet id list");
    const int nf = 2 * h->dim;
    std::vector<uint16_t> mask(h->nC, 0);
    std::vector<uint8_t> dmask(h->nC, 0);
    auto in = [](int32_t id, int32_t n, const int32_t* ids) {
        for (int32_t k = 0; k < n; ++k)
            if (ids[k] == id) return true;
        return false;
    };
    for (int c = 0; c < h->nC; ++c)
        for (int f = 0; f < nf; ++f) {
            const int32_t id = face_ids[(size_t)c * nf + f];
            if (id < 0) continue;  // interior face
            if (!in(id, n_velocity_dirichlet, velocity_dirichlet)) mask[c] |= (uint16_t)(1u << f);
            else dmask[c] |= (uint8_t)(1u << f);
            if (!in(id, n_pressure_dirichlet, pressure_dirichlet)) mask[c] |= (uint16_t)(1u << (8 + f));
        }
    CK(dalloc(&F.fmask, (size_t)h->nC));
    CK(dalloc(&F.dmask, (size_t)h->nC));
    CK(dalloc(&F.face_id, (size_t)h->nC * nf));
    CK(cudaMemcpyAsync(F.fmask, mask.data(), (size_t)h->nC * sizeof(uint16_t), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(F.dmask, dmask.data(), (size_t)h->nC, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(F.face_id, face_ids, (size_t)h->nC * nf * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PFEM2GPU_OK;
}

int pfem2gpu_fem_velocity_bc(pfem2gpu_handle* h, double rho, double dt, const double* P, int32_t n_ids,
                             const int32_t* ids, const double* velocities, int32_t* rows, double* values,
                             int64_t capacity, int64_t* n)
{
    if (!h || !n || !P || n_ids < 0 || (n_ids > 0 && (!ids || !velocities))) return PFEM2GPU_ERR_ARG;
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "no mesh");
    auto& F = h->fem;
    if (!F.dmask) return fail(h, PFEM2GPU_ERR_STATE, "no boundary ids (pfem2gpu_fem_set_boundary)");
    int rc = fem_pattern(h);
    if (rc) return rc;
    const int dim = h->dim, NV = 1 << dim;
    const size_t nd = h->nD, nloc = (size_t)h->nC * NV;
    // buffers kept with the mesh (the call comes once per time step)
    if (!F.bc_P || !F.bc_loc || !F.bc_lid || !F.bc_val || !F.bc_flag) {
        for (void** q : {(void**)&F.bc_P, (void**)&F.bc_loc, (void**)&F.bc_lid, (void**)&F.bc_val, (void**)&F.bc_flag}) {
            dfree(*q);
            *q = nullptr;
        }
        CK(dalloc(&F.bc_P, nd));
        CK(dalloc(&F.bc_loc, nloc * (dim + 1)));
        CK(dalloc(&F.bc_lid, nloc));
        CK(dalloc(&F.bc_val, nd * dim));
        CK(dalloc(&F.bc_flag, nd));
    }
    if (n_ids > F.bc_ncap || !F.bc_ids) {
        dfree(F.bc_ids);
        dfree(F.bc_vel);
        F.bc_ids = nullptr;
        F.bc_vel = nullptr;
        F.bc_ncap = 0;
        const int32_t cap = std::max<int32_t>(n_ids, 16);
        CK(dalloc(&F.bc_ids, (size_t)cap));
        CK(dalloc(&F.bc_vel, (size_t)cap * dim));
        F.bc_ncap = cap;
    }
    double *dP = F.bc_P, *loc = F.bc_loc, *vel = F.bc_vel, *val = F.bc_val;
    int32_t *lid = F.bc_lid, *dids = F.bc_ids, *flag = F.bc_flag;
    CK(cudaMemcpyAsync(dP, P, nd * 8, cudaMemcpyHostToDevice, h->stream));
    if (n_ids > 0) {
        CK(cudaMemcpyAsync(dids, ids, (size_t)n_ids * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(vel, velocities, (size_t)n_ids * dim * 8, cudaMemcpyHostToDevice, h->stream));
    }
    FemArgs f{};
    f.nC = h->nC;
    f.nD = h->nD;
    f.cellX = h->cellX;
    f.cd = h->cd;
    f.d2c_off = h->d2c_off;
    f.d2c_ent = h->d2c_ent;
    run(h, "fem_velocity_bc", [&] {
        return launch_fem_velocity_bc(dim, f, F.dmask, F.face_id, dP, loc, lid, n_ids, dids, vel, dt / rho, val, flag,
                                      h->stream);
    });
    std::vector<int32_t> hf(nd);
    std::vector<double> hv(nd * dim);
    CK(cudaMemcpyAsync(hf.data(), flag, nd * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(hv.data(), val, nd * dim * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if ((rc = check_async(h))) return rc;
    int64_t m = 0;
    for (size_t r = 0; r < nd; ++r) m += hf[r] ? 1 : 0;
    *n = m;
    if (!rows && !values) return PFEM2GPU_OK;
    if (capacity < m || !rows || !values) return fail(h, PFEM2GPU_ERR_ARG, "output arrays too small");
    int64_t k = 0;
    for (size_t r = 0; r < nd; ++r)
        if (hf[r]) {
            rows[k] = (int32_t)r;
            for (int d = 0; d < dim; ++d) values[(size_t)d * m + k] = hv[(size_t)d * nd + r];
            ++k;
        }
    return PFEM2GPU_OK;
}

static int fem_constrain(pfem2gpu_handle* h, int system, int32_t n, const int32_t* rows, const double* values,
                         double* dA, double* drhs)
{
    int nm, ns;
    if (!h) return PFEM2GPU_ERR_ARG;
    if (fem_sizes(h->dim, system, &nm, &ns)) return fail(h, PFEM2GPU_ERR_ARG, "unknown FEM system");
    if (n < 0 || (n > 0 && (!rows || !values)) || !dA || !drhs) return fail(h, PFEM2GPU_ERR_ARG, "bad constraint arrays");
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "no mesh");
    int rc = fem_pattern(h);
    if (rc) return rc;
    auto& F = h->fem;
    std::vector<int32_t> idx(h->nD, -1);
    for (int32_t k = 0; k < n; ++k) {
        if (rows[k] < 0 || rows[k] >= h->nD) return fail(h, PFEM2GPU_ERR_ARG, "constrained row out of range");
        if (idx[rows[k]] >= 0) return fail(h, PFEM2GPU_ERR_ARG, "constrained row listed twice");
        idx[rows[k]] = k;
    }
    if (!F.con_idx) CK(dalloc(&F.con_idx, (size_t)h->nD));
    const size_t nv = std::max<size_t>((size_t)ns * n, 1);
    if (nv > F.con_val_n) {
        dfree(F.con_val);
        F.con_val = nullptr;
        F.con_val_n = 0;
        CK(dalloc(&F.con_val, nv));
        F.con_val_n = nv;
    }
    CK(cudaMemcpyAsync(F.con_idx, idx.data(), (size_t)h->nD * 4, cudaMemcpyHostToDevice, h->stream));
    if (n > 0) CK(cudaMemcpyAsync(F.con_val, values, (size_t)ns * n * 8, cudaMemcpyHostToDevice, h->stream));
    run(h, "fem_constrain", [&] {
        return launch_fem_constrain(h->nD, F.nnz, nm, ns, F.row_ptr, F.cols, F.con_idx, n, F.con_val, dA, drhs,
                                    h->stream);
    });
    // the host arrays above must outlive the copies
    CK(cudaStreamSynchronize(h->stream));
    return check_async(h);
}

int pfem2gpu_fem_constrain_device(pfem2gpu_handle* h, int system, int32_t n, const int32_t* rows,
                                  const double* values, double* dA, double* drhs)
{
    return fem_constrain(h, system, n, rows, values, dA, drhs);
}

int pfem2gpu_fem_constrain(pfem2gpu_handle* h, int system, int32_t n, const int32_t* rows, const double* values,
                           double* A, double* rhs)
{
    int nm, ns;
    if (!h) return PFEM2GPU_ERR_ARG;
    if (fem_sizes(h->dim, system, &nm, &ns)) return fail(h, PFEM2GPU_ERR_ARG, "unknown FEM system");
    if (!A || !rhs) return fail(h, PFEM2GPU_ERR_ARG, "missing matrix or right-hand side");
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "no mesh");
    int rc = fem_pattern(h);
    if (rc) return rc;
    auto& F = h->fem;
    const size_t na = (size_t)nm * F.nnz, nr = (size_t)ns * h->nD;
    if (na + nr > F.io_n) {
        dfree(F.io);
        F.io = nullptr;
        F.io_n = 0;
        CK(dalloc(&F.io, na + nr));
        F.io_n = na + nr;
    }
    double* dA = F.io;
    double* dr = F.io + na;
    CK(cudaMemcpyAsync(dA, A, na * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(dr, rhs, nr * 8, cudaMemcpyHostToDevice, h->stream));
    if ((rc = fem_constrain(h, system, n, rows, values, dA, dr))) return rc;
    CK(cudaMemcpyAsync(A, dA, na * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(rhs, dr, nr * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PFEM2GPU_OK;
}

int pfem2gpu_fem_assemble_device(pfem2gpu_handle* h, int system, double rho, double mu, double dt, const double* dU,
                                 const double* dU2, const double* dP, double* dA, double* drhs)
{
    const int rc = fem_check(h, system, dU, dU2, dP, dA, drhs);
    if (rc) return rc;
    return fem_run(h, system, rho, mu, dt, dU, dU2, dP, dA, drhs);
}

int pfem2gpu_fem_assemble(pfem2gpu_handle* h, int system, double rho, double mu, double dt, const double* U,
                          const double* U2, const double* P, double* A, double* rhs)
{
    int rc = fem_check(h, system, U, U2, P, A, rhs);
    if (rc) return rc;
    int nm, ns;
    fem_sizes(h->dim, system, &nm, &ns);
    auto& F = h->fem;
    const size_t vd = (size_t)h->dim * h->nD, need = 2 * vd + h->nD + (size_t)nm * F.nnz + (size_t)ns * h->nD;
    if (need > F.io_n) {
        dfree(F.io);
        F.io = nullptr;
        F.io_n = 0;
        CK(dalloc(&F.io, need));
        F.io_n = need;
    }
    double* dU = F.io;
    double* dU2 = dU + vd;
    double* dP = dU2 + vd;
    double* dA = dP + h->nD;
    double* drhs = dA + (size_t)nm * F.nnz;
    CK(cudaMemcpyAsync(dU, U, vd * 8, cudaMemcpyHostToDevice, h->stream));
    if (U2) CK(cudaMemcpyAsync(dU2, U2, vd * 8, cudaMemcpyHostToDevice, h->stream));
    if (P) CK(cudaMemcpyAsync(dP, P, (size_t)h->nD * 8, cudaMemcpyHostToDevice, h->stream));
    if ((rc = fem_run(h, system, rho, mu, dt, dU, U2 ? dU2 : nullptr, P ? dP : nullptr, dA, drhs))) return rc;
    CK(cudaMemcpyAsync(A, dA, (size_t)nm * F.nnz * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(rhs, drhs, (size_t)ns * h->nD * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PFEM2GPU_OK;
}

int pfem2gpu_get_vertex_maps(pfem2gpu_handle* h, int32_t* offsets, int32_t* cells, double* dirs, int64_t capacity,
                             int64_t* n)
{
    if (!h || !n) return PFEM2GPU_ERR_ARG;
    if (!h->has_mesh) return fail(h, PFEM2GPU_ERR_STATE, "no mesh");
    int32_t total = 0;
    CK(cudaMemcpyAsync(&total, h->v2c_off + h->nV, 4, cudaMemcpyDeviceToHost, h->stream));
    if (offsets) CK(cudaMemcpyAsync(offsets, h->v2c_off, ((size_t)h->nV + 1) * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *n = total;
    if ((cells || dirs) && capacity < total) return fail(h, PFEM2GPU_ERR_ARG, "output arrays too small");
    if (cells) CK(cudaMemcpyAsync(cells, h->v2c_cells, (size_t)total * 4, cudaMemcpyDeviceToHost, h->stream));
    if (dirs) CK(cudaMemcpyAsync(dirs, h->v2c_dirs, (size_t)total * h->dim * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PFEM2GPU_OK;
}

int pfem2gpu_window_particles(pfem2gpu_handle* h, int32_t* cell, double* xi, double* v, int64_t capacity, int64_t* n)
{
    if (!h || !n) return PFEM2GPU_ERR_ARG;
    auto& W = h->win;
    if (!W.ready) return fail(h, PFEM2GPU_ERR_STATE, "no window forward");
    *n = W.n;
    if (capacity < (int64_t)W.n) return fail(h, PFEM2GPU_ERR_ARG, "output arrays too small");
    const int dim = h->dim;
    const size_t n0 = W.n, es = esize(h);
    std::vector<uint32_t> c(n0);
    std::vector<unsigned char> buf(n0 * es);
    CK(cudaMemcpyAsync(c.data(), W.fin_cell, n0 * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (cell)
        for (size_t p = 0; p < n0; ++p) cell[p] = c[p] == LOST ? -1 : (int32_t)c[p];
    for (int which = 0; which < 2; ++which) {
        double* out = which ? v : xi;
        if (!out) continue;
        for (int d = 0; d < dim; ++d) {
            const size_t ew = which ? 8 : es;  // velocities are FP64 in both forms
            const char* src = which ? (const char*)(W.fin_v + (size_t)d * W.ncap)
                                    : (const char*)W.fin_xi + (size_t)d * W.ncap * es;
            buf.resize(n0 * ew);
            CK(cudaMemcpyAsync(buf.data(), src, n0 * ew, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            for (size_t p = 0; p < n0; ++p)
                out[p * dim + d] = ew == 8 ? reinterpret_cast<const double*>(buf.data())[p]
                                           : (double)reinterpret_cast<const float*>(buf.data())[p];
        }
    }
    return PFEM2GPU_OK;
}

int pfem2gpu_window_size(pfem2gpu_handle* h, int64_t* n)
{
    if (!h || !n) return PFEM2GPU_ERR_ARG;
    *n = h->win.ready ? (int64_t)h->win.n : -1;
    return PFEM2GPU_OK;
}

}  // extern "C"
