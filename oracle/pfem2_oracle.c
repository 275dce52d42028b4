/*
 * pfem2_oracle.c -- FP64 CPU restatement of the PFEM-2 particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY (checker + timed CPU baseline); see the header.
 * PARITY UNPINNED against the real reference: it cannot be built here and it
 * ships no tests or golden vectors.
 *
 * Compile with -ffp-contract=off (oracle/Makefile does): every product and sum
 * below is rounded separately, in the written order, exactly as a non-FMA
 * build of the reference evaluates it.  The CUDA FP64 form is compiled with
 * --fmad=false and evaluates the same expressions in the same order, so its
 * cell ids, reference coordinates, positions and velocities match this file
 * bit for bit.
 *
 * Reference paths cited are relative to the pfem2dealii project root.
 */
#include "pfem2_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define MAXV 8 /* vertices per cell, dim <= 3 */

typedef struct orc_particle {
    double x[3];    /* location                 (src/pfem2particle.h:63) */
    double xi[3];   /* reference_location       (src/pfem2particle.h:64) */
    double v[3];    /* velocity                 (src/pfem2particle.h:71) */
    double vext[3]; /* velocity_ext             (src/pfem2particle.h:72) */
    int32_t cell;   /* tria_position            (src/pfem2particle.h:69) */
    uint32_t id;    /* id                       (src/pfem2particle.h:65) */
} orc_particle;

struct orc_handle {
    int dim, nv;
    orc_params prm;
    int S;
    double dtp;
    double h[3];
    int npart;      /* real cell parts: q0*q1*q2 */
    int npart_ext;  /* (q0+1)*(q1+1)*(q2+1): (int)(xi/h) can reach q on the upper face */
    int64_t nC, nV, nD;
    double* X;
    int32_t* cv;
    int32_t* cd;
    int32_t* v2c_off;
    int32_t* v2c_cells;
    double* v2c_dirs;
    orc_particle* P;
    int64_t n, cap;
    orc_stats st;
};

/* ------------------------------------------------------------------------ */
/* Q1 shape functions and the multilinear map (deal.II FE_Q<dim>(1) and      */
/* MappingQ1; call sites src/pfem2particlehandler.cpp:97,131,155,193,400 and  */
/* :91,394,425,463, src/pfem2particle.cpp:190).                              */
/* Vertex i has bits b_d = (i >> d) & 1 (deal.II lexicographic order) and    */
/* N_i(xi) = prod_d (b_d ? xi_d : 1 - xi_d), multiplied in d order.          */
/* ------------------------------------------------------------------------ */

static inline double lag(int b, double t) { return b ? t : 1.0 - t; }

void orc_shape_values(int dim, const double* xi, double* N)
{
    const int nv = 1 << dim;
    for (int i = 0; i < nv; ++i) {
        double n = lag(i & 1, xi[0]);
        if (dim > 1) n = n * lag((i >> 1) & 1, xi[1]);
        if (dim > 2) n = n * lag((i >> 2) & 1, xi[2]);
        N[i] = n;
    }
}

/* dN_i/dxi_k = (b_k ? 1 : -1) * prod_{m != k} L_m, product in m order. */
static void shape_grads(int dim, const double* xi, double G[MAXV][3])
{
    const int nv = 1 << dim;
    for (int i = 0; i < nv; ++i)
        for (int k = 0; k < dim; ++k) {
            double g = ((i >> k) & 1) ? 1.0 : -1.0;
            for (int m = 0; m < dim; ++m)
                if (m != k) g = g * lag((i >> m) & 1, xi[m]);
            G[i][k] = g;
        }
}

/* x = sum_i N_i(xi) X_i, X row-major (vertex, component). */
void orc_forward_map(int dim, const double* X, const double* xi, double* x)
{
    const int nv = 1 << dim;
    double N[MAXV];
    orc_shape_values(dim, xi, N);
    for (int d = 0; d < dim; ++d) {
        double acc = 0.0;
        for (int i = 0; i < nv; ++i) acc = acc + N[i] * X[i * 3 + d];
        x[d] = acc;
    }
}

static void jacobian(int dim, const double* X, const double* xi, double J[3][3])
{
    const int nv = 1 << dim;
    double G[MAXV][3];
    shape_grads(dim, xi, G);
    for (int d = 0; d < dim; ++d)
        for (int k = 0; k < dim; ++k) {
            double acc = 0.0;
            for (int i = 0; i < nv; ++i) acc = acc + G[i][k] * X[i * 3 + d];
            J[d][k] = acc;
        }
}

/* Inverse of a 2x2 / 3x3 matrix: adjugate times the reciprocal of the
 * determinant; returns the determinant. */
static double invert(int dim, const double A[3][3], double Ai[3][3])
{
    if (dim == 2) {
        const double det = A[0][0] * A[1][1] - A[0][1] * A[1][0];
        const double r = 1.0 / det;
        Ai[0][0] = A[1][1] * r;
        Ai[0][1] = -A[0][1] * r;
        Ai[1][0] = -A[1][0] * r;
        Ai[1][1] = A[0][0] * r;
        return det;
    }
    const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    const double c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    const double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    const double det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
    const double r = 1.0 / det;
    Ai[0][0] = c00 * r;
    Ai[1][0] = c01 * r;
    Ai[2][0] = c02 * r;
    Ai[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * r;
    Ai[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * r;
    Ai[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * r;
    Ai[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * r;
    Ai[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * r;
    Ai[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * r;
    return det;
}

static inline void matvec(int dim, const double A[3][3], const double* x, double* y)
{
    for (int k = 0; k < dim; ++k) {
        double acc = 0.0;
        for (int d = 0; d < dim; ++d) acc = acc + A[k][d] * x[d];
        y[k] = acc;
    }
}

static inline double norm2(int dim, const double* a)
{
    double s = 0.0;
    for (int d = 0; d < dim; ++d) s = s + a[d] * a[d];
    return s;
}

/* GeometryInfo<dim>::is_inside_unit_cell(p) (no-epsilon overload), the test at
 * src/pfem2particlehandler.cpp:427,464.  NaN compares false -> outside. */
static inline int inside_unit(int dim, const double* xi)
{
    for (int d = 0; d < dim; ++d)
        if (!(xi[d] >= 0.0 && xi[d] <= 1.0)) return 0;
    return 1;
}

static inline int inside_unit_eps(int dim, const double* xi, double eps)
{
    for (int d = 0; d < dim; ++d)
        if (!(xi[d] >= -eps && xi[d] <= 1.0 + eps)) return 0;
    return 1;
}

/* 2D closed form of the bilinear inverse.  With e = X1-X0, f = X2-X0,
 * g = X3-X1-X2+X0, r = p-X0 the map is r = xi e + eta f + xi eta g.  Crossing
 * r - eta f with e + eta g eliminates xi and leaves
 *   cross(f,g) eta^2 + (cross(f,e) - cross(r,g)) eta - cross(r,e) = 0,
 * solved with the cancellation-free quadratic formula; the root closest to
 * 1/2 is kept and xi follows by projecting r - eta f on e + eta g.
 * Returns 0 on success. */
static int bilinear_exact(const double* X, const double* p, double* xi)
{
    const double ex = X[3] - X[0], ey = X[4] - X[1];
    const double fx = X[6] - X[0], fy = X[7] - X[1];
    const double gx = ((X[9] - X[3]) - X[6]) + X[0];
    const double gy = ((X[10] - X[4]) - X[7]) + X[1];
    const double rx = p[0] - X[0], ry = p[1] - X[1];
    const double qa = fx * gy - fy * gx;
    const double qb = (fx * ey - fy * ex) - (rx * gy - ry * gx);
    const double qc = -(rx * ey - ry * ex);
    double eta;
    if (qa == 0.0) {
        if (qb == 0.0) return 1;
        eta = -qc / qb;
    } else {
        const double disc = qb * qb - 4.0 * qa * qc;
        if (!(disc >= 0.0)) return 1;
        const double sq = sqrt(disc);
        const double q = -0.5 * (qb + (qb >= 0.0 ? sq : -sq));
        if (q == 0.0) {
            eta = 0.0;
        } else {
            const double e1 = q / qa;
            const double e2 = qc / q;
            eta = (fabs(e1 - 0.5) < fabs(e2 - 0.5)) ? e1 : e2;
        }
    }
    const double wx = ex + eta * gx, wy = ey + eta * gy;
    const double tx = rx - eta * fx, ty = ry - eta * fy;
    const double ww = wx * wx + wy * wy;
    if (!(ww > 0.0)) return 1;
    xi[0] = (tx * wx + ty * wy) / ww;
    xi[1] = eta;
    return 0;
}

/* Least-squares affine approximation of the multilinear map: column k of A is
 * the mean edge vector in direction k, b = centroid - A (1/2,...). */
static int affine_guess(int dim, const double* X, const double* p, double* xi)
{
    const int nv = 1 << dim;
    const double half = (double)(nv / 2);
    double A[3][3], Ai[3][3], b[3], r[3];
    for (int d = 0; d < dim; ++d) {
        double mean = 0.0;
        for (int i = 0; i < nv; ++i) mean = mean + X[i * 3 + d];
        mean = mean / (double)nv;
        for (int k = 0; k < dim; ++k) {
            double sp = 0.0, sm = 0.0;
            for (int i = 0; i < nv; ++i) {
                if ((i >> k) & 1) sp = sp + X[i * 3 + d];
                else sm = sm + X[i * 3 + d];
            }
            A[d][k] = (sp - sm) / half;
        }
        double ac = 0.0;
        for (int k = 0; k < dim; ++k) ac = ac + A[d][k] * 0.5;
        b[d] = mean - ac;
    }
    const double det = invert(dim, A, Ai);
    if (!(det != 0.0) || !isfinite(det)) return 1;
    for (int d = 0; d < dim; ++d) r[d] = p[d] - b[d];
    matvec(dim, Ai, r, xi);
    return 0;
}

static inline void clamp_unit(int dim, double* xi)
{
    for (int d = 0; d < dim; ++d) {
        if (xi[d] < 0.0) xi[d] = 0.0;
        else if (xi[d] > 1.0) xi[d] = 1.0;
    }
}

/* MappingQ1::transform_real_to_unit_cell, restated (call sites
 * src/pfem2particlehandler.cpp:425,463).  deal.II's published strategy: in 2D
 * the closed-form inverse is accepted if it lies in the unit cell within
 * 1e-12; otherwise (and always in 3D) Newton's method starts from the affine
 * approximation projected onto the unit cell, measures the residual in
 * reference units (|J^{-1} f|), converges below 1e-11, halves the step while
 * the weighted residual does not decrease (down to 0.05), restarts once from
 * the projected iterate before giving up, fails on a non-positive Jacobian
 * determinant and after 20 iterations.  Failure corresponds to
 * ExcTransformationFailed, which the reference catches.
 * deal.II evaluates the 2D formula in long double; this restatement (and the
 * GPU) uses double.  Returns 0 on success. */
int orc_inverse_map(int dim, const double* X, const double* p, double* xi_out)
{
    double xi[3] = {0.0, 0.0, 0.0}, f[3], J[3][3], Ji[3][3], delta[3], trial[3], ft[3], dt[3], x[3];
    if (dim == 2) {
        double e[2];
        if (bilinear_exact(X, p, e) == 0 && inside_unit_eps(2, e, 1e-12)) {
            xi_out[0] = e[0];
            xi_out[1] = e[1];
            return 0;
        }
    }
    if (affine_guess(dim, X, p, xi)) return 1;
    clamp_unit(dim, xi);
    orc_forward_map(dim, X, xi, x);
    for (int d = 0; d < dim; ++d) f[d] = x[d] - p[d];
    int restarted = 0;
    for (int it = 0; it < 20; ++it) {
        jacobian(dim, X, xi, J);
        const double det = invert(dim, J, Ji);
        if (!(det > 0.0)) return 1;
        matvec(dim, Ji, f, delta);
        const double dn = norm2(dim, delta);
        if (dn <= 1e-22) {
            for (int d = 0; d < dim; ++d) xi_out[d] = xi[d];
            return 0;
        }
        double step = 1.0, tn = 0.0;
        int accepted = 0;
        for (;;) {
            for (int d = 0; d < dim; ++d) trial[d] = xi[d] - step * delta[d];
            orc_forward_map(dim, X, trial, x);
            for (int d = 0; d < dim; ++d) ft[d] = x[d] - p[d];
            matvec(dim, Ji, ft, dt);
            tn = norm2(dim, dt);
            if (tn < dn) {
                accepted = 1;
                break;
            }
            if (step > 0.05) step = step * 0.5;
            else break;
        }
        if (!accepted) {
            if (restarted) return 1;
            restarted = 1;
            clamp_unit(dim, xi);
            orc_forward_map(dim, X, xi, x);
            for (int d = 0; d < dim; ++d) f[d] = x[d] - p[d];
            continue;
        }
        for (int d = 0; d < dim; ++d) {
            xi[d] = trial[d];
            f[d] = ft[d];
        }
        if (tn <= 1e-22) {
            for (int d = 0; d < dim; ++d) xi_out[d] = xi[d];
            return 0;
        }
    }
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Handle, mesh and vertex maps                                              */
/* ------------------------------------------------------------------------ */

uint32_t orc_key(uint32_t id, uint32_t seed)
{
    if (!seed) return id;
    uint32_t x = id ^ seed; /* bijective 32-bit mixer (lowbias32, C. Wellons) */
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

orc_handle* orc_create(int dim, const orc_params* prm)
{
    if (dim != 2 && dim != 3) return NULL;
    orc_handle* h = (orc_handle*)calloc(1, sizeof(orc_handle));
    if (!h) return NULL;
    h->dim = dim;
    h->nv = 1 << dim;
    h->prm = *prm;
    /* setPfem2Solver, src/pfem2particlehandler.cpp:34-39 */
    h->S = prm->substeps == 0 ? 1 : prm->substeps;
    h->dtp = prm->dt / (double)h->S;
    h->npart = 1;
    h->npart_ext = 1;
    for (int d = 0; d < dim; ++d) {
        if (prm->q[d] < 1) {
            free(h);
            return NULL;
        }
        h->h[d] = 1.0 / prm->q[d]; /* src/pfem2particlehandler.cpp:80-82,362-364 */
        h->npart *= prm->q[d];
        h->npart_ext *= prm->q[d] + 1;
    }
    if (h->prm.n_threads < 1) h->prm.n_threads = 1;
    return h;
}

void orc_destroy(orc_handle* h)
{
    if (!h) return;
    free(h->X);
    free(h->cv);
    free(h->cd);
    free(h->v2c_off);
    free(h->v2c_cells);
    free(h->v2c_dirs);
    free(h->P);
    free(h);
}

static void cell_coords(const orc_handle* h, int64_t c, double* Xc)
{
    for (int i = 0; i < h->nv; ++i) {
        const int32_t vi = h->cv[c * h->nv + i];
        for (int d = 0; d < 3; ++d) Xc[i * 3 + d] = d < h->dim ? h->X[(int64_t)vi * h->dim + d] : 0.0;
    }
}

/* initialize_maps, src/pfem2particlehandler.cpp:320-324: GridTools::
 * vertex_to_cell_map (a std::set per vertex, i.e. cells in ascending index on
 * a single-level mesh) and vertex_to_cell_centers_directions (unit vector from
 * the vertex to the vertex-average centre of each of those cells). */
int orc_set_mesh(orc_handle* h, int64_t n_cells, int64_t n_verts, int64_t n_dofs,
                 const double* vertices, const int32_t* cell_vertices, const int32_t* cell_dofs)
{
    const int dim = h->dim, nv = h->nv;
    free(h->X);
    free(h->cv);
    free(h->cd);
    free(h->v2c_off);
    free(h->v2c_cells);
    free(h->v2c_dirs);
    h->nC = n_cells;
    h->nV = n_verts;
    h->nD = n_dofs;
    h->X = (double*)malloc(sizeof(double) * n_verts * dim);
    h->cv = (int32_t*)malloc(sizeof(int32_t) * n_cells * nv);
    h->cd = (int32_t*)malloc(sizeof(int32_t) * n_cells * nv);
    h->v2c_off = (int32_t*)calloc(n_verts + 1, sizeof(int32_t));
    if (!h->X || !h->cv || !h->cd || !h->v2c_off) return -1;
    memcpy(h->X, vertices, sizeof(double) * n_verts * dim);
    memcpy(h->cv, cell_vertices, sizeof(int32_t) * n_cells * nv);
    memcpy(h->cd, cell_dofs, sizeof(int32_t) * n_cells * nv);
    for (int64_t c = 0; c < n_cells; ++c)
        for (int i = 0; i < nv; ++i) {
            const int32_t vi = cell_vertices[c * nv + i];
            if (vi < 0 || vi >= n_verts) return -2;
            if (cell_dofs[c * nv + i] < 0 || cell_dofs[c * nv + i] >= n_dofs) return -2;
            h->v2c_off[vi + 1]++;
        }
    for (int64_t v = 0; v < n_verts; ++v) h->v2c_off[v + 1] += h->v2c_off[v];
    const int64_t tot = h->v2c_off[n_verts];
    h->v2c_cells = (int32_t*)malloc(sizeof(int32_t) * (tot ? tot : 1));
    h->v2c_dirs = (double*)malloc(sizeof(double) * (tot ? tot : 1) * dim);
    int32_t* fill = (int32_t*)calloc(n_verts, sizeof(int32_t));
    if (!h->v2c_cells || !h->v2c_dirs || !fill) return -1;
    /* cells visited in ascending order -> each list is sorted; a cell that
     * repeats a vertex (degenerate) is listed once, as in a std::set */
    for (int64_t c = 0; c < n_cells; ++c)
        for (int i = 0; i < nv; ++i) {
            const int32_t vi = cell_vertices[c * nv + i];
            const int32_t base = h->v2c_off[vi];
            if (fill[vi] > 0 && h->v2c_cells[base + fill[vi] - 1] == (int32_t)c) continue;
            h->v2c_cells[base + fill[vi]++] = (int32_t)c;
        }
    /* compact away duplicates (degenerate cells only) */
    {
        int64_t w = 0;
        int32_t* newoff = (int32_t*)malloc(sizeof(int32_t) * (n_verts + 1));
        newoff[0] = 0;
        for (int64_t v = 0; v < n_verts; ++v) {
            for (int32_t k = 0; k < fill[v]; ++k) h->v2c_cells[w++] = h->v2c_cells[h->v2c_off[v] + k];
            newoff[v + 1] = (int32_t)w;
        }
        memcpy(h->v2c_off, newoff, sizeof(int32_t) * (n_verts + 1));
        free(newoff);
    }
    free(fill);
    double Xc[MAXV * 3];
    for (int64_t v = 0; v < n_verts; ++v)
        for (int32_t k = h->v2c_off[v]; k < h->v2c_off[v + 1]; ++k) {
            const int32_t c = h->v2c_cells[k];
            cell_coords(h, c, Xc);
            double ctr[3], dir[3];
            for (int d = 0; d < dim; ++d) {
                double s = 0.0;
                for (int i = 0; i < nv; ++i) s = s + Xc[i * 3 + d];
                ctr[d] = s / (double)nv;
                dir[d] = ctr[d] - h->X[v * dim + d];
            }
            const double nrm = sqrt(norm2(dim, dir));
            for (int d = 0; d < dim; ++d) h->v2c_dirs[(int64_t)k * dim + d] = dir[d] / nrm;
        }
    return 0;
}

int64_t orc_vertex_map_size(const orc_handle* h) { return h->v2c_off ? h->v2c_off[h->nV] : 0; }

void orc_get_vertex_maps(const orc_handle* h, int32_t* offsets, int32_t* cells, double* dirs)
{
    const int64_t tot = orc_vertex_map_size(h);
    memcpy(offsets, h->v2c_off, sizeof(int32_t) * (h->nV + 1));
    memcpy(cells, h->v2c_cells, sizeof(int32_t) * tot);
    memcpy(dirs, h->v2c_dirs, sizeof(double) * tot * h->dim);
}

/* ------------------------------------------------------------------------ */
/* Particle storage                                                          */
/* ------------------------------------------------------------------------ */

static int reserve(orc_handle* h, int64_t cap)
{
    if (cap <= h->cap) return 0;
    int64_t nc = h->cap ? h->cap : 1024;
    while (nc < cap) nc *= 2;
    orc_particle* np = (orc_particle*)realloc(h->P, sizeof(orc_particle) * nc);
    if (!np) return -1;
    h->P = np;
    h->cap = nc;
    return 0;
}

/* sum_i N_i(xi) V[comp][dof_i], accumulated from zero in vertex order
 * (src/pfem2particlehandler.cpp:96-101,154-159,399-404). */
static void interp(const orc_handle* h, int64_t c, const double* xi, const double* V, double* u)
{
    double N[MAXV];
    orc_shape_values(h->dim, xi, N);
    for (int d = 0; d < h->dim; ++d) u[d] = 0.0;
    for (int i = 0; i < h->nv; ++i) {
        const int64_t dof = h->cd[c * h->nv + i];
        for (int d = 0; d < h->dim; ++d) u[d] = u[d] + N[i] * V[d * h->nD + dof];
    }
}

/* One new particle at the centre of cell part `idx` of cell c:
 * seed_particles src/pfem2particlehandler.cpp:87-104 and
 * check_particle_distribution :390-407 (same construction). */
static void make_particle(orc_handle* h, int64_t c, const int* idx, const double* V, orc_particle* p)
{
    double Xc[MAXV * 3];
    memset(p, 0, sizeof(*p));
    for (int d = 0; d < h->dim; ++d) p->xi[d] = (idx[d] + 1.0 / 2) * h->h[d];
    cell_coords(h, c, Xc);
    orc_forward_map(h->dim, Xc, p->xi, p->x);
    p->id = ++h->st.next_id;
    p->cell = (int32_t)c;
    interp(h, c, p->xi, V, p->v);
}

static void part_of_index(const orc_handle* h, int linear, int* idx)
{
    /* cellPartsIndices order, src/pfem2particlehandler.cpp:56-74: x outermost */
    const int* q = h->prm.q;
    if (h->dim == 2) {
        idx[0] = linear / q[1];
        idx[1] = linear % q[1];
    } else {
        idx[0] = linear / (q[1] * q[2]);
        idx[1] = (linear / q[2]) % q[1];
        idx[2] = linear % q[2];
    }
}

/* seed_particles, src/pfem2particlehandler.cpp:43-109 (all cells are locally
 * owned on one rank; particleCount starts at 0 so ids start at 1). */
int orc_seed(orc_handle* h, const double* V)
{
    if (!h->X) return -1;
    if (reserve(h, h->n + h->nC * h->npart)) return -1;
    int idx[3];
    for (int64_t c = 0; c < h->nC; ++c)
        for (int k = 0; k < h->npart; ++k) {
            part_of_index(h, k, idx);
            make_particle(h, c, idx, V, &h->P[h->n++]);
        }
    h->st.n_particles = h->n;
    return 0;
}

/* correct_particle_velocity, src/pfem2particlehandler.cpp:112-139:
 * deltaV = V - Vold per DoF, v += sum_i N_i deltaV_i. */
int orc_correct(orc_handle* h, const double* V, const double* Vold)
{
    const int dim = h->dim, nv = h->nv;
    for (int64_t p = 0; p < h->n; ++p) {
        orc_particle* q = &h->P[p];
        double N[MAXV], corr[3] = {0.0, 0.0, 0.0};
        orc_shape_values(dim, q->xi, N);
        for (int i = 0; i < nv; ++i) {
            const int64_t dof = h->cd[(int64_t)q->cell * nv + i];
            for (int d = 0; d < dim; ++d) {
                const double dv = V[d * h->nD + dof] - Vold[d * h->nD + dof];
                corr[d] = corr[d] + N[i] * dv;
            }
        }
        for (int d = 0; d < dim; ++d) q->v[d] = q->v[d] + corr[d];
    }
    return 0;
}

/* pfem2Particle::find_closest_vertex_of_cell, src/pfem2particle.cpp:186-211:
 * the cell vertex whose unit direction from the previous position F(xi_old)
 * has the largest dot product with unit(velocity_ext); strict '>' keeps the
 * lowest vertex on ties; NaNs never win. */
static int closest_vertex(const orc_handle* h, const double* Xc, const orc_particle* q)
{
    const int dim = h->dim;
    double old[3], vn[3], ptv[3];
    orc_forward_map(dim, Xc, q->xi, old);
    const double vnorm = sqrt(norm2(dim, q->vext));
    for (int d = 0; d < dim; ++d) vn[d] = q->vext[d] / vnorm;
    double best = 0.0;
    int closest = 0;
    for (int v = 0; v < h->nv; ++v) {
        for (int d = 0; d < dim; ++d) ptv[d] = Xc[v * 3 + d] - old[d];
        const double pn = sqrt(norm2(dim, ptv));
        for (int d = 0; d < dim; ++d) ptv[d] = ptv[d] / pn;
        double ang = vn[0] * ptv[0];
        for (int d = 1; d < dim; ++d) ang = ang + vn[d] * ptv[d];
        if (v == 0) best = ang;
        else if (ang > best) {
            best = ang;
            closest = v;
        }
    }
    return closest;
}

typedef struct {
    int64_t map_failures, near_face, searched;
} reloc_counts;

static int near_face(int dim, const double* xi)
{
    for (int d = 0; d < dim; ++d)
        if (fabs(xi[d]) < 1e-12 || fabs(1.0 - xi[d]) < 1e-12) return 1;
    return 0;
}

/* Relocation of one particle, sort_particles_into_subdomains_and_cells
 * src/pfem2particlehandler.cpp:420-491 (single rank: every found cell is
 * locally owned).  Returns 1 if a cell was found (xi and cell updated), 0 if
 * the particle is to be deleted. */
static int relocate(const orc_handle* h, orc_particle* q, reloc_counts* rc)
{
    const int dim = h->dim;
    double Xc[MAXV * 3], xi[3];
    cell_coords(h, q->cell, Xc);
    /* :424-431 inverse map in the current cell */
    int st = orc_inverse_map(dim, Xc, q->x, xi);
    if (st) rc->map_failures++;
    if (st == 0 && inside_unit(dim, xi)) {
        for (int d = 0; d < dim; ++d) q->xi[d] = xi[d];
        if (near_face(dim, xi)) rc->near_face++;
        return 1;
    }
    rc->searched++;
    /* :442-446 closest vertex and unit vertex->particle direction */
    const int cv = closest_vertex(h, Xc, q);
    double vtp[3];
    for (int d = 0; d < dim; ++d) vtp[d] = q->x[d] - Xc[cv * 3 + d];
    const double vn = sqrt(norm2(dim, vtp));
    for (int d = 0; d < dim; ++d) vtp[d] = vtp[d] / vn;
    const int32_t vid = h->cv[(int64_t)q->cell * h->nv + cv];
    const int32_t b = h->v2c_off[vid], n = h->v2c_off[vid + 1] - b;
    /* :451-456 candidates by descending centre-direction dot product; std::sort
     * on <= 16 elements is libstdc++'s insertion sort, i.e. stable */
    int32_t perm[64];
    double dots[64];
    const int nn = n < 64 ? n : 64;
    for (int k = 0; k < nn; ++k) {
        const double* cd = &h->v2c_dirs[(int64_t)(b + k) * dim];
        double s = cd[0] * vtp[0];
        for (int d = 1; d < dim; ++d) s = s + cd[d] * vtp[d];
        dots[k] = s;
        perm[k] = k;
    }
    for (int i = 1; i < nn; ++i) {
        const int32_t pi = perm[i];
        int j = i;
        while (j > 0 && dots[pi] > dots[perm[j - 1]]) {
            perm[j] = perm[j - 1];
            --j;
        }
        perm[j] = pi;
    }
    /* :458-478 first candidate whose inverse map lands inside.  The list
     * holds the particle's own cell too; its inverse map is deterministic and
     * already failed above, so it is skipped (same outcome, one solve less). */
    const int32_t own = q->cell;
    for (int k = 0; k < nn; ++k) {
        const int32_t c = h->v2c_cells[b + perm[k]];
        if (c == own) continue;
        cell_coords(h, c, Xc);
        st = orc_inverse_map(dim, Xc, q->x, xi);
        if (st) {
            rc->map_failures++;
            continue;
        }
        if (inside_unit(dim, xi)) {
            for (int d = 0; d < dim; ++d) q->xi[d] = xi[d];
            q->cell = c;
            if (near_face(dim, xi)) rc->near_face++;
            return 1;
        }
    }
    return 0; /* :488-491 deleted */
}

/* ------------------------------------------------------------------------ */
/* Parallel helper (baseline timing only)                                   */
/* ------------------------------------------------------------------------ */

typedef struct {
    orc_handle* h;
    const double* V;
    int8_t* lost_at;
    int64_t begin, end;
    reloc_counts rc;
} move_task;

/* The transport velocity of one sub-step from reference coordinates xi of
 * cell c.  Euler (the reference, move_particles :151-159): u(xi).  RK2, an
 * opt-in with no counterpart in the reference: the midpoint rule in the
 * particle's own cell, u(xi_mid) with xi_mid = xi + (h/2) J(xi)^-1 u(xi) and
 * u the cell's Q1 field (extrapolated where xi_mid lies outside the unit
 * cell).  xi_mid is the midpoint's exact reference position on affine cells
 * and within O(h^2) of it on others, so the scheme is second order.  A
 * non-positive Jacobian determinant falls back to u(xi). */
static void transport_velocity(const orc_handle* h, int64_t c, const double* xi, const double* V, double* u)
{
    interp(h, c, xi, V, u);
    if (h->prm.integrator != ORC_RK2) return;
    const int dim = h->dim;
    double Xc[MAXV * 3], J[3][3], Ji[3][3], dl[3], xm[3];
    cell_coords(h, c, Xc);
    jacobian(dim, Xc, xi, J);
    const double det = invert(dim, J, Ji);
    if (!(det > 0.0)) return;
    matvec(dim, Ji, u, dl);
    const double half = h->dtp * 0.5;
    for (int d = 0; d < dim; ++d) xm[d] = xi[d] + half * dl[d];
    interp(h, c, xm, V, u);
}

static void move_range(move_task* t)
{
    orc_handle* h = t->h;
    const int dim = h->dim;
    for (int64_t p = t->begin; p < t->end; ++p) {
        orc_particle* q = &h->P[p];
        t->lost_at[p] = -1;
        for (int s = 0; s < h->S; ++s) {
            /* move_particles :151-163 */
            double u[3], step[3];
            transport_velocity(h, q->cell, q->xi, t->V, u);
            for (int d = 0; d < dim; ++d) {
                q->vext[d] = u[d];
                step[d] = u[d] * h->dtp;
                q->x[d] = q->x[d] + step[d];
            }
            /* :166 relocation */
            if (!relocate(h, q, &t->rc)) {
                t->lost_at[p] = (int8_t)s;
                break;
            }
        }
    }
}

static void* move_thread(void* arg)
{
    move_range((move_task*)arg);
    return NULL;
}

/* check_particle_distribution, src/pfem2particlehandler.cpp:356-410. */
static int check_distribution(orc_handle* h, const double* V)
{
    const int dim = h->dim;
    const int* q = h->prm.q;
    const int maxpp = h->prm.max_per_part;
    int32_t* counts = (int32_t*)calloc((size_t)h->nC * h->npart_ext, sizeof(int32_t));
    uint8_t* touched = (uint8_t*)calloc((size_t)h->nC, 1);
    if (!counts || !touched) return -1;
#define EXT_PART(pp, out)                                                                      \
    do {                                                                                       \
        int e_ = 0;                                                                            \
        for (int d_ = 0; d_ < dim; ++d_) {                                                     \
            int k_ = (int)((pp)->xi[d_] / h->h[d_]); /* :369-370 */                           \
            if (k_ < 0) k_ = 0;                                                                \
            if (k_ > q[d_]) k_ = q[d_];                                                        \
            e_ = e_ * (q[d_] + 1) + k_;                                                        \
        }                                                                                      \
        (out) = e_;                                                                            \
    } while (0)

    if (h->prm.removal_order == ORC_ORDER_VECTOR) {
        /* :368-379 swap-with-back in vector order; '>' lets max+1 survive */
        int64_t i = 0;
        while (i < h->n) {
            orc_particle* p = &h->P[i];
            int e;
            EXT_PART(p, e);
            int32_t* cnt = &counts[(int64_t)p->cell * h->npart_ext + e];
            touched[p->cell] = 1;
            if (*cnt > maxpp) {
                h->P[i] = h->P[h->n - 1];
                h->n--;
                h->st.removed++;
            } else {
                (*cnt)++;
                ++i;
            }
        }
    } else {
        /* id order: in each (cell, part) the particles with the smallest
         * key(id) are examined first; the vector is rebuilt in (cell, part,
         * key) order. */
        const int64_t n = h->n;
        int64_t* coff = (int64_t*)calloc((size_t)h->nC + 1, sizeof(int64_t));
        int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (n ? n : 1));
        int32_t* ext = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1));
        uint32_t* key = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
        orc_particle* np = (orc_particle*)malloc(sizeof(orc_particle) * (n ? n : 1));
        if (!coff || !order || !ext || !key || !np) return -1;
        for (int64_t i = 0; i < n; ++i) {
            int e;
            EXT_PART(&h->P[i], e);
            ext[i] = e;
            key[i] = orc_key(h->P[i].id, h->prm.removal_seed);
            coff[h->P[i].cell + 1]++;
            touched[h->P[i].cell] = 1;
        }
        for (int64_t c = 0; c < h->nC; ++c) coff[c + 1] += coff[c];
        {
            int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * ((size_t)h->nC + 1));
            memcpy(fill, coff, sizeof(int64_t) * ((size_t)h->nC + 1));
            for (int64_t i = 0; i < n; ++i) order[fill[h->P[i].cell]++] = i;
            free(fill);
        }
        int64_t w = 0;
        for (int64_t c = 0; c < h->nC; ++c) {
            const int64_t b = coff[c], e = coff[c + 1];
            for (int64_t i = b + 1; i < e; ++i) { /* insertion sort by (part, key) */
                const int64_t pi = order[i];
                int64_t j = i;
                while (j > b && (ext[order[j - 1]] > ext[pi] ||
                                 (ext[order[j - 1]] == ext[pi] && key[order[j - 1]] > key[pi]))) {
                    order[j] = order[j - 1];
                    --j;
                }
                order[j] = pi;
            }
            for (int64_t i = b; i < e; ++i) {
                const int64_t pi = order[i];
                int32_t* cnt = &counts[c * h->npart_ext + ext[pi]];
                if (*cnt > maxpp) {
                    h->st.removed++;
                } else {
                    (*cnt)++;
                    np[w++] = h->P[pi];
                }
            }
        }
        memcpy(h->P, np, sizeof(orc_particle) * w);
        h->n = w;
        free(coff);
        free(order);
        free(ext);
        free(key);
        free(np);
    }
    /* :385-409 one particle at the centre of every empty part of every cell
     * that had at least one particle, cells ascending, parts in
     * cellPartsIndices order */
    int idx[3];
    for (int64_t c = 0; c < h->nC; ++c) {
        if (!touched[c]) continue;
        for (int k = 0; k < h->npart; ++k) {
            part_of_index(h, k, idx);
            int e = 0;
            for (int d = 0; d < dim; ++d) e = e * (q[d] + 1) + idx[d];
            if (counts[c * h->npart_ext + e] == 0) {
                if (reserve(h, h->n + 1)) return -1;
                make_particle(h, c, idx, V, &h->P[h->n++]);
                h->st.seeded++;
            }
        }
    }
#undef EXT_PART
    free(counts);
    free(touched);
    return 0;
}

/* move_particles, src/pfem2particlehandler.cpp:142-171.  Each particle's S
 * sub-steps are independent of the others, so they run per particle (and in
 * parallel when n_threads > 1); the vector order the reference produces by
 * deleting lost particles with swap-with-back after every sub-step
 * (:488-491) is then replayed sub-step by sub-step. */
int orc_move(orc_handle* h, const double* V)
{
    if (!h->X) return -1;
    const int64_t n = h->n;
    int8_t* lost_at = (int8_t*)malloc(n ? n : 1);
    if (!lost_at) return -1;
    const int T = h->prm.n_threads;
    move_task tasks[256];
    const int nt = T < 256 ? T : 256;
    for (int t = 0; t < nt; ++t) {
        tasks[t].h = h;
        tasks[t].V = V;
        tasks[t].lost_at = lost_at;
        tasks[t].begin = n * t / nt;
        tasks[t].end = n * (t + 1) / nt;
        memset(&tasks[t].rc, 0, sizeof(reloc_counts));
    }
    if (nt == 1) {
        move_range(&tasks[0]);
    } else {
        pthread_t th[256];
        for (int t = 0; t < nt; ++t) pthread_create(&th[t], NULL, move_thread, &tasks[t]);
        for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
    }
    for (int t = 0; t < nt; ++t) {
        h->st.map_failures += tasks[t].rc.map_failures;
        h->st.near_face += tasks[t].rc.near_face;
        h->st.searched += tasks[t].rc.searched;
    }
    /* replay the swap-with-back deletions of every sub-step; lost_at travels
     * with its particle */
    for (int s = 0; s < h->S; ++s) {
        int64_t i = 0;
        while (i < h->n) {
            if (lost_at[i] == s) {
                h->P[i] = h->P[h->n - 1];
                lost_at[i] = lost_at[h->n - 1];
                h->n--;
                h->st.lost++;
            } else {
                ++i;
            }
        }
    }
    free(lost_at);
    int rc = check_distribution(h, V);
    h->st.n_particles = h->n;
    return rc;
}

typedef struct {
    orc_handle* h;
    double* part;
    int t, nt;
} proj_task;

static void* proj_worker(void* arg)
{
    const proj_task* a = (const proj_task*)arg;
    orc_handle* h = a->h;
    const int dim = h->dim, nv = h->nv;
    const int64_t nD = h->nD;
    double* buf = a->part + (size_t)a->t * nD * (dim + 1);
    for (int64_t p = h->n * a->t / a->nt; p < h->n * (a->t + 1) / a->nt; ++p) {
        const orc_particle* q = &h->P[p];
        double N[MAXV];
        orc_shape_values(dim, q->xi, N);
        for (int i = 0; i < nv; ++i) {
            const int64_t dof = h->cd[(int64_t)q->cell * nv + i];
            for (int d = 0; d < dim; ++d) buf[d * nD + dof] += N[i] * q->v[d];
            buf[dim * nD + dof] += N[i];
        }
    }
    return NULL;
}

/* project_particle_fields, src/pfem2particlehandler.cpp:174-215: weighted
 * scatter num[d][dof] += N_i v_d, den[dof] += N_i in vector order, then
 * num/den with no guard (0/0 -> NaN where no particle touches a DoF). */
int orc_project(orc_handle* h, double* V_out)
{
    const int dim = h->dim, nv = h->nv;
    const int64_t nD = h->nD;
    double* den = (double*)calloc((size_t)nD, sizeof(double));
    if (!den) return -1;
    for (int64_t k = 0; k < nD * dim; ++k) V_out[k] = 0.0;
    const int T = h->prm.n_threads;
    if (T <= 1) {
        for (int64_t p = 0; p < h->n; ++p) {
            const orc_particle* q = &h->P[p];
            double N[MAXV];
            orc_shape_values(dim, q->xi, N);
            for (int i = 0; i < nv; ++i) {
                const int64_t dof = h->cd[(int64_t)q->cell * nv + i];
                for (int d = 0; d < dim; ++d) V_out[d * nD + dof] = V_out[d * nD + dof] + N[i] * q->v[d];
                den[dof] = den[dof] + N[i];
            }
        }
    } else {
        /* baseline timing: per-thread partial sums, added in thread order */
        const int nt = T < 64 ? T : 64;
        double* part = (double*)calloc((size_t)nt * nD * (dim + 1), sizeof(double));
        if (!part) return -1;
        proj_task pt[64];
        pthread_t th[64];
        for (int t = 0; t < nt; ++t) {
            pt[t].h = h;
            pt[t].part = part;
            pt[t].t = t;
            pt[t].nt = nt;
        }
        for (int t = 0; t < nt; ++t) pthread_create(&th[t], NULL, proj_worker, &pt[t]);
        for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
        for (int t = 0; t < nt; ++t) {
            const double* buf = part + (size_t)t * nD * (dim + 1);
            for (int64_t k = 0; k < nD * dim; ++k) V_out[k] = V_out[k] + buf[k];
            for (int64_t k = 0; k < nD; ++k) den[k] = den[k] + buf[dim * nD + k];
        }
        free(part);
    }
    int64_t nan_dofs = 0;
    for (int64_t k = 0; k < nD; ++k) {
        if (den[k] == 0.0) nan_dofs++;
        for (int d = 0; d < dim; ++d) V_out[d * nD + k] = V_out[d * nD + k] / den[k];
    }
    h->st.nan_dofs = nan_dofs;
    free(den);
    return 0;
}

int64_t orc_n_particles(const orc_handle* h) { return h->n; }

void orc_get_particles(const orc_handle* h, uint32_t* id, int32_t* cell, double* x, double* xi, double* v)
{
    const int dim = h->dim;
    for (int64_t p = 0; p < h->n; ++p) {
        const orc_particle* q = &h->P[p];
        if (id) id[p] = q->id;
        if (cell) cell[p] = q->cell;
        for (int d = 0; d < dim; ++d) {
            if (x) x[p * dim + d] = q->x[d];
            if (xi) xi[p * dim + d] = q->xi[d];
            if (v) v[p * dim + d] = q->v[d];
        }
    }
}

int orc_set_particles(orc_handle* h, int64_t n, const uint32_t* id, const int32_t* cell, const double* x,
                      const double* xi, const double* v, uint32_t next_id)
{
    const int dim = h->dim;
    if (reserve(h, n)) return -1;
    for (int64_t p = 0; p < n; ++p) {
        orc_particle* q = &h->P[p];
        memset(q, 0, sizeof(*q));
        q->id = id[p];
        q->cell = cell[p];
        for (int d = 0; d < dim; ++d) {
            q->x[d] = x[p * dim + d];
            q->xi[d] = xi[p * dim + d];
            q->v[d] = v[p * dim + d];
        }
    }
    h->n = n;
    h->st.n_particles = n;
    h->st.next_id = next_id;
    return 0;
}

void orc_get_stats(const orc_handle* h, orc_stats* s)
{
    *s = h->st;
    s->n_particles = h->n;
}

void orc_reset_stats(orc_handle* h)
{
    const uint32_t nid = h->st.next_id;
    const int64_t nan = h->st.nan_dofs;
    memset(&h->st, 0, sizeof(h->st));
    h->st.next_id = nid;
    h->st.nan_dofs = nan;
    h->st.n_particles = h->n;
}

/* ------------------------------------------------------------------------ */
/* Differentiated window (no reference counterpart: the reference has no     */
/* adjoint).  K time steps of correct_particle_velocity (:112-139, when Vold  */
/* is given) and move_particles' sub-steps with relocation (:142-167,        */
/* :413-503) from the current particles, check_particle_distribution left    */
/* out, then project_particle_fields (:174-215).  The particle set is not    */
/* changed.  The backward pass holds every particle's cell sequence fixed     */
/* (cell assignment is the discrete, non-differentiated part) and applies    */
/* the chain rule to                                                         */
/*   correction   v  += sum_i N_i(xi) dV_i                                   */
/*   sub-step     x'  = F_c(xi) + h u_c(xi),  xi' = F_c'^-1(x'),  h = dt/S    */
/*   projection   U_j = sum N_j v / sum N_j                                  */
/* with dxi'/dx' = J_c'(xi')^-1.  Particles lost inside the window do not    */
/* reach the projection and get zero gradient.                              */
/* ------------------------------------------------------------------------ */

typedef struct {
    int32_t cell;
    double xi[3];
} orc_wstate;

/* One particle through the window; states[t] = (cell, xi) before sub-step t,
 * states[K*S] = the final one (states may be NULL).  Returns 1 if the particle
 * is alive at the end. */
static int window_particle(const orc_handle* h, orc_particle* q, int K, const double* V, const double* Vold,
                           orc_wstate* states)
{
    const int dim = h->dim, nv = h->nv, S = h->S;
    reloc_counts rc = {0, 0, 0};
    for (int k = 0; k < K; ++k) {
        if (Vold) { /* orc_correct's arithmetic */
            double N[MAXV], corr[3] = {0.0, 0.0, 0.0};
            orc_shape_values(dim, q->xi, N);
            for (int i = 0; i < nv; ++i) {
                const int64_t dof = h->cd[(int64_t)q->cell * nv + i];
                for (int d = 0; d < dim; ++d) {
                    const double dv = V[d * h->nD + dof] - Vold[d * h->nD + dof];
                    corr[d] = corr[d] + N[i] * dv;
                }
            }
            for (int d = 0; d < dim; ++d) q->v[d] = q->v[d] + corr[d];
        }
        for (int s = 0; s < S; ++s) {
            if (states) {
                orc_wstate* w = &states[k * S + s];
                w->cell = q->cell;
                for (int d = 0; d < dim; ++d) w->xi[d] = q->xi[d];
            }
            double u[3], step[3];
            interp(h, q->cell, q->xi, V, u);
            for (int d = 0; d < dim; ++d) {
                q->vext[d] = u[d];
                step[d] = u[d] * h->dtp;
                q->x[d] = q->x[d] + step[d];
            }
            if (!relocate(h, q, &rc)) return 0;
        }
    }
    if (states) {
        orc_wstate* w = &states[K * S];
        w->cell = q->cell;
        for (int d = 0; d < dim; ++d) w->xi[d] = q->xi[d];
    }
    return 1;
}

/* Forward pass of the window: final particles into fin (n entries, alive[p]
 * set), projection into U with den (nD) kept. */
static int window_forward(const orc_handle* h, int K, const double* V, const double* Vold, const double* v0,
                          int empty_policy, orc_particle* fin, uint8_t* alive, double* U, double* den)
{
    const int dim = h->dim, nv = h->nv;
    const int64_t nD = h->nD;
    for (int64_t p = 0; p < h->n; ++p) {
        fin[p] = h->P[p];
        if (v0)
            for (int d = 0; d < dim; ++d) fin[p].v[d] = v0[p * dim + d];
        alive[p] = (uint8_t)window_particle(h, &fin[p], K, V, Vold, NULL);
    }
    for (int64_t k = 0; k < nD * dim; ++k) U[k] = 0.0;
    for (int64_t k = 0; k < nD; ++k) den[k] = 0.0;
    for (int64_t p = 0; p < h->n; ++p) {
        if (!alive[p]) continue;
        const orc_particle* q = &fin[p];
        double N[MAXV];
        orc_shape_values(dim, q->xi, N);
        for (int i = 0; i < nv; ++i) {
            const int64_t dof = h->cd[(int64_t)q->cell * nv + i];
            for (int d = 0; d < dim; ++d) U[d * nD + dof] = U[d * nD + dof] + N[i] * q->v[d];
            den[dof] = den[dof] + N[i];
        }
    }
    for (int64_t j = 0; j < nD; ++j)
        for (int d = 0; d < dim; ++d) {
            if (den[j] == 0.0 && empty_policy == 1) U[d * nD + j] = V[d * nD + j];
            else U[d * nD + j] = U[d * nD + j] / den[j];
        }
    return 0;
}

int orc_window_forward(orc_handle* h, int K, const double* V, const double* Vold, const double* v0,
                       int empty_policy, double* U)
{
    if (h->prm.integrator != ORC_EULER) return -2; /* the window differentiates Euler sub-steps */
    if (!h->X || K < 0) return -1;
    const int64_t n = h->n;
    orc_particle* fin = (orc_particle*)malloc(sizeof(orc_particle) * (n ? n : 1));
    uint8_t* alive = (uint8_t*)malloc(n ? n : 1);
    double* den = (double*)malloc(sizeof(double) * (h->nD ? h->nD : 1));
    int rc = (fin && alive && den) ? window_forward(h, K, V, Vold, v0, empty_policy, fin, alive, U, den) : -1;
    free(fin);
    free(alive);
    free(den);
    return rc;
}

/* Final particle states of the window (cell -1: deleted inside it), in the
 * oracle's current particle order. */
int orc_window_particles(orc_handle* h, int K, const double* V, const double* Vold, const double* v0, int32_t* cell,
                         double* x, double* xi, double* v)
{
    if (h->prm.integrator != ORC_EULER) return -2; /* the window differentiates Euler sub-steps */
    if (!h->X || K < 0) return -1;
    const int dim = h->dim;
    for (int64_t p = 0; p < h->n; ++p) {
        orc_particle q = h->P[p];
        if (v0)
            for (int d = 0; d < dim; ++d) q.v[d] = v0[p * dim + d];
        const int alive = window_particle(h, &q, K, V, Vold, NULL);
        cell[p] = alive ? q.cell : -1;
        for (int d = 0; d < dim; ++d) {
            x[p * dim + d] = q.x[d];
            xi[p * dim + d] = q.xi[d];
            v[p * dim + d] = q.v[d];
        }
    }
    return 0;
}

/* Forward + backward.  gU: dJ/dU (dim x nD).  Outputs g_v0 (n x dim, the
 * gradient with respect to the particle velocities at the window start),
 * g_V and g_Vold (dim x nD; g_Vold = 0 without Vold).  Any output may be NULL. */
int orc_window_adjoint(orc_handle* h, int K, const double* V, const double* Vold, const double* v0,
                       int empty_policy, const double* gU, double* U, double* g_v0, double* g_V, double* g_Vold)
{
    if (h->prm.integrator != ORC_EULER) return -2; /* the window differentiates Euler sub-steps */
    if (!h->X || K < 0) return -1;
    const int dim = h->dim, nv = h->nv, S = h->S;
    const int64_t n = h->n, nD = h->nD;
    const int T = K * S;
    const size_t nDd = (size_t)(nD * dim) + 1;
    orc_particle* fin = (orc_particle*)malloc(sizeof(orc_particle) * (n ? n : 1));
    uint8_t* alive = (uint8_t*)malloc(n ? n : 1);
    double* den = (double*)malloc(sizeof(double) * (nD ? nD : 1));
    double* Uw = (double*)malloc(sizeof(double) * nDd);
    double* gnum = (double*)calloc(nDd, sizeof(double));
    double* gden = (double*)calloc((size_t)nD + 1, sizeof(double));
    double* gadv = (double*)calloc(nDd, sizeof(double));
    double* gdv = (double*)calloc(nDd, sizeof(double));
    orc_wstate* st = (orc_wstate*)malloc(sizeof(orc_wstate) * (size_t)(T + 1));
    int rc = -1;
    if (!fin || !alive || !den || !Uw || !gnum || !gden || !gadv || !gdv || !st) goto done;
    rc = window_forward(h, K, V, Vold, v0, empty_policy, fin, alive, Uw, den);
    if (rc) goto done;
    if (U)
        for (int64_t k = 0; k < nD * dim; ++k) U[k] = Uw[k];
    /* projection: U_j = num_j / den_j */
    for (int64_t j = 0; j < nD; ++j) {
        if (den[j] == 0.0) {
            if (empty_policy == 1)
                for (int d = 0; d < dim; ++d) gadv[d * nD + j] = gU[d * nD + j];
            continue;
        }
        double s = 0.0;
        for (int d = 0; d < dim; ++d) {
            gnum[d * nD + j] = gU[d * nD + j] / den[j];
            s = s + gU[d * nD + j] * Uw[d * nD + j];
        }
        gden[j] = -s / den[j];
    }
    for (int64_t p = 0; p < n; ++p) {
        if (g_v0)
            for (int d = 0; d < dim; ++d) g_v0[p * dim + d] = 0.0;
        if (!alive[p]) continue;
        /* the particle's trajectory again, with its states */
        orc_particle q = h->P[p];
        if (v0)
            for (int d = 0; d < dim; ++d) q.v[d] = v0[p * dim + d];
        window_particle(h, &q, K, V, Vold, st);
        double N[MAXV], G[MAXV][3], gv[3] = {0.0, 0.0, 0.0}, gxi[3] = {0.0, 0.0, 0.0};
        {
            const orc_wstate* w = &st[T];
            orc_shape_values(dim, w->xi, N);
            shape_grads(dim, w->xi, G);
            for (int i = 0; i < nv; ++i) {
                const int64_t j = h->cd[(int64_t)w->cell * nv + i];
                double a = gden[j];
                for (int d = 0; d < dim; ++d) {
                    gv[d] = gv[d] + N[i] * gnum[d * nD + j];
                    a = a + gnum[d * nD + j] * q.v[d];
                }
                for (int k = 0; k < dim; ++k) gxi[k] = gxi[k] + G[i][k] * a;
            }
        }
        if (g_v0)
            for (int d = 0; d < dim; ++d) g_v0[p * dim + d] = gv[d];
        for (int t = T - 1; t >= 0; --t) {
            const orc_wstate* a = &st[t];
            const orc_wstate* b = &st[t + 1];
            double Xb[MAXV * 3], Xa[MAXV * 3], Jb[3][3], Bi[3][3], Ja[3][3], y[3], A[3][3];
            cell_coords(h, b->cell, Xb);
            jacobian(dim, Xb, b->xi, Jb);
            invert(dim, Jb, Bi);
            for (int d = 0; d < dim; ++d) { /* y = J_b^-T gxi */
                double s = 0.0;
                for (int k = 0; k < dim; ++k) s = s + Bi[k][d] * gxi[k];
                y[d] = s;
            }
            cell_coords(h, a->cell, Xa);
            jacobian(dim, Xa, a->xi, Ja);
            orc_shape_values(dim, a->xi, N);
            shape_grads(dim, a->xi, G);
            for (int d = 0; d < dim; ++d)
                for (int k = 0; k < dim; ++k) A[d][k] = 0.0;
            for (int i = 0; i < nv; ++i) {
                const int64_t j = h->cd[(int64_t)a->cell * nv + i];
                for (int d = 0; d < dim; ++d) {
                    const double vd = V[d * nD + j];
                    for (int k = 0; k < dim; ++k) A[d][k] = A[d][k] + vd * G[i][k];
                    gadv[d * nD + j] = gadv[d * nD + j] + (h->dtp * N[i]) * y[d];
                }
            }
            for (int k = 0; k < dim; ++k) {
                double s = 0.0, r = 0.0;
                for (int d = 0; d < dim; ++d) {
                    s = s + Ja[d][k] * y[d];
                    r = r + A[d][k] * y[d];
                }
                gxi[k] = s + h->dtp * r;
            }
            if (Vold && t % S == 0) { /* the correction at the start of step t/S */
                for (int i = 0; i < nv; ++i) {
                    const int64_t j = h->cd[(int64_t)a->cell * nv + i];
                    double c = 0.0;
                    for (int d = 0; d < dim; ++d) {
                        c = c + (V[d * nD + j] - Vold[d * nD + j]) * gv[d];
                        gdv[d * nD + j] = gdv[d * nD + j] + N[i] * gv[d];
                    }
                    for (int k = 0; k < dim; ++k) gxi[k] = gxi[k] + G[i][k] * c;
                }
            }
        }
    }
    for (int64_t k = 0; k < nD * dim; ++k) {
        if (g_V) g_V[k] = gadv[k] + gdv[k];
        if (g_Vold) g_Vold[k] = -gdv[k];
    }
    rc = 0;
done:
    free(fin);
    free(alive);
    free(den);
    free(Uw);
    free(gnum);
    free(gden);
    free(gadv);
    free(gdv);
    free(st);
    return rc;
}
