// UNV mesh reader (host code): GridIn::read_unv as the reference's solver
// calls it (src/pfem2solver.cpp:116-119), for the particle path's needs.
//
// Universal-file datasets read: 2411 (node label, then its three
// coordinates, FORTRAN 'D' exponents allowed) and 2412 (element records:
// label, type, three descriptors, node count, then the node labels; beam
// types 11/21/22/24 carry one more record line).  Quads (types 44, 94) in 2D
// and hexes (115) in 3D become cells; every other element and dataset
// (boundary edges and faces, groups 2467, units 164) is skipped.  The UNV
// node order (counter-clockwise per face) maps to deal.II's lexicographic
// order, cells whose Jacobian at the centre is negative get their first two
// directions swapped, and nodes no cell uses are dropped; vertices are
// numbered by ascending node label.

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "pfem2gpu.h"

namespace {

struct UnvMesh {
    int dim = 0;
    std::vector<double> verts;     // n_verts x dim
    std::vector<int32_t> cells;    // n_cells x 2^dim, lexicographic
    std::string error;
};

bool next_line(FILE* f, std::string& line)
{
    line.clear();
    char buf[512];
    while (std::fgets(buf, sizeof buf, f)) {
        line += buf;
        if (!line.empty() && line.back() == '\n') break;
    }
    if (line.empty()) return false;
    while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
    return true;
}

bool is_delim(const std::string& s)
{
    size_t a = s.find_first_not_of(" \t");
    if (a == std::string::npos) return false;
    size_t b = s.find_last_not_of(" \t");
    return s.compare(a, b - a + 1, "-1") == 0;
}

std::vector<long long> ints_of(const std::string& s)
{
    std::vector<long long> out;
    const char* p = s.c_str();
    char* end = nullptr;
    while (true) {
        errno = 0;
        const long long v = std::strtoll(p, &end, 10);
        if (end == p) break;
        out.push_back(v);
        p = end;
    }
    return out;
}

std::vector<double> reals_of(std::string s)
{
    for (char& c : s)
        if (c == 'D' || c == 'd') c = 'E';
    std::vector<double> out;
    const char* p = s.c_str();
    char* end = nullptr;
    while (true) {
        const double v = std::strtod(p, &end);
        if (end == p) break;
        out.push_back(v);
        p = end;
    }
    return out;
}

// Swap the first two reference directions of left-handed cells.
void orient(int dim, const std::vector<double>& X, std::vector<int32_t>& cells)
{
    const int nv = 1 << dim;
    const size_t nc = cells.size() / nv;
    for (size_t c = 0; c < nc; ++c) {
        int32_t* cv = &cells[c * nv];
        double det;
        if (dim == 2) {
            double e[2], f[2];
            for (int d = 0; d < 2; ++d) {
                e[d] = (X[cv[1] * 2 + d] + X[cv[3] * 2 + d] - X[cv[0] * 2 + d] - X[cv[2] * 2 + d]) * 0.5;
                f[d] = (X[cv[2] * 2 + d] + X[cv[3] * 2 + d] - X[cv[0] * 2 + d] - X[cv[1] * 2 + d]) * 0.5;
            }
            det = e[0] * f[1] - e[1] * f[0];
            if (det < 0) std::swap(cv[1], cv[2]);
        } else {
            double J[3][3];
            for (int k = 0; k < 3; ++k)
                for (int d = 0; d < 3; ++d) {
                    double hi = 0.0, lo = 0.0;
                    for (int i = 0; i < 8; ++i) ((i >> k) & 1 ? hi : lo) += X[cv[i] * 3 + d];
                    J[d][k] = (hi - lo) / 4;
                }
            det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                  J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
            if (det < 0) {
                std::swap(cv[1], cv[2]);
                std::swap(cv[5], cv[6]);
            }
        }
    }
}

bool parse(const char* path, int want_dim, UnvMesh& m)
{
    FILE* f = std::fopen(path, "r");
    if (!f) {
        m.error = std::string("cannot open ") + path;
        return false;
    }
    std::map<long long, std::vector<double>> nodes;
    std::vector<std::pair<int, std::vector<long long>>> elems;
    std::string line;
    bool ok = true;
    while (ok && next_line(f, line)) {
        if (!is_delim(line)) continue;
        if (!next_line(f, line)) break;
        const std::vector<long long> ds = ints_of(line);
        const long long id = ds.empty() ? -1 : ds[0];
        if (id == 2411) {
            while (next_line(f, line) && !is_delim(line)) {
                const std::vector<long long> h = ints_of(line);
                std::string xyz;
                if (h.empty() || !next_line(f, xyz)) {
                    ok = false;
                    m.error = "truncated node record";
                    break;
                }
                std::vector<double> x = reals_of(xyz);
                x.resize(3, 0.0);
                nodes[h[0]] = x;
            }
        } else if (id == 2412) {
            while (next_line(f, line) && !is_delim(line)) {
                const std::vector<long long> h = ints_of(line);
                if (h.size() < 6) {
                    ok = false;
                    m.error = "bad element record";
                    break;
                }
                const int type = (int)h[1];
                const long long nn = h[5];
                if (type == 11 || type == 21 || type == 22 || type == 24) next_line(f, line);  // beam record
                std::vector<long long> conn;
                while ((long long)conn.size() < nn && next_line(f, line)) {
                    const std::vector<long long> c = ints_of(line);
                    conn.insert(conn.end(), c.begin(), c.end());
                }
                if ((long long)conn.size() < nn) {
                    ok = false;
                    m.error = "truncated element record";
                    break;
                }
                if (type == 44 || type == 94 || type == 115) elems.emplace_back(type, conn);
            }
        } else {
            while (next_line(f, line) && !is_delim(line)) {
            }
        }
    }
    std::fclose(f);
    if (!ok) return false;
    if (elems.empty()) {
        m.error = "UNV file has no quad (44) or hex (115) elements";
        return false;
    }
    const int edim = elems[0].first == 115 ? 3 : 2;
    const int dim = want_dim ? want_dim : edim;
    if (dim != edim) {
        m.error = "UNV elements are " + std::to_string(edim) + "D, asked for " + std::to_string(dim) + "D";
        return false;
    }
    static const int ucd2d[4] = {0, 1, 3, 2}, ucd3d[8] = {0, 1, 3, 2, 4, 5, 7, 6};
    const int nv = 1 << dim;
    const int* map = dim == 2 ? ucd2d : ucd3d;
    std::map<long long, int32_t> label;  // used node labels, ascending
    std::vector<long long> conn;
    for (const auto& e : elems) {
        if ((e.first == 115) != (dim == 3)) continue;
        for (int i = 0; i < nv; ++i) {
            const long long lab = e.second[map[i]];
            conn.push_back(lab);
            label[lab] = 0;
        }
    }
    int32_t k = 0;
    for (auto& kv : label) {
        if (!nodes.count(kv.first)) {
            m.error = "element refers to a missing node";
            return false;
        }
        kv.second = k++;
    }
    m.dim = dim;
    m.verts.resize((size_t)k * dim);
    for (const auto& kv : label) {
        const std::vector<double>& x = nodes[kv.first];
        for (int d = 0; d < dim; ++d) m.verts[(size_t)kv.second * dim + d] = x[d];
    }
    m.cells.resize(conn.size());
    for (size_t i = 0; i < conn.size(); ++i) m.cells[i] = label[conn[i]];
    orient(dim, m.verts, m.cells);
    return true;
}

thread_local std::string unv_error;

}  // namespace

extern "C" int pfem2gpu_read_unv(const char* path, int dim, int32_t* dim_out, int64_t* n_verts, int64_t* n_cells,
                                 double* vertices, int32_t* cell_vertices, int64_t verts_capacity,
                                 int64_t cells_capacity)
{
    if (!path || !n_verts || !n_cells || (dim != 0 && dim != 2 && dim != 3)) return PFEM2GPU_ERR_ARG;
    UnvMesh m;
    if (!parse(path, dim, m)) {
        unv_error = m.error;
        return PFEM2GPU_ERR_ARG;
    }
    if (dim_out) *dim_out = m.dim;
    const int nv = 1 << m.dim;
    *n_verts = (int64_t)(m.verts.size() / m.dim);
    *n_cells = (int64_t)(m.cells.size() / nv);
    if (!vertices && !cell_vertices) return PFEM2GPU_OK;
    if (verts_capacity < *n_verts || cells_capacity < *n_cells) {
        unv_error = "output arrays too small";
        return PFEM2GPU_ERR_ARG;
    }
    if (vertices) std::memcpy(vertices, m.verts.data(), m.verts.size() * sizeof(double));
    if (cell_vertices) std::memcpy(cell_vertices, m.cells.data(), m.cells.size() * sizeof(int32_t));
    return PFEM2GPU_OK;
}

extern "C" const char* pfem2gpu_read_unv_error(void) { return unv_error.c_str(); }
