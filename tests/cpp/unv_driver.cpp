// Reads a UNV file with pfem2gpu::read_unv (include/pfem2gpu_handler.hpp)
// and writes the mesh as raw arrays: int64 dim, n_verts, n_cells, n_dofs,
// then vertices (f64) and cell_vertices, cell_dofs (i32).  Exit status 3 on
// a reader error (its message on stderr).
#include <cstdio>

#include "pfem2gpu_handler.hpp"

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    try {
        const pfem2gpu::Mesh m = pfem2gpu::read_unv(argv[1], 0);
        FILE* f = std::fopen(argv[2], "wb");
        if (!f) return 2;
        const int64_t dim = m.n_cells ? (int64_t)(m.cell_vertices.size() / m.n_cells == 8 ? 3 : 2) : 0;
        const int64_t hd[4] = {dim, m.n_verts, m.n_cells, m.n_dofs};
        std::fwrite(hd, sizeof hd, 1, f);
        std::fwrite(m.vertices.data(), sizeof(double), m.vertices.size(), f);
        std::fwrite(m.cell_vertices.data(), sizeof(int32_t), m.cell_vertices.size(), f);
        std::fwrite(m.cell_dofs.data(), sizeof(int32_t), m.cell_dofs.size(), f);
        std::fclose(f);
    } catch (const pfem2gpu::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 3;
    }
    return 0;
}
