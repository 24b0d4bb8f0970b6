// aw_output.cu — binary legacy-VTK writers for inspecting a grid, resampled fields and particles.
//
// The reference writes the same three datasets as ASCII text (vtx_visualization.cuh:64-218:
// exportUniformPressure_VTK, exportMultigrid_VTK, exportParticles_VTK).  These write the legacy
// format's BINARY encoding: the same header lines, then the arrays as big-endian 32-bit words.
// Host code only; the dense fields come from aw_resample_cells / aw_resample_velocity.
#include <cstdio>
#include <cstring>
#include <vector>

#include "aw_internal.cuh"

namespace aw {
namespace {

struct OutFile {
    FILE* f = nullptr;
    explicit OutFile(const char* path) : f(std::fopen(path, "wb")) {}
    ~OutFile() {
        if (f) std::fclose(f);
    }
    bool close() {
        bool ok = f && std::fclose(f) == 0;
        f = nullptr;
        return ok;
    }
};

// n 32-bit words (float or int32) written big-endian, in chunks
bool write_be32(FILE* f, const void* data, size_t n) {
    const uint32_t* w = (const uint32_t*)data;
    std::vector<uint32_t> buf(std::min<size_t>(n, (size_t)1 << 16));
    for (size_t i = 0; i < n; i += buf.size()) {
        const size_t m = std::min(buf.size(), n - i);
        for (size_t k = 0; k < m; ++k) buf[k] = __builtin_bswap32(w[i + k]);
        if (std::fwrite(buf.data(), sizeof(uint32_t), m, f) != m) return false;
    }
    return std::fputc('\n', f) != EOF;
}

bool valid_name(const char* s) {
    if (!s || !*s || std::strlen(s) > 64) return false;
    for (const char* c = s; *c; ++c)
        if (*c <= ' ' || *c > '~') return false;
    return true;
}

aw_status io_error(const char* path) { return set_error(AW_ERR_IO, "could not write %s", path); }

}  // namespace
}  // namespace aw

using namespace aw;

extern "C" aw_status aw_vtk_write_structured_points(const char* path, const int32_t dims[3], const float origin[3],
                                                    const float spacing[3], const char* name, int32_t ncomp,
                                                    const float* h_data) {
    AW_CHECK_ARG(path && dims && origin && spacing && h_data, "null argument");
    AW_CHECK_ARG(dims[0] > 0 && dims[1] > 0 && dims[2] > 0, "dims must be positive");
    AW_CHECK_ARG(ncomp == 1 || ncomp == 3, "ncomp must be 1 (scalars) or 3 (vectors)");
    AW_CHECK_ARG(valid_name(name), "name must be 1-64 printable characters without spaces");
    const size_t n = (size_t)dims[0] * dims[1] * dims[2];
    OutFile o(path);
    if (!o.f) return io_error(path);
    std::fprintf(o.f, "# vtk DataFile Version 3.0\nAnitoWave dense resample\nBINARY\nDATASET STRUCTURED_POINTS\n");
    std::fprintf(o.f, "DIMENSIONS %d %d %d\n", dims[0], dims[1], dims[2]);
    std::fprintf(o.f, "ORIGIN %.9g %.9g %.9g\n", origin[0], origin[1], origin[2]);
    std::fprintf(o.f, "SPACING %.9g %.9g %.9g\n", spacing[0], spacing[1], spacing[2]);
    std::fprintf(o.f, "POINT_DATA %zu\n", n);
    if (ncomp == 1) std::fprintf(o.f, "SCALARS %s float 1\nLOOKUP_TABLE default\n", name);
    else std::fprintf(o.f, "VECTORS %s float\n", name);
    if (!write_be32(o.f, h_data, n * ncomp) || !o.close()) return io_error(path);
    return AW_OK;
}

extern "C" aw_status aw_vtk_write_blocks(aw_msbg* g, const char* path) {
    AW_CHECK_ARG(g && path, "null argument");
    const MsbgState& G = g->st;
    const Geo& geo = G.geo;
    const int nb = G.nb;
    std::vector<uint32_t> lv(nb);
    AW_CUDA(cudaMemcpy(lv.data(), G.level.p, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    std::vector<float> pts((size_t)nb * 24);
    std::vector<int32_t> cells((size_t)nb * 9), types(nb, 12), level(nb);
    static const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                     {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int b = 0; b < nb; ++b) {
        int c[3];
        bcoord(geo, b, c);
        for (int k = 0; k < 8; ++k)
            for (int a = 0; a < 3; ++a)
                pts[(size_t)b * 24 + 3 * k + a] = geo.dmin[a] + (float)(c[a] + corner[k][a]) * geo.bs;
        cells[(size_t)b * 9] = 8;
        for (int k = 0; k < 8; ++k) cells[(size_t)b * 9 + 1 + k] = 8 * b + k;
        level[b] = (int)lv[b] < geo.L ? (int32_t)lv[b] : -1;
    }
    OutFile o(path);
    if (!o.f) return io_error(path);
    std::fprintf(o.f, "# vtk DataFile Version 3.0\nAnitoWave MSBG blocks\nBINARY\nDATASET UNSTRUCTURED_GRID\n");
    std::fprintf(o.f, "POINTS %d float\n", 8 * nb);
    bool ok = write_be32(o.f, pts.data(), pts.size());
    std::fprintf(o.f, "CELLS %d %d\n", nb, 9 * nb);
    ok = ok && write_be32(o.f, cells.data(), cells.size());
    std::fprintf(o.f, "CELL_TYPES %d\n", nb);
    ok = ok && write_be32(o.f, types.data(), types.size());
    std::fprintf(o.f, "CELL_DATA %d\nSCALARS refineLevel int 1\nLOOKUP_TABLE default\n", nb);
    ok = ok && write_be32(o.f, level.data(), level.size());
    if (!ok || !o.close()) return io_error(path);
    return AW_OK;
}

extern "C" aw_status aw_vtk_write_particles(const char* path, const float* h_pos, int64_t n, const char* name,
                                            const float* h_scalar) {
    AW_CHECK_ARG(path && (h_pos || n == 0) && n >= 0 && n < (int64_t)0x7FFFFFFF / 2, "bad argument");
    AW_CHECK_ARG(!h_scalar || valid_name(name), "name must be 1-64 printable characters without spaces");
    OutFile o(path);
    if (!o.f) return io_error(path);
    std::fprintf(o.f, "# vtk DataFile Version 3.0\nAnitoWave particles\nBINARY\nDATASET POLYDATA\n");
    std::fprintf(o.f, "POINTS %lld float\n", (long long)n);
    bool ok = write_be32(o.f, h_pos, (size_t)n * 3);
    std::vector<int32_t> verts((size_t)n * 2);
    for (int64_t i = 0; i < n; ++i) {
        verts[2 * i] = 1;
        verts[2 * i + 1] = (int32_t)i;
    }
    std::fprintf(o.f, "VERTICES %lld %lld\n", (long long)n, (long long)(2 * n));
    ok = ok && write_be32(o.f, verts.data(), verts.size());
    if (h_scalar) {
        std::fprintf(o.f, "POINT_DATA %lld\nSCALARS %s float 1\nLOOKUP_TABLE default\n", (long long)n, name);
        ok = ok && write_be32(o.f, h_scalar, (size_t)n);
    }
    if (!ok || !o.close()) return io_error(path);
    return AW_OK;
}
