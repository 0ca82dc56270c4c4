// fold3d_io.cpp -- writing a host field to files.
//
// fold3d_write_text is the reference's error-checking dump
// (Stencil-OpenACC/AN_ISO_1_OpenACC.c:1244-1260): "%f\n" per value, i
// outermost, k innermost, every cell of the field (ghosts included).  Lines
// are formatted in parallel with the C library's snprintf and written in
// order, so the file is the same bytes as the reference's.
//
// fold3d_write_vtk writes what the reference's Write_VTK_Structured_Grid
// (:1098-1135) sets out to (its loops are commented out, so it writes headers
// only): a legacy VTK STRUCTURED_POINTS file with the travel times as binary
// big-endian doubles, x fastest (the field's own order).
//
// fold3d_write_raw writes a 64-byte header (magic "FOLD3DRW", version, nx,
// ny, nz as int32, dx, dy, dz as double, padding) and then the whole field
// as little-endian doubles in the field layout.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "fold3d_internal.h"
#include "fold3dpmm.h"

namespace {

struct File {
    FILE *f;
    explicit File(const char *path) : f(std::fopen(path, "wb")) {}
    ~File()
    {
        if (f) std::fclose(f);
    }
};

bool put(FILE *f, const void *p, size_t n) { return std::fwrite(p, 1, n, f) == n; }

}  // namespace

extern "C" {

static int write_text(const char *path, const double *T, const fold3d_grid *g);
static int write_vtk(const char *path, const double *T, const fold3d_grid *g, int ghosts);

// Host exceptions (memory for the formatted lines, the row buffer, threads)
// become status codes instead of crossing the C boundary.
int fold3d_write_text(const char *path, const double *T, const fold3d_grid *g)
{
    try {
        return write_text(path, T, g);
    } catch (const std::bad_alloc &) {
        return FOLD3D_ERR_NOMEM;
    } catch (...) {
        return FOLD3D_ERR_INVALID;
    }
}

int fold3d_write_vtk(const char *path, const double *T, const fold3d_grid *g, int ghosts)
{
    try {
        return write_vtk(path, T, g, ghosts);
    } catch (const std::bad_alloc &) {
        return FOLD3D_ERR_NOMEM;
    } catch (...) {
        return FOLD3D_ERR_INVALID;
    }
}

static int write_text(const char *path, const double *T, const fold3d_grid *g)
{
    if (!path || !T || !g || g->nx < 1 || g->ny < 1 || g->nz < 1) return FOLD3D_ERR_INVALID;
    const int px = g->nx + 2, py = g->ny + 2, pz = g->nz + 2;
    const long long sy = px, sz = (long long)px * py;
    File out(path);
    if (!out.f) return FOLD3D_ERR_INVALID;
    const int nth = fold3d::init_threads();
    // one i-plane (all j, k) per task, formatted by nth threads, written in order
    const int batch = std::max(1, nth);
    std::vector<std::string> text(batch);
    std::atomic<bool> failed(false);  // a worker that ran out of memory (it must not throw)
    for (int i0 = 0; i0 < px; i0 += batch) {
        const int i1 = std::min(px, i0 + batch);
        fold3d::host_parallel_for(i0, i1, nth, [&](int i) {
            try {
                std::string &s = text[i - i0];
                s.clear();
                char buf[512];
                for (int j = 0; j < py; ++j)
                    for (int k = 0; k < pz; ++k) {
                        const int n = std::snprintf(buf, sizeof buf, "%f\n", T[i + sy * j + sz * k]);
                        s.append(buf, (size_t)n);
                    }
            } catch (...) {
                failed = true;
            }
        });
        if (failed) return FOLD3D_ERR_NOMEM;
        for (int i = i0; i < i1; ++i)
            if (!put(out.f, text[i - i0].data(), text[i - i0].size())) return FOLD3D_ERR_INVALID;
    }
    return FOLD3D_OK;
}

static int write_vtk(const char *path, const double *T, const fold3d_grid *g, int ghosts)
{
    if (!path || !T || !g || g->nx < 1 || g->ny < 1 || g->nz < 1) return FOLD3D_ERR_INVALID;
    const int px = g->nx + 2, py = g->ny + 2;
    const int e = ghosts ? 0 : 1;  // first index written
    const int nx = g->nx + (ghosts ? 2 : 0), ny = g->ny + (ghosts ? 2 : 0), nz = g->nz + (ghosts ? 2 : 0);
    File out(path);
    if (!out.f) return FOLD3D_ERR_INVALID;
    char head[1024];
    const long long npts = (long long)nx * ny * nz;
    const int n = std::snprintf(head, sizeof head,
                                "# vtk DataFile Version 3.0\n"
                                "fold3dpmm travel times\n"
                                "BINARY\n"
                                "DATASET STRUCTURED_POINTS\n"
                                "DIMENSIONS %d %d %d\n"
                                "ORIGIN %.17g %.17g %.17g\n"
                                "SPACING %.17g %.17g %.17g\n"
                                "POINT_DATA %lld\n"
                                "SCALARS traveltime double 1\n"
                                "LOOKUP_TABLE default\n",
                                nx, ny, nz, (e - 1) * g->dx, (e - 1) * g->dy, (e - 1) * g->dz, g->dx, g->dy, g->dz,
                                npts);
    if (!put(out.f, head, (size_t)n)) return FOLD3D_ERR_INVALID;
    std::vector<uint64_t> row(nx);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            const double *src = T + (e + (long long)px * ((j + e) + (long long)py * (k + e)));
            for (int i = 0; i < nx; ++i) {
                uint64_t b;
                std::memcpy(&b, src + i, 8);
                row[i] = __builtin_bswap64(b);  // VTK binary is big-endian
            }
            if (!put(out.f, row.data(), (size_t)nx * 8)) return FOLD3D_ERR_INVALID;
        }
    if (!put(out.f, "\n", 1)) return FOLD3D_ERR_INVALID;
    return FOLD3D_OK;
}

int fold3d_write_raw(const char *path, const double *T, const fold3d_grid *g)
{
    if (!path || !T || !g || g->nx < 1 || g->ny < 1 || g->nz < 1) return FOLD3D_ERR_INVALID;
    File out(path);
    if (!out.f) return FOLD3D_ERR_INVALID;
    unsigned char head[64];
    std::memset(head, 0, sizeof head);
    std::memcpy(head, "FOLD3DRW", 8);
    const int32_t v[4] = {1, g->nx, g->ny, g->nz};
    const double h[3] = {g->dx, g->dy, g->dz};
    std::memcpy(head + 8, v, sizeof v);
    std::memcpy(head + 24, h, sizeof h);
    if (!put(out.f, head, sizeof head)) return FOLD3D_ERR_INVALID;
    const size_t cells = (size_t)(g->nx + 2) * (g->ny + 2) * (g->nz + 2);
    if (!put(out.f, T, cells * sizeof(double))) return FOLD3D_ERR_INVALID;
    return FOLD3D_OK;
}

}  // extern "C"
