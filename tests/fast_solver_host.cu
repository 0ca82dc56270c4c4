// Host build of the library's point update (csrc/fold3d_fast.cuh) with its
// direction tables (csrc/fold3d_tables.cpp), swept over a field in the
// reference driver's order (Stencil-OpenACC/AN_ISO_1_OpenACC.c:1195-1236).
// Every operation of the update is an IEEE double +, -, *, /, sqrt or fma
// with no contraction on either side, so the host build computes the bits the
// kernels compute; tests/test_solver_host.py runs it against the oracle.
// Test code only: the library has no host solver.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "fold3d_fast.cuh"
#include "fold3d_internal.h"

using namespace fold3d;

namespace {

// axis normal to the planes, sign of the target (src + sg), axis and sign of
// the local x and y neighbours; one row per reference sweep function
struct HostDir {
    int nrm, sg, xa, xs, ya, ys;
};
const HostDir kHostDirs[6] = {
    {0, +1, 2, +1, 1, +1}, {0, -1, 2, -1, 1, -1}, {2, +1, 1, +1, 0, +1},
    {2, -1, 1, -1, 0, -1}, {1, -1, 0, -1, 2, -1}, {1, +1, 0, +1, 2, +1},
};

// The local frame of direction dir, as the library forms it: drift permuted
// and signed per direction, the reference driver's diagonals (:1158-1160).
LocalFrameH host_frame(int dir, const double h[3], double F, const double a[3])
{
    const HostDir &d = kHostDirs[dir];
    LocalFrameH L;
    L.F = F;
    L.ax = d.xs * a[d.xa];
    L.ay = d.ys * a[d.ya];
    L.az = d.sg * a[d.nrm];
    L.hz = h[d.nrm];
    L.hx = h[d.xa];
    L.hy = h[d.ya];
    L.hxy = std::sqrt(L.hx * L.hx + L.hy * L.hy);
    L.hxz = std::sqrt(L.hx * L.hx + L.hz * L.hz);
    L.hyz = std::sqrt(L.hy * L.hy + L.hz * L.hz);
    return L;
}

void clear_bounds(SideTable &t)
{
    for (int k = 0; k < 8; ++k) {
        t.surf[k].B = 0.0;
        t.edge[k].B = 0.0;
        t.surf[k].nest.B = 0.0;
    }
}

}  // namespace

// Runs `sweeps` sweeps on T ((nz+2)(ny+2)(nx+2) doubles, x fastest).  skip:
// 1 the tables as solves build them (searched bounds), 2 the closed-form
// bounds only (the tables of fold3d_solve_noalloc), 0 no bounds at all.
extern "C" int fast_host_sweeps(double *T, int nx, int ny, int nz, double dx, double dy, double dz, double F,
                                double a0, double a1, double a2, int sweeps, int skip)
{
    const int n[3] = {nx, ny, nz};
    const int64_t stride[3] = {1, (int64_t)nx + 2, ((int64_t)nx + 2) * (ny + 2)};
    const double h[3] = {dx, dy, dz}, a[3] = {a0, a1, a2};
    DirTable tabs[6];
    for (int dir = 0; dir < 6; ++dir) {
        build_dir_table(host_frame(dir, h, F, a), tabs[dir], skip != 2);
        if (!skip) {
            clear_bounds(tabs[dir].side[0]);
            clear_bounds(tabs[dir].side[1]);
        }
    }
    for (int s = 0; s < sweeps; ++s)
        for (int dir = 0; dir < 6; ++dir) {
            const HostDir &d = kHostDirs[dir];
            const int u = (d.nrm == 0) ? 1 : 0, v = (d.nrm == 2) ? 1 : 2;
            const int64_t sx = d.xs * stride[d.xa], sy = d.ys * stride[d.ya], sn = stride[d.nrm];
            const int nn = n[d.nrm];
            for (int q = 0; q < nn - 1; ++q) {
                const int src = d.sg > 0 ? 1 + q : nn - q;
                for (int b = 1; b <= n[v]; ++b)
                    for (int c = 1; c <= n[u]; ++c) {
                        const int64_t si = (int64_t)src * sn + c * stride[u] + b * stride[v];
                        const int64_t ti = si + d.sg * sn;
                        const double *p = T + si;
                        T[ti] = point_update_fast(T[ti], std::fabs(p[0]), std::fabs(p[sx]), std::fabs(p[sy]),
                                                  std::fabs(p[-sx]), std::fabs(p[-sy]), std::fabs(p[sx + sy]),
                                                  std::fabs(p[sx - sy]), std::fabs(p[-sx + sy]),
                                                  std::fabs(p[-sx - sy]), &tabs[dir]);
                    }
            }
        }
    return 0;
}

// The skip bounds of every direction and side: 24 values at
// out[24 (2 dir + side)]: the eight FoldSurf3Points calls' B, the eight
// FoldEdge2Points calls' B, the eight nested edges' B.
extern "C" void fast_host_bounds(double dx, double dy, double dz, double F, double a0, double a1, double a2,
                                 double *out)
{
    const double h[3] = {dx, dy, dz}, a[3] = {a0, a1, a2};
    for (int dir = 0; dir < 6; ++dir) {
        DirTable t;
        build_dir_table(host_frame(dir, h, F, a), t);
        for (int sd = 0; sd < 2; ++sd) {
            double *o = out + 24 * (2 * dir + sd);
            for (int k = 0; k < 8; ++k) {
                o[k] = t.side[sd].surf[k].B;
                o[8 + k] = t.side[sd].edge[k].B;
                o[16 + k] = t.side[sd].surf[k].nest.B;
            }
        }
    }
}
