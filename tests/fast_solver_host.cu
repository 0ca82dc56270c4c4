// Host build of the library's point update (csrc/fold3d_fast.cuh) with its
// direction tables (csrc/fold3d_tables.cpp), swept over a field in the
// reference driver's order (Stencil-OpenACC/AN_ISO_1_OpenACC.c:1195-1236).
// Every operation of the update is an IEEE double +, -, *, /, sqrt or fma
// with no contraction on either side, so the host build computes the bits the
// kernels compute; tests/test_solver_host.py runs it against the oracle.
// Test code only: the library has no host solver.
#include <algorithm>
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
// bounds only (the tables of fold3d_solve_noalloc), 0 no bounds at all; plus
// 4: with the gradient bins of the searched bounds (as WAVEFRONT solves).
extern "C" int fast_host_sweeps(double *T, int nx, int ny, int nz, double dx, double dy, double dz, double F,
                                double a0, double a1, double a2, int sweeps, int skip)
{
    const int n[3] = {nx, ny, nz};
    const int64_t stride[3] = {1, (int64_t)nx + 2, ((int64_t)nx + 2) * (ny + 2)};
    const double h[3] = {dx, dy, dz}, a[3] = {a0, a1, a2};
    const bool bins = (skip & 4) != 0;
    skip &= 3;
    DirTable tabs[6];
    static DirBins dbins[6];
    for (int dir = 0; dir < 6; ++dir) {
        build_dir_table(host_frame(dir, h, F, a), tabs[dir], skip != 2, bins ? &dbins[dir] : nullptr);
        if (bins) attach_dir_bins(tabs[dir], &dbins[dir]);
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

// The gradient bins' bounds against the increments the bodies accept at
// sampled gradients inside each bin (fold3d_fast.cuh, 5.): returns how many
// samples were accepted below their bin's bound (0 when every bound holds),
// and the number of accepted samples in *checked.
extern "C" long long fast_host_check_bins(double dx, double dy, double dz, double F, double a0, double a1, double a2,
                                          long long *checked)
{
    const double h[3] = {dx, dy, dz}, a[3] = {a0, a1, a2};
    long long bad = 0, n = 0;
    auto edge_incr = [](const EdgeK &k, double Fs, double d) {
        const double c0 = 1.0 - d * k.ax, Q = k.g * (c0 * c0 - d * d * k.ga);
        if (!(Q > 0.0)) return HUGE_VAL;
        const double c = (-k.az * c0 + std::sqrt(Q)) / k.ga, D = k.hz * c - std::min(0.0, d * k.hx);
        if (!(D > 0.0)) return HUGE_VAL;
        const double G = std::sqrt((d * d + c * c) * Fs * Fs / k.g), xe = -k.hz * (d + k.ax * G) / (c + k.az * G);
        return (0.0 < xe && xe < k.hx) ? D : HUGE_VAL;
    };
    auto check_edge = [&](const EdgeK &k, double Fs) {
        if (!k.bins) return;
        const double lo = k.blo, w = 1.0 / k.binv;
        for (int i = 0; i < kEdgeBins; ++i)
            for (int j = 0; j <= 64; ++j) {
                const double d = lo + (i + j / 64.0) * w;
                if (k.early && d > 0.0) continue;
                const double D = edge_incr(k, Fs, d);
                if (D == HUGE_VAL) continue;
                ++n;
                if (D < (double)k.bins[i]) ++bad;
            }
    };
    for (int dir = 0; dir < 6; ++dir) {
        DirTable t;
        static DirBins b;
        build_dir_table(host_frame(dir, h, F, a), t, true, &b);
        attach_dir_bins(t, &b);
        for (int sd = 0; sd < 2; ++sd) {
            const SideTable &s = t.side[sd];
            for (int k = 0; k < 8; ++k) {
                check_edge(s.edge[k], s.F);
                check_edge(s.surf[k].nest, s.F);
                const SurfK &K = s.surf[k];
                if (!K.bins) continue;
                const double lo = K.blo, w = 1.0 / K.binv;
                for (int i = 0; i < kSurfBins; ++i)
                    for (int j = 0; j < kSurfBins; ++j)
                        for (int p = 0; p <= 8; ++p)
                            for (int q = 0; q <= 8; ++q) {
                                const double gx = lo + (i + p / 8.0) * w, gy = lo + (j + q / 8.0) * w;
                                if ((K.e1 && gx > 0.0) || (K.e2 && gy > 0.0)) continue;
                                const double dd = gx * gx + gy * gy, al = 1.0 - K.ax * gx - K.ay * gy;
                                const double qq = al * al - dd * s.g;
                                if (!(qq > 0.0)) continue;
                                const double al2 = (-s.az * al + s.F * std::sqrt(qq)) / s.g;
                                const double D = s.hz * al2 - std::min(0.0, std::min(gx * K.hx, gx * K.hx + gy * K.hy));
                                if (!(D > 0.0)) continue;
                                const double r = std::sqrt(dd + al2 * al2), m = -s.hz / (s.F * al2 + s.az * r);
                                const double xe = m * (s.F * gx + K.ax * r), ye = m * (s.F * gy + K.ay * r);
                                if (!(0.0 <= std::min(xe, ye) && ye * K.hx <= xe * K.hy && xe <= K.hx)) continue;
                                ++n;
                                if (D < (double)K.bins[i * kSurfBins + j]) ++bad;
                            }
            }
        }
    }
    *checked = n;
    return bad;
}
