// Host build of the library's elliptical point update
// (csrc/fold3d_ellip.cuh: ell_local, ell_skip_bound, point_update_ellip),
// swept over a field in the reference driver's direction order
// (Stencil-OpenACC/AN_ISO_1_OpenACC.c:1195-1236) with the winner record the
// kernels keep.  The solver uses IEEE +, -, *, / and sqrt only, in double or
// in float, with no contraction on either side, so the host build computes the
// bits the kernels compute; tests/test_solver_host.py runs it against the
// oracle's CPU statements.  Test code only: the library has no host solver.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "fold3d_ellip.cuh"

using namespace fold3d;

namespace {

struct HostDir {
    int nrm, sg, xa, xs, ya, ys;
};
const HostDir kHostDirs[6] = {
    {0, +1, 2, +1, 1, +1}, {0, -1, 2, -1, 1, -1}, {2, +1, 1, +1, 0, +1},
    {2, -1, 1, -1, 0, -1}, {1, -1, 0, -1, 2, -1}, {1, +1, 0, +1, 2, +1},
};
constexpr int kCands = 33;

// The direction's metric gather and signs, as the library forms them.
EllipDir host_dir(int dir, const double h[3])
{
    static const int pair[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    const HostDir &d = kHostDirs[dir];
    EllipDir e;
    e.hx = h[d.xa];
    e.hy = h[d.ya];
    e.hz = h[d.nrm];
    e.sxy = d.xs * d.ys;
    e.sxz = d.xs * d.sg;
    e.syz = d.ys * d.sg;
    e.ixx = pair[d.xa][d.xa];
    e.iyy = pair[d.ya][d.ya];
    e.izz = pair[d.nrm][d.nrm];
    e.ixy = pair[d.xa][d.ya];
    e.ixz = pair[d.xa][d.nrm];
    e.iyz = pair[d.ya][d.nrm];
    return e;
}

template <class R>
void sweeps(R *T, unsigned char *W, const float *const *M, int nx, int ny, int nz, const double h[3], int count)
{
    const int n[3] = {nx, ny, nz};
    const int64_t stride[3] = {1, (int64_t)nx + 2, ((int64_t)nx + 2) * (ny + 2)};
    EllipMedium med;
    for (int k = 0; k < 6; ++k) med.m[k] = M[k];
    for (int s = 0; s < count; ++s)
        for (int dir = 0; dir < 6; ++dir) {
            const HostDir &d = kHostDirs[dir];
            const EllipDir D = host_dir(dir, h);
            const int u = (d.nrm == 0) ? 1 : 0, v = (d.nrm == 2) ? 1 : 2;
            const int64_t sx = d.xs * stride[d.xa], sy = d.ys * stride[d.ya], sn = stride[d.nrm];
            const int nn = n[d.nrm];
            for (int q = 0; q < nn - 1; ++q) {
                const int src = d.sg > 0 ? 1 + q : nn - q;
                for (int b = 1; b <= n[v]; ++b)
                    for (int c = 1; c <= n[u]; ++c) {
                        const int64_t si = (int64_t)src * sn + c * stride[u] + b * stride[v];
                        const int64_t ti = si + d.sg * sn;
                        const R *p = T + si;
                        const R nb[8] = {std::fabs(p[sx]),       std::fabs(p[sx + sy]), std::fabs(p[sy]),
                                         std::fabs(p[-sx + sy]), std::fabs(p[-sx]),     std::fabs(p[-sx - sy]),
                                         std::fabs(p[-sy]),      std::fabs(p[sx - sy])};
                        int win;
                        const R told = T[ti];
                        const R tnew = point_update_ellip(told, std::fabs(p[0]), nb, ell_local<R>(med, D, ti), win);
                        if (std::memcmp(&tnew, &told, sizeof(R)) != 0) {
                            W[ti] = (win < 0) ? 0xffu : (unsigned char)(dir * kCands + win);
                            T[ti] = tnew;
                        }
                    }
            }
        }
}

}  // namespace

// `count` sweeps on T ((nz+2)(ny+2)(nx+2) values, x fastest; double when
// f32 == 0, float otherwise) with its winner record W (same layout, bytes);
// M: the six float metric arrays xx xy xz yy yz zz in the field layout.
extern "C" int ellip_host_sweeps(void *T, unsigned char *W, const float *const *M, int nx, int ny, int nz, double dx,
                                 double dy, double dz, int count, int f32)
{
    const double h[3] = {dx, dy, dz};
    if (f32)
        sweeps(static_cast<float *>(T), W, M, nx, ny, nz, h, count);
    else
        sweeps(static_cast<double *>(T), W, M, nx, ny, nz, h, count);
    return 0;
}

// The skip bound the solver uses for one local metric (scaled entries).
extern "C" double ellip_host_bound(double xx, double yy, double zz, double xy, double xz, double yz)
{
    EllipAT<double> A{xx, yy, zz, xy, xz, yz};
    return ell_skip_bound(A);
}
