// fold3d_init.cpp -- source initialisation of a host field.
//
// The implicit-surface initialiser follows ImplicitInitialiser
// (Stencil-OpenACC/Fold3dPMM.c:129-389) with run-time sizes and medium:
//   1. sample the implicit surface on every node (ghosts included) and set
//      T = sign(surface) * MAXT (:137-147);
//   2. for every voxel, find the points where the surface crosses its 12
//      edges (:163-269), and from each crossing, and from blends of it with
//      earlier crossings of the same voxel (:271-383), min-update 44 nearby
//      nodes with the exact homogeneous travel time (updateVoxel / InitNode,
//      :35-112).
// The min-update keeps the node's sign and never changes it, so the final
// field does not depend on the order of the updates.  Step 2 therefore runs
// in parallel over slabs of voxels along i, in two phases (even slabs, then
// odd slabs): a voxel at i writes nodes i-1..i+2, so slabs at least four
// voxels wide that run at the same time never write the same node.
//
// The arithmetic keeps the reference's operand order; this file is compiled
// with -ffp-contract=off, and sin/cos come from the same libm as the
// reference's host build, so the result is bit-identical to it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <thread>
#include <vector>

#include "fold3dpmm.h"

namespace {

constexpr double kMaxT = 10e15 * 1.0;  // Fold3dPMM.h:6

inline double side(double a) { return (a > 0) ? 1.0 : -1.0; }  // sign(), 0 -> -1

// Fold3dPMM.c:9-26
double exact_time(double F, double ax, double ay, double az, double x, double y, double z)
{
    double xsq = x * x + y * y + z * z;
    double adotx = ax * x + ay * y + az * z;
    double q = (F * F - (ax * ax + ay * ay + az * az)) * xsq + adotx * adotx;
    if (q > 0.0) {
        q = adotx + std::sqrt(q);
        if (q > 0.0) return xsq / q;
    }
    return 1.0 * kMaxT;
}

// Fold3dPMM.c:29-33
double surface(double x, double y, double z)
{
    return 5.0 + (std::sin(x) + std::cos(y + x) + std::sin(x + y + z)) * 0.4 - z +
           (x - 5.0) * (y - 5.0) * (z - 5) / 55.0;
}

// surface() with sin(x) and cos(y + x) given (the same values, computed once
// per node column and row of the grid).
inline double surface_tab(double x, double y, double z, double sin_x, double cos_yx)
{
    return 5.0 + (sin_x + cos_yx + std::sin(x + y + z)) * 0.4 - z + (x - 5.0) * (y - 5.0) * (z - 5) / 55.0;
}

// Node updates of one seeding point (updateVoxel, Fold3dPMM.c:62-110, in
// order): position shift in multiples of the spacing (+1, -1 or -2), then the
// node offset.  Two rows keep the reference's position/index mismatch
// (:82 shifts y by +1 but writes node j; :86 shifts x by -1, y by -2 but
// writes node i+2, j).
struct NodeStep {
    signed char px, py, pz, di, dj, dk;
};
constexpr NodeStep kSteps[44] = {
    {0, 0, 0, 0, 0, 0},     {-1, 0, 0, 1, 0, 0},    {0, -1, 0, 0, 1, 0},    {0, 0, -1, 0, 0, 1},
    {-1, -1, 0, 1, 1, 0},   {-1, 0, -1, 1, 0, 1},   {0, -1, -1, 0, 1, 1},   {-1, -1, -1, 1, 1, 1},
    {1, 0, 0, -1, 0, 0},    {1, -1, 0, -1, 1, 0},   {1, 0, -1, -1, 0, 1},   {1, -1, -1, -1, 1, 1},
    {-2, 0, 0, 2, 0, 0},    {-2, -1, 0, 2, 1, 0},   {-2, 0, -1, 2, 0, 1},   {-2, -1, -1, 2, 1, 1},
    {0, 1, 0, 0, -1, 0},    {-1, 1, 0, 1, 0, 0},    {0, 1, -1, 0, -1, 1},   {-1, 1, -1, 1, -1, 1},
    {0, -2, 0, 0, 2, 0},    {-1, -2, 0, 2, 0, 0},   {0, -2, -1, 0, 2, 1},   {-1, -2, -1, 1, 2, 1},
    {0, 0, 1, 0, 0, -1},    {-1, 0, 1, 1, 0, -1},   {0, -1, 1, 0, 1, -1},   {-1, -1, 1, 1, 1, -1},
    {0, 0, -2, 0, 0, 2},    {-1, 0, -2, 1, 0, 2},   {0, -1, -2, 0, 1, 2},   {-1, -1, -2, 1, 1, 2},
    {0, 1, 1, 0, -1, -1},   {1, 0, 1, -1, 0, -1},   {1, 1, 0, -1, -1, 0},   {0, -2, -2, 0, 2, 2},
    {-2, 0, -2, 2, 0, 2},   {-2, -2, 0, 2, 2, 0},   {-1, 1, 1, 1, -1, -1},  {1, -1, 1, -1, 1, -1},
    {1, 1, -1, -1, -1, 1},  {-1, -2, -2, 1, 2, 2},  {-2, -1, -2, 2, 1, 2},  {-2, -2, -1, 2, 2, 1},
};

inline double shifted(double p, int m, double h)
{
    switch (m) {
    case 0: return p;
    case 1: return p + h;
    case -1: return p - h;
    default: return p - 2 * h;
    }
}

// Blends of crossing l with earlier crossings (:274-382), in order.  A blend
// is (sum of w[t] * P[l - off[t]]) / div; its z coordinate takes the y
// coordinate of term `zy` instead of the z coordinate (the reference's
// ypos[l-2] / ypos[l-3] in the zp lines, :309-379), or -1 for none.
struct Blend {
    int minl, div, n, off[3], w[3], zy;
};
constexpr Blend kBlends[] = {
    {1, 3, 2, {0, 1, 0}, {2, 1, 0}, -1}, {1, 3, 2, {0, 1, 0}, {1, 2, 0}, -1},
    {2, 3, 2, {0, 2, 0}, {2, 1, 0}, -1}, {2, 3, 2, {0, 2, 0}, {1, 2, 0}, -1},
    {3, 3, 2, {0, 3, 0}, {2, 1, 0}, -1}, {3, 3, 2, {0, 3, 0}, {1, 2, 0}, -1},
    {3, 3, 3, {0, 2, 3}, {1, 1, 1}, 1},  {3, 4, 3, {0, 2, 3}, {2, 1, 1}, 1},
    {3, 4, 3, {0, 2, 3}, {1, 2, 1}, 1},  {3, 4, 3, {0, 2, 3}, {1, 1, 2}, 1},
    {4, 3, 2, {0, 4, 0}, {2, 1, 0}, -1}, {4, 3, 2, {0, 4, 0}, {1, 2, 0}, -1},
    {4, 3, 3, {0, 2, 3}, {1, 1, 1}, 1},  {4, 3, 3, {0, 2, 4}, {1, 1, 1}, 1},
    {4, 3, 3, {0, 3, 4}, {1, 1, 1}, 1},  {5, 3, 2, {0, 5, 0}, {2, 1, 0}, -1},
    {5, 3, 2, {0, 5, 0}, {1, 2, 0}, -1}, {5, 3, 3, {0, 2, 3}, {1, 1, 1}, 1},
    {5, 3, 3, {0, 2, 4}, {1, 1, 1}, 1},  {5, 3, 3, {0, 2, 5}, {1, 1, 1}, 1},
    {5, 3, 3, {0, 3, 5}, {1, 1, 1}, 1},  {5, 3, 3, {0, 3, 4}, {1, 1, 1}, 1},
};

struct Seeder {
    double *T;
    long long sy, sz;
    double F, a[3];
    double h[3];

    // InitNode, Fold3dPMM.c:35-54
    void node(double x, double y, double z, int i, int j, int k) const
    {
        double *t = T + i + sy * j + sz * k;
        double ax = a[0], ay = a[1], az = a[2];
        if (*t < 0.0) {
            ax *= -1;
            ay *= -1;
            az *= -1;
        }
        double tn = exact_time(F, ax, ay, az, -x, -y, -z);
        if (tn < std::fabs(*t)) *t = (side(*t) * 1.0) * tn;
    }

    void voxel(int i, int j, int k, double xp, double yp, double zp) const
    {
        for (const NodeStep &s : kSteps)
            node(shifted(xp, s.px, h[0]), shifted(yp, s.py, h[1]), shifted(zp, s.pz, h[2]), i + s.di,
                 j + s.dj, k + s.dk);
    }

    void seed_voxel(const double *IF, int i, int j, int k) const
    {
        const long long id = i + sy * j + sz * k;
        const double f = IF[id], fx = IF[id + 1], fy = IF[id + sy], fz = IF[id + sz];
        const double fxy = IF[id + 1 + sy], fzx = IF[id + 1 + sz], fzy = IF[id + sy + sz];
        const double fxyz = IF[id + 1 + sy + sz];
        // Skip voxels no edge of which can report a crossing.  An edge (a, b)
        // reports one when p = h*a/(a-b) lands in [0, h].  For a and b of the
        // same strict sign that needs a - b to round to a (one value below
        // ~2^-52 of the other); with every corner of one sign and within a
        // factor 2^40 of every other, each p lies strictly outside [0, h].
        {
            const double c[8] = {f, fx, fy, fz, fxy, fzx, fzy, fxyz};
            bool pos = true, neg = true;
            double lo = std::fabs(f), hi = lo;
            for (int q = 0; q < 8; ++q) {
                pos = pos && c[q] > 0.0;
                neg = neg && c[q] < 0.0;
                lo = std::min(lo, std::fabs(c[q]));
                hi = std::max(hi, std::fabs(c[q]));
            }
            if ((pos || neg) && lo > hi * 0x1p-40) return;
        }
        const double hx = h[0], hy = h[1], hz = h[2];
        double P[12][3];
        int np = 0;
        auto cross = [&](double p, double lim, double x, double y, double z) {
            if (0.0 <= p && p <= lim) {
                P[np][0] = x;
                P[np][1] = y;
                P[np][2] = z;
                ++np;
            }
        };
        double p;
        p = hx * f / (f - fx);       cross(p, hx, p, 0.0, 0.0);
        p = hx * fz / (fz - fzx);    cross(p, hx, p, 0.0, hz);
        p = hx * fy / (fy - fxy);    cross(p, hx, p, hy, 0.0);
        p = hx * fzy / (fzy - fxyz); cross(p, hx, p, hy, hz);
        p = hy * f / (f - fy);       cross(p, hy, 0.0, p, 0.0);
        p = hy * fz / (fz - fzy);    cross(p, hy, 0.0, p, hz);
        p = hy * fx / (fx - fxy);    cross(p, hy, hx, p, 0.0);
        p = hy * fzx / (fzx - fxyz); cross(p, hy, hx, p, hz);
        p = hz * f / (f - fz);       cross(p, hz, 0.0, 0.0, p);
        p = hz * fxy / (fxy - fxyz); cross(p, hz, hx, hy, p);
        p = hz * fx / (fx - fzx);    cross(p, hz, hx, 0.0, p);
        p = hz * fy / (fy - fzy);    cross(p, hz, 0.0, hy, p);
        for (int l = 0; l < np; ++l) {
            voxel(i, j, k, P[l][0], P[l][1], P[l][2]);
            for (const Blend &b : kBlends) {
                if (l < b.minl) continue;
                double c[3];
                for (int ax = 0; ax < 3; ++ax) {
                    double acc = 0.0;
                    for (int t = 0; t < b.n; ++t) {
                        const int src_ax = (ax == 2 && t == b.zy) ? 1 : ax;
                        const double term = b.w[t] * P[l - b.off[t]][src_ax];
                        acc = (t == 0) ? term : acc + term;
                    }
                    c[ax] = acc / b.div;
                }
                voxel(i, j, k, c[0], c[1], c[2]);
            }
        }
    }
};

int host_threads()
{
    const char *e = std::getenv("FOLD3D_HOST_THREADS");
    int n = e ? std::atoi(e) : 0;
    if (n <= 0) n = (int)std::thread::hardware_concurrency();
    return std::max(1, std::min(n, 256));
}

template <class Fn>
void parallel_for(int lo, int hi, int nthreads, Fn fn)
{
    const int n = hi - lo;
    if (n <= 0) return;
    nthreads = std::max(1, std::min(nthreads, n));
    if (nthreads == 1) {
        for (int i = lo; i < hi; ++i) fn(i);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nthreads);
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([=]() {
            const int a = lo + (int)((long long)n * t / nthreads);
            const int b = lo + (int)((long long)n * (t + 1) / nthreads);
            for (int i = a; i < b; ++i) fn(i);
        });
    for (auto &x : th) x.join();
}

}  // namespace

extern "C" {

double InitFoldFromPoint(double F, double ax, double ay, double az, double x, double y, double z)
{
    return exact_time(F, ax, ay, az, x, y, z);
}

double ImpSurfF(double x, double y, double z) { return surface(x, y, z); }

double fold3d_exact_time(const fold3d_medium *m, double x, double y, double z)
{
    if (!m) return kMaxT;
    return exact_time(m->F, m->ax, m->ay, m->az, x, y, z);
}

int fold3d_init_implicit(double *T, const fold3d_grid *g, const fold3d_medium *m)
{
    if (!T || !g || !m) return FOLD3D_ERR_INVALID;
    if (g->nx < 2 || g->ny < 2 || g->nz < 2) return FOLD3D_ERR_INVALID;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const long long sy = nx + 2, sz = (long long)(nx + 2) * (ny + 2);
    const size_t cells = (size_t)sz * (nz + 2);
    std::vector<double> IF;
    try {
        IF.resize(cells);
    } catch (...) {
        return FOLD3D_ERR_NOMEM;
    }
    const int nth = host_threads();
    const double hx = g->dx, hy = g->dy, hz = g->dz;
    // :137-147, node coordinates from x/y/z (:115-126)
    std::vector<double> sin_x, cos_yx;
    try {
        sin_x.resize(nx + 2);
        cos_yx.resize((size_t)sy * (ny + 2));
    } catch (...) {
        return FOLD3D_ERR_NOMEM;
    }
    for (int i = 0; i < nx + 2; ++i) sin_x[i] = std::sin((i - 1) * hx + 0.);
    parallel_for(0, ny + 2, nth, [&](int j) {
        const double y = (j - 1) * hy + 0.;
        for (int i = 0; i < nx + 2; ++i) cos_yx[(size_t)j * sy + i] = std::cos(y + ((i - 1) * hx + 0.));
    });
    parallel_for(0, nz + 2, nth, [&](int k) {
        const double z = (k - 1) * hz + 0.;
        for (int j = 0; j < ny + 2; ++j) {
            const double y = (j - 1) * hy + 0.;
            for (int i = 0; i < nx + 2; ++i) {
                const long long id = i + sy * j + sz * k;
                IF[id] = surface_tab((i - 1) * hx + 0., y, z, sin_x[i], cos_yx[(size_t)j * sy + i]);
                T[id] = (side(IF[id]) * 1.0) * kMaxT;
            }
        }
    });
    Seeder s{T, sy, sz, m->F, {m->ax, m->ay, m->az}, {hx, hy, hz}};
    // Voxels i = 1..nx-1 in slabs of >= 4 (the surface crosses every slab,
    // which balances the threads), even slabs then odd slabs: a voxel
    // min-updates nodes within 2 cells of it, so slabs of one phase never
    // touch the same node, and min-updates commute.  x innermost.
    const int nvox = nx - 1;
    int width = std::max(4, (nvox + 2 * nth - 1) / (2 * nth));
    const int nslabs = (nvox + width - 1) / width;
    for (int phase = 0; phase < 2; ++phase) {
        const int count = (nslabs - phase + 1) / 2;
        parallel_for(0, count, nth, [&](int q) {
            const int slab = 2 * q + phase;
            const int i0 = 1 + slab * width, i1 = std::min(nx - 1, i0 + width - 1);
            for (int k = 1; k < nz; ++k)
                for (int j = 1; j < ny; ++j)
                    for (int i = i0; i <= i1; ++i) s.seed_voxel(IF.data(), i, j, k);
        });
    }
    return FOLD3D_OK;
}

int fold3d_init_point(double *T, const fold3d_grid *g, int si, int sj, int sk)
{
    if (!T || !g) return FOLD3D_ERR_INVALID;
    if (si < 1 || si > g->nx || sj < 1 || sj > g->ny || sk < 1 || sk > g->nz) return FOLD3D_ERR_INVALID;
    const size_t cells = (size_t)(g->nx + 2) * (g->ny + 2) * (g->nz + 2);
    std::fill(T, T + cells, kMaxT);
    T[si + (long long)(g->nx + 2) * (sj + (long long)(g->ny + 2) * sk)] = 0.0;
    return FOLD3D_OK;
}

// Reference signature (Fold3dPMM.h:81-85): the reference medium constants
// (:49-52) and pitch nx+2.
void ImplicitInitialiser(double *T, int nx, int ny, int nz, double dxx, double dyy, double dzz)
{
    const fold3d_grid g = {nx, ny, nz, dxx, dyy, dzz};
    const fold3d_medium m = {1.1, -0.35, 0.4, 0.7};
    fold3d_init_implicit(T, &g, &m);
}

}  // extern "C"
