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
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#include "fold3d_internal.h"
#include "fold3d_seed.h"
#include "fold3dpmm.h"

namespace {

using fold3d_seed::exact_time;
using fold3d_seed::kMaxT;
using fold3d_seed::side;

// Fold3dPMM.c:29-33
double surface(double x, double y, double z)
{
    return 5.0 + (std::sin(x) + std::cos(y + x) + std::sin(x + y + z)) * 0.4 - z +
           (x - 5.0) * (y - 5.0) * (z - 5) / 55.0;
}

// surface() with sin(x), cos(y + x) and sin(x + y + z) given (the same
// values, computed once per node column, row or distinct argument).
inline double surface_tab(double x, double y, double z, double sin_x, double cos_yx, double sin_xyz)
{
    return 5.0 + (sin_x + cos_yx + sin_xyz) * 0.4 - z + (x - 5.0) * (y - 5.0) * (z - 5) / 55.0;
}

constexpr fold3d_seed::NodeStep kSteps[fold3d_seed::kNodeSteps] = FOLD3D_SEED_STEPS;
constexpr fold3d_seed::Blend kBlends[fold3d_seed::kBlendCount] = FOLD3D_SEED_BLENDS;

// InitNode (Fold3dPMM.c:35-54) on the host field.
struct HostNode {
    double *T;
    long long sy, sz;
    double F, a[3];

    void operator()(double x, double y, double z, int i, int j, int k) const
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
    auto range = [=](int t) {
        const int a = lo + (int)((long long)n * t / nthreads);
        const int b = lo + (int)((long long)n * (t + 1) / nthreads);
        for (int i = a; i < b; ++i) fn(i);
    };
    std::vector<std::thread> th;
    int started = 0;
    try {
        th.reserve(nthreads);
        for (; started < nthreads; ++started) th.emplace_back(range, started);
    } catch (...) {  // no more threads: this thread runs the ranges left
    }
    for (int t = started; t < nthreads; ++t) range(t);
    for (auto &x : th) x.join();
}

}  // namespace

namespace fold3d {

bool surface_tables(const fold3d_grid &g, SurfaceTables &t, int nth)
{
    const int nx = g.nx, ny = g.ny;
    const size_t sy = (size_t)nx + 2, pairs = sy * (ny + 2);
    try {
        t.sin_x.resize(sy);
        t.cos_yx.resize(pairs);
        t.sums.clear();
        t.sum_of.clear();
    } catch (...) {
        return false;
    }
    for (int i = 0; i < nx + 2; ++i) t.sin_x[i] = std::sin((i - 1) * g.dx + 0.);
    parallel_for(0, ny + 2, nth, [&](int j) {
        const double y = (j - 1) * g.dy + 0.;
        for (int i = 0; i < nx + 2; ++i) t.cos_yx[(size_t)j * sy + i] = std::cos(y + ((i - 1) * g.dx + 0.));
    });
    // the distinct rounded sums x_i + y_j (compared as bits); kept only when
    // they are at most half of the pairs
    try {
        std::vector<uint64_t> bits(pairs);
        for (int j = 0; j < ny + 2; ++j) {
            const double y = (j - 1) * g.dy + 0.;
            for (int i = 0; i < nx + 2; ++i) {
                const double u = ((i - 1) * g.dx + 0.) + y;
                std::memcpy(&bits[(size_t)j * sy + i], &u, sizeof u);
            }
        }
        std::vector<uint64_t> uniq(bits);
        std::sort(uniq.begin(), uniq.end());
        uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
        if (uniq.size() * 2 > pairs) return true;
        t.sums.resize(uniq.size());
        for (size_t d = 0; d < uniq.size(); ++d) std::memcpy(&t.sums[d], &uniq[d], sizeof(double));
        t.sum_of.resize(pairs);
        for (size_t q = 0; q < pairs; ++q)
            t.sum_of[q] = (int)(std::lower_bound(uniq.begin(), uniq.end(), bits[q]) - uniq.begin());
    } catch (...) {
        t.sums.clear();  // evaluate every node directly instead
        t.sum_of.clear();
    }
    return true;
}

// Implicit surface (Fold3dPMM.c:137-147) on node planes k0 <= k < k1, ghosts
// included, into IF (plane k0 first).
void surface_planes(double *IF, const fold3d_grid &g, int k0, int k1, const SurfaceTables &t, int nth)
{
    const long long sy = g.nx + 2, sz = sy * (g.ny + 2);
    parallel_for(k0, k1, nth, [&](int k) {
        const double z = (k - 1) * g.dz + 0.;
        std::vector<double> sin_u;  // sin(sum + z) for each distinct sum of the tables
        if (!t.sums.empty()) {
            try {
                sin_u.resize(t.sums.size());
                for (size_t d = 0; d < t.sums.size(); ++d) sin_u[d] = std::sin(t.sums[d] + z);
            } catch (...) {
                sin_u.clear();
            }
        }
        for (int j = 0; j < g.ny + 2; ++j) {
            const double y = (j - 1) * g.dy + 0.;
            double *row = IF + sz * (k - k0) + sy * j;
            const size_t r = (size_t)j * sy;
            for (int i = 0; i < g.nx + 2; ++i) {
                const double x = (i - 1) * g.dx + 0.;
                // x + y + z rounds as (x + y) + z: the tabulated sum plus z
                const double sxyz = sin_u.empty() ? std::sin(x + y + z) : sin_u[t.sum_of[r + i]];
                row[i] = surface_tab(x, y, z, t.sin_x[i], t.cos_yx[r + i], sxyz);
            }
        }
    });
}

int init_threads() { return host_threads(); }

void host_parallel_for(int lo, int hi, int nthreads, const std::function<void(int)> &fn)
{
    parallel_for(lo, hi, nthreads, fn);
}

}  // namespace fold3d

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

static int init_implicit_host(double *T, const fold3d_grid *g, const fold3d_medium *m);

int fold3d_init_implicit(double *T, const fold3d_grid *g, const fold3d_medium *m)
{
    try {  // host threads and tables: an exception becomes a status code, not a crash
        return init_implicit_host(T, g, m);
    } catch (const std::bad_alloc &) {
        return FOLD3D_ERR_NOMEM;
    } catch (...) {
        return FOLD3D_ERR_INVALID;
    }
}

static int init_implicit_host(double *T, const fold3d_grid *g, const fold3d_medium *m)
{
    if (!T || !g || !m) return FOLD3D_ERR_INVALID;
    if (g->nx < 2 || g->ny < 2 || g->nz < 2) return FOLD3D_ERR_INVALID;
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const long long sy = nx + 2, sz = (long long)(nx + 2) * (ny + 2);
    const size_t cells = (size_t)sz * (nz + 2);
    // not zero-filled: the parallel sampling pass writes (and first touches) every element
    std::unique_ptr<double[]> IF_buf(new (std::nothrow) double[cells]);
    if (!IF_buf) return FOLD3D_ERR_NOMEM;
    double *const IF = IF_buf.get();
    const int nth = host_threads();
    const double hx = g->dx, hy = g->dy, hz = g->dz;
    // :137-147, node coordinates from x/y/z (:115-126)
    fold3d::SurfaceTables tabs;
    if (!fold3d::surface_tables(*g, tabs, nth)) return FOLD3D_ERR_NOMEM;
    fold3d::surface_planes(IF, *g, 0, nz + 2, tabs, nth);
    parallel_for(0, nz + 2, nth, [&](int k) {
        for (long long id = sz * k; id < sz * (k + 1); ++id) T[id] = (side(IF[id]) * 1.0) * kMaxT;
    });
    HostNode node{T, sy, sz, m->F, {m->ax, m->ay, m->az}};
    const double h[3] = {hx, hy, hz};
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
                    for (int i = i0; i <= i1; ++i)
                        fold3d_seed::seed_voxel(IF, sy, sz, h, i, j, k, kSteps, kBlends, node);
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
// (:49-52) and pitch nx+2.  The grid is remembered as the pitch of InitNode
// and updateVoxel, whose reference signatures carry no size.
void ImplicitInitialiser(double *T, int nx, int ny, int nz, double dxx, double dyy, double dzz)
{
    const fold3d_grid g = {nx, ny, nz, dxx, dyy, dzz};
    const fold3d_medium m = {1.1, -0.35, 0.4, 0.7};
    fold3d::compat_note_host_grid(nx, ny, nz);
    fold3d_init_implicit(T, &g, &m);
}

// InitNode (Fold3dPMM.h:64, Fold3dPMM.c:35-54): min-update of node (i, j, k)
// with the reference medium's exact time from a point at (x, y, z) relative
// to the node, keeping the node's sign.  The reference indexes T with its
// compile-time HEIGHT; here the pitch is the host grid (see
// fold3d::compat_host_pitch).  Without one, nothing is written and
// fold3d_last_error says why.
void InitNode(double x, double y, double z, int i, int j, int k, double *T)
{
    long long sy, sz;
    if (!T || !fold3d::compat_host_pitch(sy, sz)) return;
    const HostNode node{T, sy, sz, 1.1, {-0.35, 0.4, 0.7}};
    node(x, y, z, i, j, k);
}

// updateVoxel (Fold3dPMM.h:67-70, Fold3dPMM.c:56-112): the 44 node updates of
// one seeding point, in the reference's order and with its index slips (the
// same table the initialisers use).
void updateVoxel(double *T, int i, int j, int k, double xp, double yp, double zp, double dxx, double dyy, double dzz)
{
    long long sy, sz;
    if (!T || !fold3d::compat_host_pitch(sy, sz)) return;
    HostNode node{T, sy, sz, 1.1, {-0.35, 0.4, 0.7}};
    const double h[3] = {dxx, dyy, dzz};
    fold3d_seed::seed_point(kSteps, h, i, j, k, xp, yp, zp, node);
}

// Node coordinates (Fold3dPMM.h:72-76, Fold3dPMM.c:115-126): the reference's
// domain starts at 0 on every axis (_xmin, _ymin, _zmin).
double x(int i, double DX) { return (i - 1) * DX + 0.; }
double y(int j, double dy) { return (j - 1) * dy + 0.; }
double z(int k, double dz) { return (k - 1) * dz + 0.; }

}  // extern "C"
