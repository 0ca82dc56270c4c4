// fold3d_seed.h -- the implicit-surface seeding of ImplicitInitialiser
// (Stencil-OpenACC/Fold3dPMM.c:35-112, :163-383), shared by the host
// initialiser (fold3d_init.cpp, g++) and the device one (fold3d_init_dev.cu,
// nvcc), so that both compile the same arithmetic.  Both builds disable FMA
// contraction, and the operations are IEEE +, -, *, / and sqrt, so the two
// give the same bits.
//
// seed_voxel finds where the surface crosses the 12 edges of a voxel
// (:163-269) and, from each crossing and from blends of it with earlier
// crossings of the same voxel (:271-383), min-updates 44 nearby nodes
// (updateVoxel / InitNode).  The node update is a functor: the host writes
// the field directly, the device takes an atomic minimum.  The tables come
// as pointers (host arrays, or __constant__ copies on the device) filled from
// the initializers below.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define F3D_HD __host__ __device__
#else
#define F3D_HD
#endif

namespace fold3d_seed {

constexpr double kMaxT = 10e15 * 1.0;  // Fold3dPMM.h:6

F3D_HD inline double side(double a) { return (a > 0) ? 1.0 : -1.0; }  // sign(), 0 -> -1

// Fold3dPMM.c:9-26
F3D_HD inline double exact_time(double F, double ax, double ay, double az, double x, double y, double z)
{
    double xsq = x * x + y * y + z * z;
    double adotx = ax * x + ay * y + az * z;
    double q = (F * F - (ax * ax + ay * ay + az * az)) * xsq + adotx * adotx;
    if (q > 0.0) {
        q = adotx + sqrt(q);
        if (q > 0.0) return xsq / q;
    }
    return 1.0 * kMaxT;
}

// Node updates of one seeding point (updateVoxel, Fold3dPMM.c:62-110, in
// order): position shift in multiples of the spacing (+1, -1 or -2), then the
// node offset.  Two rows keep the reference's position/index mismatch
// (:82 shifts y by +1 but writes node j; :86 shifts x by -1, y by -2 but
// writes node i+2, j).
struct NodeStep {
    signed char px, py, pz, di, dj, dk;
};
constexpr int kNodeSteps = 44;
#define FOLD3D_SEED_STEPS { \
    {0, 0, 0, 0, 0, 0},     {-1, 0, 0, 1, 0, 0},    {0, -1, 0, 0, 1, 0},    {0, 0, -1, 0, 0, 1}, \
    {-1, -1, 0, 1, 1, 0},   {-1, 0, -1, 1, 0, 1},   {0, -1, -1, 0, 1, 1},   {-1, -1, -1, 1, 1, 1}, \
    {1, 0, 0, -1, 0, 0},    {1, -1, 0, -1, 1, 0},   {1, 0, -1, -1, 0, 1},   {1, -1, -1, -1, 1, 1}, \
    {-2, 0, 0, 2, 0, 0},    {-2, -1, 0, 2, 1, 0},   {-2, 0, -1, 2, 0, 1},   {-2, -1, -1, 2, 1, 1}, \
    {0, 1, 0, 0, -1, 0},    {-1, 1, 0, 1, 0, 0},    {0, 1, -1, 0, -1, 1},   {-1, 1, -1, 1, -1, 1}, \
    {0, -2, 0, 0, 2, 0},    {-1, -2, 0, 2, 0, 0},   {0, -2, -1, 0, 2, 1},   {-1, -2, -1, 1, 2, 1}, \
    {0, 0, 1, 0, 0, -1},    {-1, 0, 1, 1, 0, -1},   {0, -1, 1, 0, 1, -1},   {-1, -1, 1, 1, 1, -1}, \
    {0, 0, -2, 0, 0, 2},    {-1, 0, -2, 1, 0, 2},   {0, -1, -2, 0, 1, 2},   {-1, -1, -2, 1, 1, 2}, \
    {0, 1, 1, 0, -1, -1},   {1, 0, 1, -1, 0, -1},   {1, 1, 0, -1, -1, 0},   {0, -2, -2, 0, 2, 2}, \
    {-2, 0, -2, 2, 0, 2},   {-2, -2, 0, 2, 2, 0},   {-1, 1, 1, 1, -1, -1},  {1, -1, 1, -1, 1, -1}, \
    {1, 1, -1, -1, -1, 1},  {-1, -2, -2, 1, 2, 2},  {-2, -1, -2, 2, 1, 2},  {-2, -2, -1, 2, 2, 1}, \
}

// p, p + h, p - h or p - 2h (Fold3dPMM.c:62-110) for m = 0, 1, -1, -2: m*h is
// exact and p + (-x) is p - x, so one expression gives the same bits.
F3D_HD inline double shifted(double p, int m, double h) { return (m == 0) ? p : p + (double)m * h; }

// Blends of crossing l with earlier crossings (:274-382), in order.  A blend
// is (sum of w[t] * P[l - off[t]]) / div; its z coordinate takes the y
// coordinate of term `zy` instead of the z coordinate (the reference's
// ypos[l-2] / ypos[l-3] in the zp lines, :309-379), or -1 for none.
struct Blend {
    int minl, div, n, off[3], w[3], zy;
};
constexpr int kBlendCount = 22;
#define FOLD3D_SEED_BLENDS { \
    {1, 3, 2, {0, 1, 0}, {2, 1, 0}, -1}, {1, 3, 2, {0, 1, 0}, {1, 2, 0}, -1}, \
    {2, 3, 2, {0, 2, 0}, {2, 1, 0}, -1}, {2, 3, 2, {0, 2, 0}, {1, 2, 0}, -1}, \
    {3, 3, 2, {0, 3, 0}, {2, 1, 0}, -1}, {3, 3, 2, {0, 3, 0}, {1, 2, 0}, -1}, \
    {3, 3, 3, {0, 2, 3}, {1, 1, 1}, 1},  {3, 4, 3, {0, 2, 3}, {2, 1, 1}, 1}, \
    {3, 4, 3, {0, 2, 3}, {1, 2, 1}, 1},  {3, 4, 3, {0, 2, 3}, {1, 1, 2}, 1}, \
    {4, 3, 2, {0, 4, 0}, {2, 1, 0}, -1}, {4, 3, 2, {0, 4, 0}, {1, 2, 0}, -1}, \
    {4, 3, 3, {0, 2, 3}, {1, 1, 1}, 1},  {4, 3, 3, {0, 2, 4}, {1, 1, 1}, 1}, \
    {4, 3, 3, {0, 3, 4}, {1, 1, 1}, 1},  {5, 3, 2, {0, 5, 0}, {2, 1, 0}, -1}, \
    {5, 3, 2, {0, 5, 0}, {1, 2, 0}, -1}, {5, 3, 3, {0, 2, 3}, {1, 1, 1}, 1}, \
    {5, 3, 3, {0, 2, 4}, {1, 1, 1}, 1},  {5, 3, 3, {0, 2, 5}, {1, 1, 1}, 1}, \
    {5, 3, 3, {0, 3, 5}, {1, 1, 1}, 1},  {5, 3, 3, {0, 3, 4}, {1, 1, 1}, 1}, \
}

// Node (i, j, k) of the grid whose seeding point is at (x, y, z) from it:
// node(x, y, z, i, j, k) is the caller's InitNode.
template <class Node>
F3D_HD inline void seed_point(const NodeStep *steps, const double h[3], int i, int j, int k, double xp, double yp,
                              double zp, Node &node)
{
#ifdef __CUDA_ARCH__
#pragma unroll 4
#else
#pragma GCC unroll 4
#endif
    for (int s = 0; s < kNodeSteps; ++s) {
        const NodeStep &st = steps[s];
        node(shifted(xp, st.px, h[0]), shifted(yp, st.py, h[1]), shifted(zp, st.pz, h[2]), i + st.di, j + st.dj,
             k + st.dk);
    }
}

// Voxel (i, j, k): corners from IF (field layout, strides sy, sz).
template <class Node>
F3D_HD inline void seed_voxel(const double *IF, long long sy, long long sz, const double h[3], int i, int j, int k,
                              const NodeStep *steps, const Blend *blends, Node &node)
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
        double lo = fabs(f), hi = lo;
        for (int q = 0; q < 8; ++q) {
            pos = pos && c[q] > 0.0;
            neg = neg && c[q] < 0.0;
            const double a = fabs(c[q]);
            lo = (a < lo) ? a : lo;
            hi = (a > hi) ? a : hi;
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
        seed_point(steps, h, i, j, k, P[l][0], P[l][1], P[l][2], node);
        for (int bl = 0; bl < kBlendCount; ++bl) {
            const Blend &b = blends[bl];
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
            seed_point(steps, h, i, j, k, c[0], c[1], c[2], node);
        }
    }
}

}  // namespace fold3d_seed
