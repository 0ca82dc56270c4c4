// fold3d_ellip.cuh -- local solver for a per-cell elliptical (tilted
// transversely isotropic) medium.  No counterpart in the reference, whose
// solver only knows the drift medium.
//
// The medium is a per-cell symmetric positive definite metric M: the travel
// time along a short straight segment d is sqrt(d^T M d).  For a tilted
// elliptical medium with vertical speed Vz, Thomsen epsilon and symmetry
// axis n, M = a I + b n n^T with a = 1/(Vz^2 (1 + 2 eps)), b = 1/Vz^2 - a.
//
// In a sweep direction's local frame (x, y in the source plane, z towards
// the target) the target X is at (0, 0, hz) above the source point st and
// the eight neighbours are at (i hx, j hy, 0).  With the time linear on each
// vertex, edge and triangle of that 3 x 3 fan, the new time is the minimum
// of t(p) + ||X - p||_M over the fan, made of: the 9 vertex values, the
// interior stationary points of the 16 edges (8 spokes st-P, 8 rim edges
// between adjacent neighbours) and of the 8 triangles (st, P, next P), all in
// closed form.  Every candidate exceeds the smallest time it is built from,
// and each is only computed while the running time is above that smallest
// time, so, like the drift solver, the update is min(T_old, candidates): the
// WAVEFRONT engine's tile skipping holds unchanged.
//
// Each candidate is t(p) + ||X - p||_M at a point p of its vertex, edge or
// triangle (the closed forms are the exact stationary values), and t(p) is
// at least the smallest time it is built from.  ||X - p||_M is at least
// B = min over the whole source plane of ||X - p||_M, which in the scaled
// local frame (X = (0, 0, 1)) is the square root of the Schur complement
// Azz - [Axz Ayz] [[Axx Axy] [Axy Ayy]]^-1 [Axz Ayz]^T.  So a candidate is
// only computed while the running time is above its smallest input plus
// B (1 - 1e-3): a candidate skipped that way could not have lowered it.  The
// margin 1e-3 is far above the rounding of the closed forms near that bound
// (their square roots are well conditioned there), in float as in double;
// with B = 0 (a rounded Schur complement <= 0) the gates are the plain ones.
//
// oracle/fold3d_oracle.c (orc_ell_*) states the same computation on the
// CPU; this file follows it operation by operation (no FMA contraction), so
// the two agree bit for bit.
#pragma once

namespace fold3d {

// Constants of one sweep direction for the elliptical solver.
struct EllipDir {
    double hx, hy, hz;  // spacings along local x, y and the normal
    int sxy, sxz, syz;  // signs of the local off-diagonal metric entries
    int ixx, iyy, izz, ixy, ixz, iyz;  // which global metric array feeds each local entry
};

// How the per-cell medium is stored (field layout, axes i, j, k):
//  kMetricF32: six float32 arrays of the metric, ordered xx xy xz yy yz zz;
//  kParamF64:  four float64 arrays of the tilted elliptical medium's
//              parameters -- slowness s = 1/Vz, Thomsen epsilon, and the x
//              and y components of the unit symmetry axis n (its z
//              component sqrt(1 - nx^2 - ny^2) >= 0; n and -n are the same
//              axis) -- from which the metric is formed per cell in FP64
//              (ell_metric_from_param).
enum { kMetricF32 = 0, kParamF64 = 1 };
struct EllipMedium {
    const void *m[6];
    int kind;
};

struct EllipParam {
    EllipDir dir;
    EllipMedium med;
};

#ifdef __CUDACC__
// The solver is written once for the field's type R: double (the default
// build) or float (the float32 build).  All arithmetic stays in R (literals
// included), so the float build is float arithmetic throughout.  It also
// compiles for the host, where a test runs it against the CPU statement.

// Local metric scaled by the spacings (Axx = M'xx hx hx, Axy = M'xy hx hy, ...).
template <class R> struct EllipAT {
    R xx, yy, zz, xy, xz, yz;
};
using EllipA = EllipAT<double>;

template <class R> __host__ __device__ __forceinline__ R ell_sqrt(R x);
template <> __host__ __device__ __forceinline__ double ell_sqrt<double>(double x) { return sqrt(x); }
template <> __host__ __device__ __forceinline__ float ell_sqrt<float>(float x) { return sqrtf(x); }

// A read-only metric word (through the read-only data cache on the device).
__host__ __device__ __forceinline__ float ell_ld(const float *p)
{
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

// u^T M' v with u = (ui hx, uj hy, uk hz) and v likewise.
template <class R>
__host__ __device__ __forceinline__ R ell_bf(const EllipAT<R> &A, int ui, int uj, int uk, int vi, int vj, int vk)
{
    return (R)(ui * vi) * A.xx + (R)(uj * vj) * A.yy + (R)(uk * vk) * A.zz + (R)(ui * vj + uj * vi) * A.xy +
           (R)(ui * vk + uk * vi) * A.xz + (R)(uj * vk + uk * vj) * A.yz;
}

template <class R> __host__ __device__ __forceinline__ R ell_min(R a, R b) { return (a < b) ? a : b; }

// B (1 - 1e-3), B the smallest ||X - p||_M over the source plane (header
// comment), or 0 when the rounded Schur complement is not positive.
template <class R> __host__ __device__ __forceinline__ R ell_skip_bound(const EllipAT<R> &A)
{
    const R cof = A.xx * A.yy - A.xy * A.xy;
    if (!(cof > R(0))) return R(0);
    const R sch = A.zz - (A.xz * (A.xz * A.yy - A.yz * A.xy) + A.yz * (A.yz * A.xx - A.xz * A.xy)) / cof;
    return (sch > R(0)) ? ell_sqrt(sch) * R(0.999) : R(0);
}

// Candidate ids (the adjoint's winner record): 0 vertex st, 1+r rim vertex r,
// 9+r spoke st-rim[r], 17+r rim edge rim[r]-rim[r+1], 25+r triangle
// (st, rim[r], rim[r+1]).  Each routine sets win when it lowers tn, and runs
// only while tn is above its smallest input time plus gate (ell_skip_bound).
template <class R>
__host__ __device__ __forceinline__ void ell_vertex(R &tn, int &win, int id, const EllipAT<R> &A, R gate, R tp, int i,
                                                    int j)
{
    if (!(tn > tp + gate)) return;
    const R c = ell_bf(A, -i, -j, 1, -i, -j, 1);
    if (c > R(0)) {
        const R cand = tp + ell_sqrt(c);
        if (cand < tn) {
            tn = cand;
            win = id;
        }
    }
}

template <bool kOwnBound, class R>
__host__ __device__ __forceinline__ void ell_edge(R &tn, int &win, int id, const EllipAT<R> &A, R gate, R tp, R tq,
                                                  int pi, int pj, int qi, int qj)
{
    const R mn = ell_min(tp, tq);
    if (!(tn > mn + gate)) return;
    const int ei = qi - pi, ej = qj - pj;
    const R a = ell_bf(A, ei, ej, 0, ei, ej, 0);
    const R b = ell_bf(A, ei, ej, 0, -pi, -pj, 1);
    const R c = ell_bf(A, -pi, -pj, 1, -pi, -pj, 1);
    // kOwnBound (the rim edges, away from the foot of X): the edge's own
    // distance bound.  The candidate is at least mn plus the smallest
    // ||X - p|| over the segment, whose square is c (b <= 0), c - 2b + a
    // (b >= a) or (ac - b^2)/a; skip while tn - mn is at most 0.999 of it,
    // compared in squares (ac - b^2 = ac sin^2 of the angle between the edge
    // and X - P, far from 0 for an edge of the source plane).
    if (kOwnBound && a > R(0)) {
        const R e2 = (tn - mn) * (tn - mn);
        const bool skip = !(b > R(0))  ? e2 <= R(0.998) * c
                          : !(b < a)   ? e2 <= R(0.998) * (c - R(2) * b + a)
                                       : e2 * a <= R(0.998) * (a * c - b * b);
        if (skip) return;
    }
    const R d = tq - tp;
    const R den = a - d * d;
    const R disc = a * c - b * b;
    if (den > R(0) && disc > R(0)) {
        const R n = ell_sqrt(disc / den);
        const R lam = (b - d * n) / a;
        if (lam > R(0) && lam < R(1)) {
            const R cand = tp + lam * d + n;
            if (cand < tn) {
                tn = cand;
                win = id;
            }
        }
    }
}

template <class R>
__host__ __device__ __forceinline__ void ell_tri(R &tn, int &win, int id, const EllipAT<R> &A, R gate, R t0, R ta,
                                                 R tb, int ai, int aj, int bi, int bj)
{
    if (!(tn > ell_min(t0, ell_min(ta, tb)) + gate)) return;
    const R p11 = ell_bf(A, ai, aj, 0, ai, aj, 0);
    const R p12 = ell_bf(A, ai, aj, 0, bi, bj, 0);
    const R p22 = ell_bf(A, bi, bj, 0, bi, bj, 0);
    const R q1 = ell_bf(A, ai, aj, 0, 0, 0, 1);
    const R q2 = ell_bf(A, bi, bj, 0, 0, 0, 1);
    const R c = A.zz;
    const R d1 = ta - t0, d2 = tb - t0;
    const R det = p11 * p22 - p12 * p12;
    if (!(det > R(0))) return;
    const R u1 = p22 * d1 - p12 * d2, u2 = p11 * d2 - p12 * d1;
    const R w1 = p22 * q1 - p12 * q2, w2 = p11 * q2 - p12 * q1;
    const R s = (d1 * u1 + d2 * u2) / det;
    const R r = c - (q1 * w1 + q2 * w2) / det;
    if (s < R(1) && r > R(0)) {
        const R n = ell_sqrt(r / (R(1) - s));
        const R l1 = (w1 - n * u1) / det, l2 = (w2 - n * u2) / det;
        if (l1 > R(0) && l2 > R(0) && l1 + l2 < R(1)) {
            const R cand = t0 + (l1 * d1 + l2 * d2) + n;
            if (cand < tn) {
                tn = cand;
                win = id;
            }
        }
    }
}

// Rim of the fan in order: (1,0) xt, (1,1) txy, (0,1) yt, (-1,1) tym,
// (-1,0) xnt, (-1,-1) txnyn, (0,-1) ynt, (1,-1) txm.
__host__ __device__ __forceinline__ int ell_ri(int r)
{
    return (r == 0 || r == 1 || r == 7) ? 1 : (r >= 3 && r <= 5) ? -1 : 0;
}
__host__ __device__ __forceinline__ int ell_rj(int r) { return (r >= 1 && r <= 3) ? 1 : (r >= 5) ? -1 : 0; }

__host__ __device__ __forceinline__ double ell_ld(const double *p)
{
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

// The metric M = a I + b n n^T of the tilted elliptical medium from its
// parameters: a = s^2 / (1 + 2 eps), b = s^2 - a, n = (nx, ny, nz) with
// nz = sqrt(max(0, (1 - nx nx) - ny ny)).  Entries xx xy xz yy yz zz, in this
// operation order on every side (the oracle's orc_tti_metric states the
// same), so host and device agree bit for bit.
__host__ __device__ __forceinline__ void ell_metric_from_param(double s, double eps, double nx, double ny,
                                                               double out[6])
{
    const double s2 = s * s;
    const double a = s2 / (1.0 + 2.0 * eps);
    const double b = s2 - a;
    const double q = (1.0 - nx * nx) - ny * ny;
    const double nz = sqrt(q > 0.0 ? q : 0.0);
    const double bx = b * nx, by = b * ny, bz = b * nz;
    out[0] = a + bx * nx;
    out[1] = bx * ny;
    out[2] = bx * nz;
    out[3] = a + by * ny;
    out[4] = by * nz;
    out[5] = a + bz * nz;
}

// Metric entry k (xx xy xz yy yz zz) of cell t, stored as float32.
__host__ __device__ __forceinline__ double ell_entry(const EllipMedium &M, int k, long long t)
{
    return (double)ell_ld(static_cast<const float *>(M.m[k]) + t);
}

// Scaled local metric of the target at field index t.
template <class R>
__host__ __device__ __forceinline__ EllipAT<R> ell_local(const EllipMedium &M, const EllipDir &D, long long t)
{
    const R hx = (R)D.hx, hy = (R)D.hy, hz = (R)D.hz;
    EllipAT<R> A;
    if (M.kind == kParamF64) {
        double m[6];
        ell_metric_from_param(ell_ld(static_cast<const double *>(M.m[0]) + t),
                              ell_ld(static_cast<const double *>(M.m[1]) + t),
                              ell_ld(static_cast<const double *>(M.m[2]) + t),
                              ell_ld(static_cast<const double *>(M.m[3]) + t), m);
        A.xx = (R)m[D.ixx] * hx * hx;
        A.yy = (R)m[D.iyy] * hy * hy;
        A.zz = (R)m[D.izz] * hz * hz;
        A.xy = (R)D.sxy * (R)m[D.ixy] * hx * hy;
        A.xz = (R)D.sxz * (R)m[D.ixz] * hx * hz;
        A.yz = (R)D.syz * (R)m[D.iyz] * hy * hz;
        return A;
    }
    const float *const *f = reinterpret_cast<const float *const *>(M.m);
    A.xx = (R)ell_ld(f[D.ixx] + t) * hx * hx;
    A.yy = (R)ell_ld(f[D.iyy] + t) * hy * hy;
    A.zz = (R)ell_ld(f[D.izz] + t) * hz * hz;
    A.xy = (R)D.sxy * (R)ell_ld(f[D.ixy] + t) * hx * hy;
    A.xz = (R)D.sxz * (R)ell_ld(f[D.ixz] + t) * hx * hz;
    A.yz = (R)D.syz * (R)ell_ld(f[D.iyz] + t) * hy * hz;
    return A;
}

// New signed value of a target from st and its rim values (rim order above);
// win: id of the candidate that set it, -1 if none did.
template <class R>
__host__ __device__ __forceinline__ R point_update_ellip(R told, R st, const R nb[8], const EllipAT<R> &A, int &win)
{
    R tn = fabs(told);
    win = -1;
    const R gate = ell_skip_bound(A);
    ell_vertex(tn, win, 0, A, gate, st, 0, 0);
    R m = st;
#pragma unroll
    for (int r = 0; r < 8; ++r) m = ell_min(m, nb[r]);
    if (tn > m + gate) {  // otherwise every routine below would return at its gate
#pragma unroll
        for (int r = 0; r < 8; ++r) ell_vertex(tn, win, 1 + r, A, gate, nb[r], ell_ri(r), ell_rj(r));
#pragma unroll
        for (int r = 0; r < 8; ++r) ell_edge<false>(tn, win, 9 + r, A, gate, st, nb[r], 0, 0, ell_ri(r), ell_rj(r));
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int s = (r + 1) & 7;
            ell_edge<true>(tn, win, 17 + r, A, gate, nb[r], nb[s], ell_ri(r), ell_rj(r), ell_ri(s), ell_rj(s));
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int s = (r + 1) & 7;
            ell_tri(tn, win, 25 + r, A, gate, st, nb[r], nb[s], ell_ri(r), ell_rj(r), ell_ri(s), ell_rj(s));
        }
    }
    return ((told > R(0)) ? R(1) : R(-1)) * tn;
}
#endif  // __CUDACC__

}  // namespace fold3d
