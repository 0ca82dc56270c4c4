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

// The six metric arrays, field layout, ordered xx xy xz yy yz zz (axes i, j, k).
struct EllipMedium {
    const float *m[6];
};

struct EllipParam {
    EllipDir dir;
    EllipMedium med;
};

#ifdef __CUDACC__
// Local metric scaled by the spacings (Axx = M'xx hx hx, Axy = M'xy hx hy, ...).
struct EllipA {
    double xx, yy, zz, xy, xz, yz;
};

// u^T M' v with u = (ui hx, uj hy, uk hz) and v likewise.
__device__ __forceinline__ double ell_bf(const EllipA &A, int ui, int uj, int uk, int vi, int vj, int vk)
{
    return (double)(ui * vi) * A.xx + (double)(uj * vj) * A.yy + (double)(uk * vk) * A.zz +
           (double)(ui * vj + uj * vi) * A.xy + (double)(ui * vk + uk * vi) * A.xz +
           (double)(uj * vk + uk * vj) * A.yz;
}

__device__ __forceinline__ double ell_min(double a, double b) { return (a < b) ? a : b; }

// Candidate ids (the adjoint's winner record): 0 vertex st, 1+r rim vertex r,
// 9+r spoke st-rim[r], 17+r rim edge rim[r]-rim[r+1], 25+r triangle
// (st, rim[r], rim[r+1]).  Each routine sets win when it lowers tn.
__device__ __forceinline__ void ell_vertex(double &tn, int &win, int id, const EllipA &A, double tp, int i, int j)
{
    if (!(tn > tp)) return;
    const double c = ell_bf(A, -i, -j, 1, -i, -j, 1);
    if (c > 0.0) {
        const double cand = tp + sqrt(c);
        if (cand < tn) {
            tn = cand;
            win = id;
        }
    }
}

__device__ __forceinline__ void ell_edge(double &tn, int &win, int id, const EllipA &A, double tp, double tq, int pi,
                                         int pj, int qi, int qj)
{
    if (!(tn > ell_min(tp, tq))) return;
    const int ei = qi - pi, ej = qj - pj;
    const double a = ell_bf(A, ei, ej, 0, ei, ej, 0);
    const double b = ell_bf(A, ei, ej, 0, -pi, -pj, 1);
    const double c = ell_bf(A, -pi, -pj, 1, -pi, -pj, 1);
    const double d = tq - tp;
    const double den = a - d * d;
    const double disc = a * c - b * b;
    if (den > 0.0 && disc > 0.0) {
        const double n = sqrt(disc / den);
        const double lam = (b - d * n) / a;
        if (lam > 0.0 && lam < 1.0) {
            const double cand = tp + lam * d + n;
            if (cand < tn) {
                tn = cand;
                win = id;
            }
        }
    }
}

__device__ __forceinline__ void ell_tri(double &tn, int &win, int id, const EllipA &A, double t0, double ta, double tb,
                                        int ai, int aj, int bi, int bj)
{
    if (!(tn > ell_min(t0, ell_min(ta, tb)))) return;
    const double p11 = ell_bf(A, ai, aj, 0, ai, aj, 0);
    const double p12 = ell_bf(A, ai, aj, 0, bi, bj, 0);
    const double p22 = ell_bf(A, bi, bj, 0, bi, bj, 0);
    const double q1 = ell_bf(A, ai, aj, 0, 0, 0, 1);
    const double q2 = ell_bf(A, bi, bj, 0, 0, 0, 1);
    const double c = A.zz;
    const double d1 = ta - t0, d2 = tb - t0;
    const double det = p11 * p22 - p12 * p12;
    if (!(det > 0.0)) return;
    const double u1 = p22 * d1 - p12 * d2, u2 = p11 * d2 - p12 * d1;
    const double w1 = p22 * q1 - p12 * q2, w2 = p11 * q2 - p12 * q1;
    const double s = (d1 * u1 + d2 * u2) / det;
    const double r = c - (q1 * w1 + q2 * w2) / det;
    if (s < 1.0 && r > 0.0) {
        const double n = sqrt(r / (1.0 - s));
        const double l1 = (w1 - n * u1) / det, l2 = (w2 - n * u2) / det;
        if (l1 > 0.0 && l2 > 0.0 && l1 + l2 < 1.0) {
            const double cand = t0 + (l1 * d1 + l2 * d2) + n;
            if (cand < tn) {
                tn = cand;
                win = id;
            }
        }
    }
}

// Rim of the fan in order: (1,0) xt, (1,1) txy, (0,1) yt, (-1,1) tym,
// (-1,0) xnt, (-1,-1) txnyn, (0,-1) ynt, (1,-1) txm.
__device__ __forceinline__ int ell_ri(int r) { return (r == 0 || r == 1 || r == 7) ? 1 : (r >= 3 && r <= 5) ? -1 : 0; }
__device__ __forceinline__ int ell_rj(int r) { return (r >= 1 && r <= 3) ? 1 : (r >= 5) ? -1 : 0; }

// Scaled local metric of the target at field index t.
__device__ __forceinline__ EllipA ell_local(const EllipMedium &M, const EllipDir &D, long long t)
{
    EllipA A;
    A.xx = (double)__ldg(M.m[D.ixx] + t) * D.hx * D.hx;
    A.yy = (double)__ldg(M.m[D.iyy] + t) * D.hy * D.hy;
    A.zz = (double)__ldg(M.m[D.izz] + t) * D.hz * D.hz;
    A.xy = (double)D.sxy * (double)__ldg(M.m[D.ixy] + t) * D.hx * D.hy;
    A.xz = (double)D.sxz * (double)__ldg(M.m[D.ixz] + t) * D.hx * D.hz;
    A.yz = (double)D.syz * (double)__ldg(M.m[D.iyz] + t) * D.hy * D.hz;
    return A;
}

// New signed value of a target from st and its rim values (rim order above);
// win: id of the candidate that set it, -1 if none did.
__device__ __forceinline__ double point_update_ellip(double told, double st, const double nb[8], const EllipA &A,
                                                     int &win)
{
    double tn = fabs(told);
    win = -1;
    ell_vertex(tn, win, 0, A, st, 0, 0);
    double m = st;
#pragma unroll
    for (int r = 0; r < 8; ++r) m = ell_min(m, nb[r]);
    if (tn > m) {
#pragma unroll
        for (int r = 0; r < 8; ++r) ell_vertex(tn, win, 1 + r, A, nb[r], ell_ri(r), ell_rj(r));
#pragma unroll
        for (int r = 0; r < 8; ++r) ell_edge(tn, win, 9 + r, A, st, nb[r], 0, 0, ell_ri(r), ell_rj(r));
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int s = (r + 1) & 7;
            ell_edge(tn, win, 17 + r, A, nb[r], nb[s], ell_ri(r), ell_rj(r), ell_ri(s), ell_rj(s));
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int s = (r + 1) & 7;
            ell_tri(tn, win, 25 + r, A, st, nb[r], nb[s], ell_ri(r), ell_rj(r), ell_ri(s), ell_rj(s));
        }
    }
    return ((told > 0) ? 1.0 : -1.0) * tn;
}
#endif  // __CUDACC__

}  // namespace fold3d
