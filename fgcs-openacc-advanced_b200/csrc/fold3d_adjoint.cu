// fold3d_adjoint.cu -- adjoint (reverse-mode derivative) of a converged
// elliptical-medium solve.  No counterpart in the reference.
//
// The forward solve records, per cell, the candidate that last set its time
// (its "winner": sweep direction and candidate id, 2 bytes).  At convergence
// a cell's time is that candidate, t(footpoint) + ||X - footpoint||_M, with
// the footpoint on a vertex, edge or triangle of the direction's source
// plane.  By the envelope theorem its derivative with respect to each source
// time is that source's barycentric weight at the footpoint, and with respect
// to the scaled local metric entry A_ij it is c_i c_j / (2 n) (c the
// footpoint-to-target vector in spacing units, n its length; off-diagonal
// entries appear twice).
//
// Given r = dL/dT, the total derivative lambda = dL/dT_total solves
// lambda(p) = r(p) + sum over cells x whose winner uses p of w_xp lambda(x).
// Winners only depend on smaller times (a property of the converged field
// that the tests check), so lambda flows against the sweeps: each backward
// pass walks one direction's target planes in reverse order and, for every
// cell whose winner came from that direction, pushes the part of lambda(x)
// not yet pushed to its footpoint's source points (double atomicAdd).  A
// chain of winners of one direction is done in one pass; backward sweeps
// (all six directions, reversed) repeat until a sweep pushes nothing.
// Finally dL/dM(x) = lambda(x) * d(time)/dM(x).
#include <math_constants.h>

#include <cstring>

#include "fold3d_ellip.cuh"
#include "fold3d_internal.h"

namespace fold3d {

namespace {
constexpr unsigned short kNoWinner = 0xffffu;

// Point p of the fan: 0 the source point st, 1..8 rim point p-1.
__device__ __forceinline__ int fan_i(int p) { return p == 0 ? 0 : ell_ri(p - 1); }
__device__ __forceinline__ int fan_j(int p) { return p == 0 ? 0 : ell_rj(p - 1); }

// Candidate `id` without gates (same expressions as the forward solver):
// returns its value or +inf, the footpoint's weights over fan points pt[],
// and the footpoint-to-target vector c (spacing units) with its length n.
__device__ double ell_cand(const EllipA &A, const double tv[9], int id, int pt[3], double w[3], int &np, double c[3],
                           double &nlen)
{
    np = 0;
    if (id <= 8) {
        const int i = fan_i(id), j = fan_j(id);
        const double q = ell_bf(A, -i, -j, 1, -i, -j, 1);
        if (!(q > 0.0)) return CUDART_INF;
        np = 1;
        pt[0] = id;
        w[0] = 1.0;
        c[0] = -i;
        c[1] = -j;
        c[2] = 1.0;
        nlen = sqrt(q);
        return tv[id] + nlen;
    }
    if (id <= 24) {
        int P, Q;
        if (id <= 16) {
            P = 0;
            Q = id - 8;
        } else {
            P = id - 16;
            Q = (id - 16) % 8 + 1;
        }
        const int pi = fan_i(P), pj = fan_j(P), qi = fan_i(Q), qj = fan_j(Q);
        const int ei = qi - pi, ej = qj - pj;
        const double a = ell_bf(A, ei, ej, 0, ei, ej, 0);
        const double b = ell_bf(A, ei, ej, 0, -pi, -pj, 1);
        const double cc = ell_bf(A, -pi, -pj, 1, -pi, -pj, 1);
        const double d = tv[Q] - tv[P];
        const double den = a - d * d;
        const double disc = a * cc - b * b;
        if (!(den > 0.0 && disc > 0.0)) return CUDART_INF;
        const double n = sqrt(disc / den);
        const double lam = (b - d * n) / a;
        if (!(lam > 0.0 && lam < 1.0)) return CUDART_INF;
        np = 2;
        pt[0] = P;
        pt[1] = Q;
        w[0] = 1.0 - lam;
        w[1] = lam;
        c[0] = -pi - lam * ei;
        c[1] = -pj - lam * ej;
        c[2] = 1.0;
        nlen = n;
        return tv[P] + lam * d + n;
    }
    const int r = id - 25, Pa = r + 1, Pb = (r + 1) % 8 + 1;
    const int ai = fan_i(Pa), aj = fan_j(Pa), bi = fan_i(Pb), bj = fan_j(Pb);
    const double p11 = ell_bf(A, ai, aj, 0, ai, aj, 0);
    const double p12 = ell_bf(A, ai, aj, 0, bi, bj, 0);
    const double p22 = ell_bf(A, bi, bj, 0, bi, bj, 0);
    const double q1 = ell_bf(A, ai, aj, 0, 0, 0, 1);
    const double q2 = ell_bf(A, bi, bj, 0, 0, 0, 1);
    const double cz = A.zz;
    const double d1 = tv[Pa] - tv[0], d2 = tv[Pb] - tv[0];
    const double det = p11 * p22 - p12 * p12;
    if (!(det > 0.0)) return CUDART_INF;
    const double u1 = p22 * d1 - p12 * d2, u2 = p11 * d2 - p12 * d1;
    const double w1 = p22 * q1 - p12 * q2, w2 = p11 * q2 - p12 * q1;
    const double s = (d1 * u1 + d2 * u2) / det;
    const double rr = cz - (q1 * w1 + q2 * w2) / det;
    if (!(s < 1.0 && rr > 0.0)) return CUDART_INF;
    const double n = sqrt(rr / (1.0 - s));
    const double l1 = (w1 - n * u1) / det, l2 = (w2 - n * u2) / det;
    if (!(l1 > 0.0 && l2 > 0.0 && l1 + l2 < 1.0)) return CUDART_INF;
    np = 3;
    pt[0] = 0;
    pt[1] = Pa;
    pt[2] = Pb;
    w[0] = 1.0 - l1 - l2;
    w[1] = l1;
    w[2] = l2;
    c[0] = -l1 * ai - l2 * bi;
    c[1] = -l1 * aj - l2 * bj;
    c[2] = 1.0;
    nlen = n;
    return tv[0] + (l1 * d1 + l2 * d2) + n;
}

// Fan times and field indices of the winner's direction for target x.
__device__ __forceinline__ void fan_of(const double *T, long long x, const PlaneGeom &g, long long idx[9], double tv[9])
{
    const long long st = x - g.sn;
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        idx[p] = st + fan_i(p) * g.sx + fan_j(p) * g.sy;
        tv[p] = fabs(T[idx[p]]);
    }
}
}  // namespace

// One backward step of direction dir: the cells of one target plane whose
// winner came from this direction push what they have not pushed yet.
__global__ void __launch_bounds__(256) adj_push_kernel(const double *__restrict__ T, double *lam, double *pushed,
                                                       const unsigned short *__restrict__ W, PlaneGeom g,
                                                       EllipParam ep, int dir, long long tgt_off,
                                                       unsigned long long *maxd)
{
    const int u = blockIdx.x * 32 + threadIdx.x + 1;
    const int v = blockIdx.y * 8 + threadIdx.y + 1;
    double dmax = 0.0;
    if (u <= g.nu && v <= g.nv) {
        const long long x = tgt_off + (long long)u * g.su + (long long)v * g.sv;
        const unsigned w = W[x];
        if (w != kNoWinner && (int)(w >> 6) == dir) {
            const double L = lam[x];
            const double D = L - pushed[x];
            if (D != 0.0) {
                pushed[x] = L;
                long long idx[9];
                double tv[9];
                fan_of(T, x, g, idx, tv);
                int pt[3], np;
                double wt[3], c[3], n;
                if (ell_cand(ell_local(ep.med, ep.dir, x), tv, (int)(w & 63u), pt, wt, np, c, n) < CUDART_INF)
                    for (int q = 0; q < np; ++q) atomicAdd(lam + idx[pt[q]], wt[q] * D);
                dmax = fabs(D);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if ((threadIdx.x & 31) == 0 && dmax > 0.0) atomicMax(maxd, (unsigned long long)__double_as_longlong(dmax));
}

// dL/dM(x) = lambda(x) d(time(x))/dM(x), six arrays (component-major) in the
// field layout, accumulated in the order of the CPU statement.  Every cell is
// written: ghosts and cells without a winner get 0.
__global__ void __launch_bounds__(256) adj_grad_kernel(const double *__restrict__ T, const double *__restrict__ lam,
                                                       const unsigned short *__restrict__ W,
                                                       const __grid_constant__ AdjGeom geo, EllipMedium med, int nx,
                                                       int ny, int nz, double *dLdM)
{
    const long long sy = nx + 2, sz = (long long)(nx + 2) * (ny + 2);
    const long long cells = sz * (nz + 2);
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < cells;
         x += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(x % sy), j = (int)((x / sy) % (ny + 2)), k = (int)(x / sz);
        const bool interior = i >= 1 && i <= nx && j >= 1 && j <= ny && k >= 1 && k <= nz;
        double dM[6] = {0, 0, 0, 0, 0, 0};
        const unsigned w = interior ? W[x] : kNoWinner;
        if (w != kNoWinner && (w >> 6) < 6u) {
            const int dir = (int)(w >> 6);
            const EllipDir &D = geo.d[dir];
            long long idx[9];
            double tv[9];
            fan_of(T, x, geo.pg[dir], idx, tv);
            int pt[3], np;
            double wt[3], c[3], n;
            if (ell_cand(ell_local(med, D, x), tv, (int)(w & 63u), pt, wt, np, c, n) < CUDART_INF) {
                const double hh[3] = {D.hx, D.hy, D.hz};
                const int sxy[3][3] = {{1, D.sxy, D.sxz}, {D.sxy, 1, D.syz}, {D.sxz, D.syz, 1}};
                const int comp[3][3] = {{D.ixx, D.ixy, D.ixz}, {D.ixy, D.iyy, D.iyz}, {D.ixz, D.iyz, D.izz}};
#pragma unroll
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int r = p; r < 3; ++r) {
                        const double dA = c[p] * c[r] / ((p == r ? 2.0 : 1.0) * n);
                        dM[comp[p][r]] += dA * (double)sxy[p][r] * hh[p] * hh[r];
                    }
            }
        }
        const double L = interior ? lam[x] : 0.0;
#pragma unroll
        for (int m = 0; m < 6; ++m) dLdM[m * cells + x] = L * dM[m];
    }
}

cudaError_t launch_adj_push(const double *T, double *lam, double *pushed, const unsigned short *W,
                            const PlaneGeom &pg, const EllipParam &ep, int dir, int tgt, unsigned long long *maxd,
                            cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((pg.nu + 31) / 32, (pg.nv + 7) / 8);
    adj_push_kernel<<<grid, block, 0, s>>>(T, lam, pushed, W, pg, ep, dir, (long long)tgt * pg.s_nrm, maxd);
    return cudaGetLastError();
}

cudaError_t launch_adj_grad(const double *T, const double *lam, const unsigned short *W, const AdjGeom &geo,
                            const EllipMedium &med, const fold3d_grid &g, double *dLdM, cudaStream_t s)
{
    adj_grad_kernel<<<148 * 8, 256, 0, s>>>(T, lam, W, geo, med, g.nx, g.ny, g.nz, dLdM);
    return cudaGetLastError();
}

}  // namespace fold3d
