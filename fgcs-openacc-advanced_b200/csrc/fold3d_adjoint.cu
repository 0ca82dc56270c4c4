// fold3d_adjoint.cu -- adjoint (reverse-mode derivative) of a converged
// elliptical-medium solve.  No counterpart in the reference.
//
// The forward solve records, per cell, the candidate that last set its time
// (its "winner": sweep direction and candidate id, 1 byte).  At convergence
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
//
// A backward pass is one persistent launch over (step, 32 x kWaveTV tile)
// items, like a forward WAVEFRONT pass run the other way: the cells of step
// p's target plane receive their pushes from the 3 x 3 tiles around them at
// step p-1 (the plane behind them in this walk), so item (p, t) waits for
// exactly those items' completion flags (bounded waits), then pushes and
// publishes its own flag.
#include <math_constants.h>

#include <cstring>

#include "fold3d_ellip.cuh"
#include "fold3d_internal.h"
#include "fold3d_sync.cuh"

namespace fold3d {

namespace {

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

// Fan times of the winner's direction for target x (source point first,
// then the rim in order).
__device__ __forceinline__ void fan_times(const double *T, long long x, const PlaneGeom &g, double tv[9])
{
    const long long st = x - g.sn;
#pragma unroll
    for (int p = 0; p < 9; ++p) tv[p] = fabs(T[st + fan_i(p) * g.sx + fan_j(p) * g.sy]);
}

// Field index of fan point p of target x.
__device__ __forceinline__ long long fan_index(long long x, const PlaneGeom &g, int p)
{
    return x - g.sn + fan_i(p) * g.sx + fan_j(p) * g.sy;
}
}  // namespace

constexpr int kAdjThreads = 32 * kWaveTV;

// One backward pass of direction b.a.dir (see the top of the file).
__global__ void __launch_bounds__(kAdjThreads, 1024 / kAdjThreads)
    adj_pass_kernel(AdjWaveArgs b, const __grid_constant__ EllipParam ep)
{
    __shared__ int s_next;
    const WaveArgs &a = b.a;
    const PlaneGeom &g = a.pg;
    const int ntiles = a.ntu * a.ntv;
    const long long total = (long long)a.steps * ntiles;
    const unsigned want = a.epoch << 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double dmax = 0.0;
    if (tid == 0) {
        const unsigned w = atomicAdd(a.work, 1u);
        s_next = (w < total) ? (int)w : -1;
    }
    __syncthreads();
    for (;;) {
        const int item = s_next;
        if (item < 0) break;
        __syncthreads();  // every thread has read s_next
        if (tid == 0) {  // claim the next item now; it is processed after this one
            int it = -1;
            if (*(volatile unsigned *)a.status == 0) {
                const unsigned w = atomicAdd(a.work, 1u);
                if (w < total) it = (int)w;
            }
            s_next = it;
        }
        const int p = item / ntiles, t = item - p * ntiles;
        const int tu = t % a.ntu, tv = t / a.ntu;
        const int tgt = a.first_src - p * a.sg;
        // Everything but lambda is fixed during the adjoint: find this
        // thread's cell, its winner's source points and weights, and what it
        // pushed before, while the items it waits for are still running.
        const int u = tu * 32 + lane + 1;
        const int v = tv * kWaveTV + warp + 1;
        long long x = -1, src[3] = {0, 0, 0};
        double wt[3] = {0.0, 0.0, 0.0}, P = 0.0;
        int np = 0;
        if (u <= g.nu && v <= g.nv) {
            const long long xc = (long long)tgt * g.s_nrm + (long long)u * g.su + (long long)v * g.sv;
            const unsigned w = b.W[xc];
            if (w != kNoWinner && (int)(w / kEllipCands) == a.dir) {
                x = xc;
                P = b.pushed[x];
                double tv9[9], c[3], n;
                int pt[3];
                fan_times(b.T, x, g, tv9);
                if (!(ell_cand(ell_local(ep.med, ep.dir, x), tv9, (int)(w % kEllipCands), pt, wt, np, c, n) < CUDART_INF))
                    np = 0;
#pragma unroll
                for (int q = 0; q < 3; ++q) src[q] = (q < np) ? fan_index(x, g, pt[q]) : 0;
            }
        }
        int timed_out = 0;
        if (tid < 9 && p > 0) {
            const int nu = tu + tid % 3 - 1, nv = tv + tid / 3 - 1;
            if (nu >= 0 && nu < a.ntu && nv >= 0 && nv < a.ntv) {
                const unsigned *fl = a.flags + (long long)(p - 1) * ntiles + nv * a.ntu + nu;
                const unsigned long long t0 = global_ns();
                unsigned spins = 0;
                while (ld_acquire(fl) < want) {
                    if (++spins > (1u << 26) || global_ns() - t0 > a.timeout_ns ||
                        *(volatile unsigned *)a.status != 0) {
                        atomicCAS(a.status, 0u, 1u);  // FOLD3D_ERR_TIMEOUT
                        timed_out = 1;
                        break;
                    }
                    if (kPollNs) __nanosleep(kPollNs);
                }
            }
        }
        if (__syncthreads_or(timed_out)) break;
        if (x >= 0) {
            const double L = __ldcg(b.lam + x);
            const double D = L - P;
            if (D != 0.0) {
                b.pushed[x] = L;
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    if (q < np) atomicAdd(b.lam + src[q], wt[q] * D);
                dmax = fmax(dmax, fabs(D));
            }
        }
        // publish: the barrier makes every thread's atomics precede thread 0's
        // release store, which orders them (cumulatively) before the flag
        __syncthreads();
        if (tid == 0) st_release(a.flags + item, want);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if (lane == 0 && dmax > 0.0) atomicMax(a.maxd, (unsigned long long)__double_as_longlong(dmax));
}

// dL/dM(x) = lambda(x) d(time(x))/dM(x), six arrays (component-major) in the
// field layout, accumulated in the order of the CPU statement.  Every cell is
// written: ghosts and cells without a winner get 0.
__global__ void __launch_bounds__(256) adj_grad_kernel(const double *__restrict__ T, const double *__restrict__ lam,
                                                       const unsigned char *__restrict__ W,
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
        if (w < 6u * kEllipCands) {
            const int dir = (int)(w / kEllipCands);
            const EllipDir &D = geo.d[dir];
            double tv[9];
            fan_times(T, x, geo.pg[dir], tv);
            int pt[3], np;
            double wt[3], c[3], n;
            if (ell_cand(ell_local(med, D, x), tv, (int)(w % kEllipCands), pt, wt, np, c, n) < CUDART_INF) {
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

cudaError_t launch_adj_pass(const AdjWaveArgs &b, const EllipParam &ep, int grid, cudaStream_t s)
{
    adj_pass_kernel<<<grid, kAdjThreads, 0, s>>>(b, ep);
    return cudaGetLastError();
}

int adj_blocks_per_sm()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adj_pass_kernel, kAdjThreads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_adj_grad(const double *T, const double *lam, const unsigned char *W, const AdjGeom &geo,
                            const EllipMedium &med, const fold3d_grid &g, double *dLdM, cudaStream_t s)
{
    adj_grad_kernel<<<148 * 8, 256, 0, s>>>(T, lam, W, geo, med, g.nx, g.ny, g.nz, dLdM);
    return cudaGetLastError();
}

}  // namespace fold3d
