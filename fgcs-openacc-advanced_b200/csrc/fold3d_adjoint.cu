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

template <class R> __device__ __forceinline__ R r_inf();
template <> __device__ __forceinline__ double r_inf<double>() { return CUDART_INF; }
template <> __device__ __forceinline__ float r_inf<float>() { return CUDART_INF_F; }

// Candidate `id` without gates (same expressions as the forward solver):
// returns its value or +inf, the footpoint's weights over fan points pt[],
// and the footpoint-to-target vector c (spacing units) with its length n.
template <class R>
__device__ R ell_cand(const EllipAT<R> &A, const R tv[9], int id, int pt[3], R w[3], int &np, R c[3], R &nlen)
{
    np = 0;
    if (id <= 8) {
        const int i = fan_i(id), j = fan_j(id);
        const R q = ell_bf(A, -i, -j, 1, -i, -j, 1);
        if (!(q > R(0))) return r_inf<R>();
        np = 1;
        pt[0] = id;
        w[0] = R(1);
        c[0] = (R)(-i);
        c[1] = (R)(-j);
        c[2] = R(1);
        nlen = ell_sqrt(q);
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
        const R a = ell_bf(A, ei, ej, 0, ei, ej, 0);
        const R b = ell_bf(A, ei, ej, 0, -pi, -pj, 1);
        const R cc = ell_bf(A, -pi, -pj, 1, -pi, -pj, 1);
        const R d = tv[Q] - tv[P];
        const R den = a - d * d;
        const R disc = a * cc - b * b;
        if (!(den > R(0) && disc > R(0))) return r_inf<R>();
        const R n = ell_sqrt(disc / den);
        const R lam = (b - d * n) / a;
        if (!(lam > R(0) && lam < R(1))) return r_inf<R>();
        np = 2;
        pt[0] = P;
        pt[1] = Q;
        w[0] = R(1) - lam;
        w[1] = lam;
        c[0] = (R)(-pi) - lam * (R)ei;
        c[1] = (R)(-pj) - lam * (R)ej;
        c[2] = R(1);
        nlen = n;
        return tv[P] + lam * d + n;
    }
    const int r = id - 25, Pa = r + 1, Pb = (r + 1) % 8 + 1;
    const int ai = fan_i(Pa), aj = fan_j(Pa), bi = fan_i(Pb), bj = fan_j(Pb);
    const R p11 = ell_bf(A, ai, aj, 0, ai, aj, 0);
    const R p12 = ell_bf(A, ai, aj, 0, bi, bj, 0);
    const R p22 = ell_bf(A, bi, bj, 0, bi, bj, 0);
    const R q1 = ell_bf(A, ai, aj, 0, 0, 0, 1);
    const R q2 = ell_bf(A, bi, bj, 0, 0, 0, 1);
    const R cz = A.zz;
    const R d1 = tv[Pa] - tv[0], d2 = tv[Pb] - tv[0];
    const R det = p11 * p22 - p12 * p12;
    if (!(det > R(0))) return r_inf<R>();
    const R u1 = p22 * d1 - p12 * d2, u2 = p11 * d2 - p12 * d1;
    const R w1 = p22 * q1 - p12 * q2, w2 = p11 * q2 - p12 * q1;
    const R s = (d1 * u1 + d2 * u2) / det;
    const R rr = cz - (q1 * w1 + q2 * w2) / det;
    if (!(s < R(1) && rr > R(0))) return r_inf<R>();
    const R n = ell_sqrt(rr / (R(1) - s));
    const R l1 = (w1 - n * u1) / det, l2 = (w2 - n * u2) / det;
    if (!(l1 > R(0) && l2 > R(0) && l1 + l2 < R(1))) return r_inf<R>();
    np = 3;
    pt[0] = 0;
    pt[1] = Pa;
    pt[2] = Pb;
    w[0] = R(1) - l1 - l2;
    w[1] = l1;
    w[2] = l2;
    c[0] = -l1 * (R)ai - l2 * (R)bi;
    c[1] = -l1 * (R)aj - l2 * (R)bj;
    c[2] = R(1);
    nlen = n;
    return tv[0] + (l1 * d1 + l2 * d2) + n;
}

// Fan times of the winner's direction for target x (source point first,
// then the rim in order).
template <class R> __device__ __forceinline__ void fan_times(const R *T, long long x, const PlaneGeom &g, R tv[9])
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

// The source points and weights of target x's winner `w` (a cell of the
// pass's direction): np = 0 when the candidate is not finite.
template <class R>
__device__ __forceinline__ void adj_weights(const R *T, const EllipParam &ep, const PlaneGeom &g, long long x,
                                            unsigned w, long long src[3], R wt[3], int &np)
{
    R tv9[9], c[3], n;
    int pt[3];
    fan_times(T, x, g, tv9);
    if (!(ell_cand(ell_local<R>(ep.med, ep.dir, x), tv9, (int)(w % kEllipCands), pt, wt, np, c, n) < r_inf<R>()))
        np = 0;
#pragma unroll
    for (int q = 0; q < 3; ++q) src[q] = (q < np) ? fan_index(x, g, pt[q]) : 0;
}

// One item (step p, tile t) of a backward pass, for all threads of the CTA:
// prepare the pushes, wait for those of the 3 x 3 tiles of step p-1 that
// have work, push, publish.
// Adds the largest pushed |amount| into dmax.  Returns false if a wait gave
// up (the item is then left unpublished and the caller must leave).
//
// A cell pushes only when its lambda moved since its last push.  Its winner's
// weights (fan times, local metric, one candidate) are worked out while the
// items it waits for still run when lambda has already moved before the
// wait, which is every cell of the first backward sweeps; a cell whose
// lambda only moves during the wait works them out after it, and a cell
// whose lambda did not move, the most of them in the later sweeps, never.
template <class R>
__device__ __forceinline__ bool adj_item(const AdjWaveArgs &b, const EllipParam &ep, int item, double &dmax)
{
    const R *T = static_cast<const R *>(b.T);
    R *lam = static_cast<R *>(b.lam);
    R *pushed = static_cast<R *>(b.pushed);
    const WaveArgs &a = b.a;
    const PlaneGeom &g = a.pg;
    const int ntiles = a.ntu * a.ntv;
    const unsigned want = a.epoch << 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int p = item / ntiles, t = item - p * ntiles;
    const int tu = t % a.ntu, tv = t / a.ntu;
    const int tgt = a.first_src - p * a.sg;
    const int u = tu * 32 + lane + 1;
    const int v = tv * kWaveTV + warp + 1;
    long long x = -1, src[3] = {0, 0, 0};
    R wt[3] = {R(0), R(0), R(0)}, P = R(0);
    int np = 0;
    unsigned win = 0;
    bool ready = false;
    if (u <= g.nu && v <= g.nv) {
        const long long xc = (long long)tgt * g.s_nrm + (long long)u * g.su + (long long)v * g.sv;
        win = b.W[xc];
        if (win != kNoWinner && (int)(win / kEllipCands) == a.dir) {
            x = xc;
            P = pushed[x];
            if (__ldcg(lam + x) != P) {
                adj_weights<R>(T, ep, g, x, win, src, wt, np);
                ready = true;
            }
        }
    }
    int timed_out = 0;
    if (tid < 9 && p > 0) {
        const int nu = tu + tid % 3 - 1, nv = tv + tid / 3 - 1;
        // step p-1 works on plane tgt + sg; its tiles without work are not
        // in the queue and never publish (nor push)
        if (nu >= 0 && nu < a.ntu && nv >= 0 && nv < a.ntv &&
            b.has[(long long)(tgt + a.sg) * ntiles + nv * a.ntu + nu]) {
            const unsigned *fl = a.flags + (long long)(p - 1) * ntiles + nv * a.ntu + nu;
            const unsigned long long t0 = global_ns();
            unsigned spins = 0;
            while (ld_acquire(fl) < want) {
                if (++spins > (1u << 26) || global_ns() - t0 > a.timeout_ns || *(volatile unsigned *)a.status != 0) {
                    atomicCAS(a.status, 0u, 1u);  // FOLD3D_ERR_TIMEOUT
                    timed_out = 1;
                    break;
                }
                if (kPollNs) __nanosleep(kPollNs);
            }
        }
    }
    if (__syncthreads_or(timed_out)) return false;
    if (x >= 0) {
        const R L = __ldcg(lam + x);
        const R D = L - P;
        if (D != R(0)) {
            if (!ready) adj_weights<R>(T, ep, g, x, win, src, wt, np);
            pushed[x] = L;
#pragma unroll
            for (int q = 0; q < 3; ++q)
                if (q < np) atomicAdd(lam + src[q], wt[q] * D);
            dmax = fmax(dmax, (double)fabs(D));
        }
    }
    // publish: the barrier makes every thread's atomics precede thread 0's
    // release store, which orders them (cumulatively) before the flag
    __syncthreads();
    if (tid == 0) st_release(a.flags + item, want);
    return true;
}

// Work map (see AdjTiles): every interior cell with a winner marks its tile
// in its winner direction's orientation.
__global__ void __launch_bounds__(256) adj_tiles_kernel(const unsigned char *__restrict__ W, int nx, int ny, int nz,
                                                        AdjTiles t)
{
    const long long sy = nx + 2, sz = (long long)(nx + 2) * (ny + 2);
    const long long cells = sz * (nz + 2);
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < cells;
         x += (long long)gridDim.x * blockDim.x) {
        const int c[3] = {(int)(x % sy), (int)((x / sy) % (ny + 2)), (int)(x / sz)};
        if (c[0] < 1 || c[0] > nx || c[1] < 1 || c[1] > ny || c[2] < 1 || c[2] > nz) continue;
        const unsigned w = W[x];
        if (w >= 6u * kEllipCands) continue;
        const int d = (int)(w / kEllipCands);
        const int nrm = t.nrm[d];
        const int ub = (nrm == 0) ? 1 : 0, vb = (nrm == 2) ? 1 : 2;
        const int tile = ((c[vb] - 1) / kWaveTV) * t.ntu[nrm] + ((c[ub] - 1) >> 5);
        t.has[d][(long long)c[nrm] * t.ntiles[nrm] + tile] = 1;
    }
}

// Warp maximum of d into *out (IEEE bits of a non-negative double).
__device__ __forceinline__ void adj_flush(double d, unsigned long long *out)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((threadIdx.x & 31) == 0 && d > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(d));
}

// Backward passes of one direction of one or many instances in one launch.
// The items are listed in ba.items (instance slot << 40 | item within the
// instance's pass), tiles with work only, ordered step-major across the
// instances: every item an item waits for comes earlier in the list.
template <class R>
__global__ void __launch_bounds__(kAdjThreads, 1024 / kAdjThreads) batch_adj_pass_kernel(BatchAdjArgs ba)
{
    __shared__ long long s_next;
    __shared__ int s_il;
    __shared__ BatchAdjInst s_inst;
    if (threadIdx.x == 0) {
        const unsigned w = atomicAdd(ba.work, 1u);
        s_next = (w < ba.total) ? (long long)ba.items[w] : -1ll;
        s_il = -1;
    }
    __syncthreads();
    for (;;) {
        const long long e = s_next;
        if (e < 0) break;
        const int il = (int)(e >> 40), local = (int)(e & ((1ll << 40) - 1));
        __syncthreads();  // every thread has read s_next and s_il
        if (threadIdx.x == 0) {  // claim the next item now; it is processed after this one
            long long it = -1;
            if (*(volatile unsigned *)ba.status == 0) {
                const unsigned w = atomicAdd(ba.work, 1u);
                if (w < ba.total) it = (long long)ba.items[w];
            }
            s_next = it;
        }
        if (il != s_il) {  // consecutive items mostly share their instance
            const unsigned *src = reinterpret_cast<const unsigned *>(ba.inst + il);
            unsigned *dst = reinterpret_cast<unsigned *>(&s_inst);
            for (int w = threadIdx.x; w < (int)(sizeof(BatchAdjInst) / 4); w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            if (threadIdx.x == 0) {
                s_inst.b.a.epoch = ba.epoch;  // the pass number is per launch
                s_il = il;
            }
            __syncthreads();
        }
        double dmax = 0.0;
        if (!adj_item<R>(s_inst.b, s_inst.ep, local, dmax)) break;
        adj_flush(dmax, s_inst.b.a.maxd);
    }
}

// The item list of one backward pass (see batch_adj_pass_kernel), built in
// two steps over blocks (step p, instance slot q): count the tiles of step p
// that have work, then (after an exclusive scan of the counts in step-major
// order, on the host) write their items in tile order.
constexpr int kListThreads = 256;

__device__ __forceinline__ const unsigned char *step_tiles(const AdjWaveArgs &b, int p)
{
    return b.has + (long long)(b.a.first_src - p * b.a.sg) * (b.a.ntu * b.a.ntv);
}

__global__ void __launch_bounds__(kListThreads) adj_count_kernel(const BatchAdjInst *inst, int k, int *cnt)
{
    const int p = blockIdx.x, q = blockIdx.y;
    const AdjWaveArgs &b = inst[q].b;
    const int ntiles = b.a.ntu * b.a.ntv;
    int c = 0;
    if (p < b.a.steps) {
        const unsigned char *h = step_tiles(b, p);
        for (int t0 = 0; t0 < ntiles; t0 += kListThreads) {
            const int t = t0 + threadIdx.x;
            c += __syncthreads_count(t < ntiles && h[t]);
        }
    }
    if (threadIdx.x == 0) cnt[(long long)p * k + q] = c;
}

__global__ void __launch_bounds__(kListThreads) adj_fill_kernel(const BatchAdjInst *inst, int k, const long long *off,
                                                                unsigned long long *items)
{
    __shared__ int wcnt[kListThreads / 32];
    const int p = blockIdx.x, q = blockIdx.y;
    const AdjWaveArgs &b = inst[q].b;
    if (p >= b.a.steps) return;
    const int ntiles = b.a.ntu * b.a.ntv;
    const unsigned char *h = step_tiles(b, p);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long base = off[(long long)p * k + q];
    for (int t0 = 0; t0 < ntiles; t0 += kListThreads) {
        const int t = t0 + threadIdx.x;
        const bool f = t < ntiles && h[t];
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) wcnt[warp] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kListThreads / 32; ++w) {
            before += (w < warp) ? wcnt[w] : 0;
            total += wcnt[w];
        }
        if (f)
            items[base + before + __popc(m & ((1u << lane) - 1u))] =
                ((unsigned long long)q << 40) | (unsigned long long)((long long)p * ntiles + t);
        base += total;
        __syncthreads();
    }
}

// dL/dM(x) = lambda(x) d(time(x))/dM(x), six arrays (component-major) in the
// field layout, accumulated in the order of the CPU statement.  Every cell is
// written (ghosts and cells without a winner get 0), or, with accumulate,
// added to.  For a medium given by its parameters (kParamF64) the four
// arrays written are the gradients with respect to s, eps, nx and ny instead
// (the chain rule through M = a I + b n n^T, nz depending on nx and ny; where
// nz = 0 the axis components get only their direct terms).
template <class R>
__global__ void __launch_bounds__(256) adj_grad_kernel(const R *__restrict__ T, const R *__restrict__ lam,
                                                       const unsigned char *__restrict__ W,
                                                       const __grid_constant__ AdjGeom geo, EllipMedium med, int nx,
                                                       int ny, int nz, R *dLdM, int accumulate)
{
    const long long sy = nx + 2, sz = (long long)(nx + 2) * (ny + 2);
    const long long cells = sz * (nz + 2);
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < cells;
         x += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(x % sy), j = (int)((x / sy) % (ny + 2)), k = (int)(x / sz);
        const bool interior = i >= 1 && i <= nx && j >= 1 && j <= ny && k >= 1 && k <= nz;
        R dM[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
        const unsigned w = interior ? W[x] : kNoWinner;
        if (w < 6u * kEllipCands) {
            const int dir = (int)(w / kEllipCands);
            const EllipDir &D = geo.d[dir];
            R tv[9];
            fan_times(T, x, geo.pg[dir], tv);
            int pt[3], np;
            R wt[3], c[3], n;
            if (ell_cand(ell_local<R>(med, D, x), tv, (int)(w % kEllipCands), pt, wt, np, c, n) < r_inf<R>()) {
                const R hh[3] = {(R)D.hx, (R)D.hy, (R)D.hz};
                const int sxy[3][3] = {{1, D.sxy, D.sxz}, {D.sxy, 1, D.syz}, {D.sxz, D.syz, 1}};
                const int comp[3][3] = {{D.ixx, D.ixy, D.ixz}, {D.ixy, D.iyy, D.iyz}, {D.ixz, D.iyz, D.izz}};
#pragma unroll
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int r = p; r < 3; ++r) {
                        const R dA = c[p] * c[r] / ((p == r ? R(2) : R(1)) * n);
                        dM[comp[p][r]] += dA * (R)sxy[p][r] * hh[p] * hh[r];
                    }
            }
        }
        const R L = interior ? lam[x] : R(0);
        if (med.kind == kParamF64) {
            // chain to the parameters (s, eps, nx, ny) of M = a I + b n n^T
            // (ell_metric_from_param), nz depending on nx and ny
            R g[4] = {R(0), R(0), R(0), R(0)};
            if (interior) {
                const double *P[4] = {static_cast<const double *>(med.m[0]), static_cast<const double *>(med.m[1]),
                                      static_cast<const double *>(med.m[2]), static_cast<const double *>(med.m[3])};
                const double ps = P[0][x], eps = P[1][x], nx_ = P[2][x], ny_ = P[3][x];
                const double s2 = ps * ps, den = 1.0 + 2.0 * eps;
                const double a = s2 / den, b = s2 - a;
                const double q = (1.0 - nx_ * nx_) - ny_ * ny_;
                const double nz_ = sqrt(q > 0.0 ? q : 0.0);
                double gm[6];
#pragma unroll
                for (int m = 0; m < 6; ++m) gm[m] = (double)L * (double)dM[m];
                const double ga = gm[0] + gm[3] + gm[5];
                const double gb = gm[0] * nx_ * nx_ + gm[3] * ny_ * ny_ + gm[5] * nz_ * nz_ + gm[1] * nx_ * ny_ +
                                  gm[2] * nx_ * nz_ + gm[4] * ny_ * nz_;
                double gnx = 2.0 * b * nx_ * gm[0] + b * ny_ * gm[1] + b * nz_ * gm[2];
                double gny = 2.0 * b * ny_ * gm[3] + b * nx_ * gm[1] + b * nz_ * gm[4];
                const double gnz = 2.0 * b * nz_ * gm[5] + b * nx_ * gm[2] + b * ny_ * gm[4];
                if (nz_ > 0.0) {
                    gnx -= gnz * nx_ / nz_;
                    gny -= gnz * ny_ / nz_;
                }
                const double da_ds = 2.0 * ps / den, da_de = -2.0 * s2 / (den * den);
                g[0] = (R)(ga * da_ds + gb * (2.0 * ps - da_ds));
                g[1] = (R)(ga * da_de - gb * da_de);
                g[2] = (R)gnx;
                g[3] = (R)gny;
            }
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                R *o = dLdM + m * cells + x;
                *o = accumulate ? *o + g[m] : g[m];
            }
            continue;
        }
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            R *o = dLdM + m * cells + x;
            *o = accumulate ? *o + L * dM[m] : L * dM[m];
        }
    }
}

cudaError_t launch_adj_grad(const void *T, const void *lam, const unsigned char *W, const AdjGeom &geo,
                            const EllipMedium &med, const fold3d_grid &g, void *dLdM, int accumulate, bool f32,
                            cudaStream_t s)
{
    if (f32)
        adj_grad_kernel<float><<<148 * 8, 256, 0, s>>>(static_cast<const float *>(T), static_cast<const float *>(lam),
                                                       W, geo, med, g.nx, g.ny, g.nz, static_cast<float *>(dLdM),
                                                       accumulate);
    else
        adj_grad_kernel<double><<<148 * 8, 256, 0, s>>>(static_cast<const double *>(T),
                                                        static_cast<const double *>(lam), W, geo, med, g.nx, g.ny,
                                                        g.nz, static_cast<double *>(dLdM), accumulate);
    return cudaGetLastError();
}

cudaError_t launch_adj_tiles(const unsigned char *W, const fold3d_grid &g, const AdjTiles &t, cudaStream_t s)
{
    adj_tiles_kernel<<<148 * 8, 256, 0, s>>>(W, g.nx, g.ny, g.nz, t);
    return cudaGetLastError();
}

cudaError_t launch_batch_adj_pass(const BatchAdjArgs &b, bool f32, int grid, cudaStream_t s)
{
    if (f32) batch_adj_pass_kernel<float><<<grid, kAdjThreads, 0, s>>>(b);
    else batch_adj_pass_kernel<double><<<grid, kAdjThreads, 0, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_adj_list(const BatchAdjInst *inst, int k, int max_steps, int *cnt, const long long *off,
                            unsigned long long *items, cudaStream_t s)
{
    const dim3 grid(max_steps, k);
    if (!off) adj_count_kernel<<<grid, kListThreads, 0, s>>>(inst, k, cnt);
    else adj_fill_kernel<<<grid, kListThreads, 0, s>>>(inst, k, off, items);
    return cudaGetLastError();
}

int batch_adj_blocks_per_sm(bool f32)
{
    int n = 0;
    const cudaError_t e =
        f32 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_adj_pass_kernel<float>, kAdjThreads, 0)
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_adj_pass_kernel<double>, kAdjThreads, 0);
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

}  // namespace fold3d
