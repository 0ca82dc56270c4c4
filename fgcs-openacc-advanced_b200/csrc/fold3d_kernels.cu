// fold3d_kernels.cu -- per-plane sweep kernels (the PLANES engine).
//
// One thread per target point of a plane, as in the reference's OpenACC
// regions (AN_ISO_1_OpenACC.c:188-193), with the block shaped 32 x 8 over the
// plane's two axes so that, for the y and z directions, each warp reads whole
// 256-byte rows.  The kernel also folds |T_new - T_old| into a per-sweep
// maximum (warp shuffle, shared memory, then one atomicMax per block on the
// IEEE bit pattern, which orders like the value for non-negative doubles).
//
// Two solver variants give identical results: the default takes the
// direction's constants from a table passed as a __grid_constant__
// parameter (fold3d_fast.cuh); the literal variant evaluates the reference's
// expressions point by point (fold3d_solver.cuh) and serves as a cross-check.
#include <cstring>

#include "fold3d_fast.cuh"
#include "fold3d_internal.h"
#include "fold3d_solver.cuh"

namespace fold3d {

static_assert(sizeof(LocalFrame) == sizeof(LocalFrameH), "frame layout");

__device__ __forceinline__ void block_max_to(double d, unsigned long long *out)
{
    __shared__ double wmax[32];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nthreads = blockDim.x * blockDim.y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((tid & 31) == 0) wmax[tid >> 5] = d;
    __syncthreads();
    if (tid < 32) {
        d = (tid < (nthreads >> 5)) ? wmax[tid] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
        if (tid == 0 && d > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(d));
    }
}

// The nine previous-plane magnitudes around the target whose source point
// is `src` (the source plane is not written by the launch: read-only path).
struct Nbr9 {
    double st, xt, yt, xnt, ynt, txy, txm, tym, txnyn;
};
__device__ __forceinline__ Nbr9 load_nbr(const double *__restrict__ T, long long src, const PlaneGeom &g)
{
    Nbr9 s;
    s.st = fabs(__ldg(T + src));
    s.xt = fabs(__ldg(T + src + g.sx));
    s.yt = fabs(__ldg(T + src + g.sy));
    s.xnt = fabs(__ldg(T + src - g.sx));
    s.ynt = fabs(__ldg(T + src - g.sy));
    s.txm = fabs(__ldg(T + src + g.sx - g.sy));
    s.txy = fabs(__ldg(T + src + g.sx + g.sy));
    s.tym = fabs(__ldg(T + src - g.sx + g.sy));
    s.txnyn = fabs(__ldg(T + src - g.sx - g.sy));
    return s;
}

__global__ void __launch_bounds__(256) plane_kernel_fast(double *__restrict__ T, long long src_off, PlaneGeom g,
                                                         const __grid_constant__ DirTable tab,
                                                         unsigned long long *__restrict__ maxd)
{
    const int u = blockIdx.x * 32 + threadIdx.x + 1;
    const int v = blockIdx.y * 8 + threadIdx.y + 1;
    double delta = 0.0;
    if (u <= g.nu && v <= g.nv) {
        const long long src = src_off + (long long)u * g.su + (long long)v * g.sv;
        const long long tgt = src + g.sn;
        const Nbr9 s = load_nbr(T, src, g);
        const double told = T[tgt];
        const double tnew =
            point_update_fast(told, s.st, s.xt, s.yt, s.xnt, s.ynt, s.txy, s.txm, s.tym, s.txnyn, &tab);
        T[tgt] = tnew;
        delta = fabs(tnew - told);
    }
    if (maxd) block_max_to(delta, maxd);
}

__global__ void __launch_bounds__(256) plane_kernel_literal(double *__restrict__ T, long long src_off,
                                                            PlaneGeom g, LocalFrame L,
                                                            unsigned long long *__restrict__ maxd)
{
    const int u = blockIdx.x * 32 + threadIdx.x + 1;
    const int v = blockIdx.y * 8 + threadIdx.y + 1;
    double delta = 0.0;
    if (u <= g.nu && v <= g.nv) {
        const long long src = src_off + (long long)u * g.su + (long long)v * g.sv;
        const long long tgt = src + g.sn;
        const Nbr9 n = load_nbr(T, src, g);
        const Stencil9 s = {n.st, n.xt, n.yt, n.xnt, n.ynt, n.txy, n.txm, n.tym, n.txnyn};
        const double told = T[tgt];
        const double tnew = point_update(told, s, L);
        T[tgt] = tnew;
        delta = fabs(tnew - told);
    }
    if (maxd) block_max_to(delta, maxd);
}

// ---------------------------------------------------------------------------
// Compacted variant.  A block of 256 target points (32 x 8 over the plane)
// stages the nine previous-plane magnitudes of each point in shared memory,
// evaluates every solver call's entry gates once against the point's time
// after the 1-D candidate, and lists the calls that pass as (slot, point)
// items, slot-major per warp: one list of FoldSurf3Points bodies, one of
// their nested FoldEdge2Points calls and one of the eight outer
// FoldEdge2Points calls.  All threads then work through the lists densely,
// so no lane idles on a point whose call was gated off, and fold each
// accepted candidate into the point's minimum with a shared-memory atomicMin
// on the IEEE bits (positive doubles order like their bit patterns).  Gates
// use a time that is never below the reference's at that call, so the items
// are a superset of the calls the reference makes, and every extra call only
// yields candidates at or above the final time: the result is identical.
// ---------------------------------------------------------------------------
namespace {
constexpr int kPts = 256;             // points per block
// Stencil slots: 0 st, 1 xt, 2 yt, 3 xnt, 4 ynt, 5 txy, 6 txm, 7 tym, 8 txnyn.
// Per call slot k (4 bits each, k = 0 in the lowest nibble):
constexpr unsigned kSurfS1 = 0x22443311u;  // xt xt xnt xnt ynt ynt yt yt
constexpr unsigned kSurfS2 = 0x75687865u;  // txy txm txnyn tym txnyn txm txy tym
constexpr unsigned kEdgeS1 = 0x64837251u;  // xt txy yt tym xnt txnyn ynt txm
}  // namespace

__global__ void __launch_bounds__(kPts) plane_kernel_compact(double *__restrict__ T, long long src_off,
                                                             PlaneGeom g, const __grid_constant__ DirTable tab,
                                                             unsigned long long *__restrict__ maxd)
{
    __shared__ double s_nb[9][kPts];
    __shared__ unsigned long long s_best[kPts];
    __shared__ unsigned char s_side[kPts];
    __shared__ unsigned char s_list[3][8][kPts];  // per (list, slot): point indices
    __shared__ int s_cnt[3][8];
    __shared__ int s_pre[3][9];  // segment starts of each list

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int u = blockIdx.x * 32 + lane + 1;
    const int v = blockIdx.y * 8 + (tid >> 5) + 1;
    const bool active = (u <= g.nu && v <= g.nv);
    if (tid < 24) (&s_cnt[0][0])[tid] = 0;

    long long tgt = 0;
    double told = 0.0;
    unsigned msurf = 0, mnest = 0, medge = 0;
    if (active) {
        const long long src = src_off + (long long)u * g.su + (long long)v * g.sv;
        tgt = src + g.sn;
        const Nbr9 n = load_nbr(T, src, g);
        told = T[tgt];
        const int side = told < 0 ? 1 : 0;
        const SideTable &t = tab.side[side];
        double tn = fabs(told);
        if (n.st < tn && t.d1_ok) tn = kmin(tn, n.st + t.K1);  // 1-D candidate (:214-228)
        s_nb[0][tid] = n.st;
        s_nb[1][tid] = n.xt;
        s_nb[2][tid] = n.yt;
        s_nb[3][tid] = n.xnt;
        s_nb[4][tid] = n.ynt;
        s_nb[5][tid] = n.txy;
        s_nb[6][tid] = n.txm;
        s_nb[7][tid] = n.tym;
        s_nb[8][tid] = n.txnyn;
        s_best[tid] = (unsigned long long)__double_as_longlong(tn);
        s_side[tid] = (unsigned char)side;
        if (!(tn < n.st && tn < kmin(n.xt, n.yt) && tn < kmin(n.txy, n.txm) && tn < kmin(n.txnyn, n.tym))) {
            const double S1[8] = {n.xt, n.xt, n.xnt, n.xnt, n.ynt, n.ynt, n.yt, n.yt};
            const double S2[8] = {n.txy, n.txm, n.txnyn, n.tym, n.txnyn, n.txm, n.txy, n.tym};
            const double E1[8] = {n.xt, n.txy, n.yt, n.tym, n.xnt, n.txnyn, n.ynt, n.txm};
            const unsigned me1 = t.m_e1, me2 = t.m_e2, mnb = t.m_nblock, mne = t.m_nest_early,
                           mee = t.m_edge_early;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const double s1 = S1[k], s2 = S2[k];
                // FoldSurf3Points entry (:132) and the nested call's gates (:170, :71)
                const bool fixed_out = (((me1 >> k) & 1u) && s1 > n.st) || (((me2 >> k) & 1u) && s2 > s1);
                if (!fixed_out && !(tn < kmin(n.st, kmin(s1, s2)))) {
                    msurf |= 1u << k;
                    if (tn > kmin(s1, s2) && !(((mnb >> k) & 1u) && s1 > s2) && !(((mne >> k) & 1u) && s2 > s1))
                        mnest |= 1u << k;
                }
                if (!(tn < kmin(E1[k], n.st) || (((mee >> k) & 1u) && E1[k] > n.st))) medge |= 1u << k;
            }
        }
    }
    __syncthreads();
    // item lists, one segment per (list, slot) so that the threads of a warp
    // mostly share a slot (and read the same table entries); one
    // warp-aggregated reservation per (list, slot)
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const unsigned m = (l == 0) ? msurf : (l == 1) ? mnest : medge;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const bool on = (m >> k) & 1u;
            const unsigned b = __ballot_sync(0xffffffffu, on);
            if (b) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&s_cnt[l][k], __popc(b));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (on) s_list[l][k][base + __popc(b & lt)] = (unsigned char)tid;
            }
        }
    }
    __syncthreads();
    if (tid < 3) {
        int acc = 0;
        s_pre[tid][0] = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) s_pre[tid][k + 1] = (acc += s_cnt[tid][k]);
    }
    __syncthreads();
    // FoldSurf3Points bodies
    for (int i = tid; i < s_pre[0][8]; i += kPts) {
        int k = 0;
#pragma unroll
        for (int j = 1; j < 8; ++j) k += (i >= s_pre[0][j]);
        const int p = s_list[0][k][i - s_pre[0][k]];
        const SideTable &t = tab.side[s_side[p]];
        const double s0 = s_nb[0][p];
        const double s1 = s_nb[(kSurfS1 >> (4 * k)) & 15u][p];
        const double s2 = s_nb[(kSurfS2 >> (4 * k)) & 15u][p];
        const double th = __longlong_as_double((long long)*(volatile unsigned long long *)&s_best[p]);
        const double c = surf_cand(th, s0, s1, s2, t.surf[k], t);
        if (c < th) atomicMin(&s_best[p], (unsigned long long)__double_as_longlong(c));
    }
    // nested FoldEdge2Points calls (on s1-s2 of each triangle)
    for (int i = tid; i < s_pre[1][8]; i += kPts) {
        int k = 0;
#pragma unroll
        for (int j = 1; j < 8; ++j) k += (i >= s_pre[1][j]);
        const int p = s_list[1][k][i - s_pre[1][k]];
        const SideTable &t = tab.side[s_side[p]];
        const double s1 = s_nb[(kSurfS1 >> (4 * k)) & 15u][p];
        const double s2 = s_nb[(kSurfS2 >> (4 * k)) & 15u][p];
        const double th = __longlong_as_double((long long)*(volatile unsigned long long *)&s_best[p]);
        const double c = edge_cand(th, s1, s2, t.surf[k].nest, t.F);
        if (c < th) atomicMin(&s_best[p], (unsigned long long)__double_as_longlong(c));
    }
    // outer FoldEdge2Points calls
    for (int i = tid; i < s_pre[2][8]; i += kPts) {
        int k = 0;
#pragma unroll
        for (int j = 1; j < 8; ++j) k += (i >= s_pre[2][j]);
        const int p = s_list[2][k][i - s_pre[2][k]];
        const SideTable &t = tab.side[s_side[p]];
        const double s0 = s_nb[0][p];
        const double s1 = s_nb[(kEdgeS1 >> (4 * k)) & 15u][p];
        const double th = __longlong_as_double((long long)*(volatile unsigned long long *)&s_best[p]);
        const double c = edge_cand(th, s0, s1, t.edge[k], t.F);
        if (c < th) atomicMin(&s_best[p], (unsigned long long)__double_as_longlong(c));
    }
    __syncthreads();
    double delta = 0.0;
    if (active) {
        const double tn = __longlong_as_double((long long)s_best[tid]);
        const double tnew = ((told > 0) ? 1.0 : -1.0) * tn;  // :326
        T[tgt] = tnew;
        delta = fabs(tnew - told);
    }
    if (maxd) block_max_to(delta, maxd);
}

cudaError_t launch_plane(double *T, const PlaneGeom &pg, const LocalFrameH &Lh, const DirTable *tab,
                         int variant, int src, unsigned long long *maxd, cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((pg.nu + 31) / 32, (pg.nv + 7) / 8);
    const long long off = (long long)src * pg.s_nrm;
    if (variant == kVariantCompact) {
        if (!tab) return cudaErrorInvalidValue;
        plane_kernel_compact<<<grid, kPts, 0, s>>>(T, off, pg, *tab, maxd);
        return cudaGetLastError();
    }
    if (variant == kVariantLiteral) {
        LocalFrame L;
        memcpy(&L, &Lh, sizeof(L));
        plane_kernel_literal<<<grid, block, 0, s>>>(T, off, pg, L, maxd);
    } else {
        if (!tab) return cudaErrorInvalidValue;
        plane_kernel_fast<<<grid, block, 0, s>>>(T, off, pg, *tab, maxd);
    }
    return cudaGetLastError();
}

}  // namespace fold3d
