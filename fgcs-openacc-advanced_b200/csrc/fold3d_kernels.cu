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

cudaError_t launch_plane(double *T, const PlaneGeom &pg, const LocalFrameH &Lh, const DirTable *tab,
                         int variant, int src, unsigned long long *maxd, cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((pg.nu + 31) / 32, (pg.nv + 7) / 8);
    const long long off = (long long)src * pg.s_nrm;
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
