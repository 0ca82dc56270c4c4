// fold3d_init_dev.cu -- ImplicitInitialiser (Stencil-OpenACC/Fold3dPMM.c:129-389)
// into a device field.  The reference's initialiser is host-only.
//
// The implicit surface is sampled on the host, where sin and cos are the
// reference's own (glibc): the crossing points depend on those bits.  It goes
// to the device in slabs of node planes through two pinned buffers, the copy
// of one slab overlapping the sampling of the next.  The seeding runs on the
// GPU, one thread per voxel, with the host's code (fold3d_seed.h).  A node
// update is a minimum of |T| that keeps the node's sign, and the sign is the
// surface's (T < 0 where the surface is <= 0); for non-negative doubles the
// order of the bit patterns is the numeric one, so an atomicMin on the bits
// of |T| gives the host's result, bit for bit, in any order.
#include <algorithm>
#include <vector>

#include "fold3d_internal.h"
#include "fold3d_seed.h"

namespace fold3d {

namespace {

__constant__ fold3d_seed::NodeStep c_steps[fold3d_seed::kNodeSteps] = FOLD3D_SEED_STEPS;
__constant__ fold3d_seed::Blend c_blends[fold3d_seed::kBlendCount] = FOLD3D_SEED_BLENDS;

// InitNode (Fold3dPMM.c:35-54) as an atomic minimum on |T| (bits in A).
struct DevNode {
    unsigned long long *A;
    const double *IF;
    long long sy, sz;
    double F, a[3];

    __device__ void operator()(double x, double y, double z, int i, int j, int k) const
    {
        const long long id = i + sy * j + sz * k;
        double ax = a[0], ay = a[1], az = a[2];
        if (!(IF[id] > 0)) {  // the node's time is negative
            ax *= -1;
            ay *= -1;
            az *= -1;
        }
        const double tn = fold3d_seed::exact_time(F, ax, ay, az, -x, -y, -z);
        atomicMin(A + id, (unsigned long long)__double_as_longlong(tn));
    }
};

__global__ void seed_fill_kernel(unsigned long long *A, long long cells)
{
    const unsigned long long m = (unsigned long long)__double_as_longlong(fold3d_seed::kMaxT);
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < cells;
         x += (long long)gridDim.x * blockDim.x)
        A[x] = m;
}

__global__ void __launch_bounds__(256) seed_voxels_kernel(const double *__restrict__ IF, unsigned long long *A, int nx,
                                                          int ny, int nz, double hx, double hy, double hz, double F,
                                                          double ax, double ay, double az)
{
    const long long sy = nx + 2, sz = sy * (ny + 2);
    const long long vx = nx - 1, vy = ny - 1, nvox = vx * vy * (nz - 1);
    DevNode node{A, IF, sy, sz, F, {ax, ay, az}};
    const double h[3] = {hx, hy, hz};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox;
         v += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(v % vx) + 1, j = (int)((v / vx) % vy) + 1, k = (int)(v / (vx * vy)) + 1;
        fold3d_seed::seed_voxel(IF, sy, sz, h, i, j, k, c_steps, c_blends, node);
    }
}

// T = sign(surface) * |T| in place over the bits of |T|.
__global__ void seed_sign_kernel(const double *__restrict__ IF, double *T, long long cells)
{
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < cells;
         x += (long long)gridDim.x * blockDim.x) {
        const double a = __longlong_as_double((long long)reinterpret_cast<unsigned long long *>(T)[x]);
        T[x] = (fold3d_seed::side(IF[x]) * 1.0) * a;
    }
}

}  // namespace

int init_implicit_device(const fold3d_grid &g, const fold3d_medium &m, double *T, double *IF_dev,
                         double *stage[2], size_t stage_planes, cudaStream_t s)
{
    const long long sy = g.nx + 2, sz = sy * (g.ny + 2), cells = sz * (g.nz + 2);
    const int nth = init_threads();
    SurfaceTables tabs;
    if (!surface_tables(g, tabs, nth)) return set_error(FOLD3D_ERR_NOMEM, "surface tables");
    cudaEvent_t done[2];
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2; ++b)
        if ((e = cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming)) != cudaSuccess)
            return cuda_error(e, "cudaEventCreate");
    bool used[2] = {false, false};
    int b = 0;
    for (int k0 = 0; k0 < g.nz + 2 && e == cudaSuccess; k0 += (int)stage_planes, b ^= 1) {
        const int k1 = std::min(g.nz + 2, k0 + (int)stage_planes);
        if (used[b] && (e = cudaEventSynchronize(done[b])) != cudaSuccess) break;  // its last copy is done
        surface_planes(stage[b], g, k0, k1, tabs, nth);
        if ((e = cudaMemcpyAsync(IF_dev + sz * k0, stage[b], (size_t)sz * (k1 - k0) * sizeof(double),
                                 cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaEventRecord(done[b], s)) != cudaSuccess)
            break;
        used[b] = true;
    }
    unsigned long long *A = reinterpret_cast<unsigned long long *>(T);
    if (e == cudaSuccess) {
        seed_fill_kernel<<<148 * 8, 256, 0, s>>>(A, cells);
        seed_voxels_kernel<<<148 * 16, 256, 0, s>>>(IF_dev, A, g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, m.F, m.ax, m.ay,
                                                     m.az);
        seed_sign_kernel<<<148 * 8, 256, 0, s>>>(IF_dev, T, cells);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    for (int q = 0; q < 2; ++q) cudaEventDestroy(done[q]);
    return e == cudaSuccess ? FOLD3D_OK : cuda_error(e, "device initialiser");
}

}  // namespace fold3d
