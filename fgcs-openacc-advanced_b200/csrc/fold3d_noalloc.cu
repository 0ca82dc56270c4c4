// fold3d_noalloc.cu -- a whole solve that allocates no memory.
//
// Some callers cannot let a library allocate device memory behind their
// back: a host program whose device memory is handed out by another runtime
// (an OpenACC driver that owns every device buffer through acc_malloc, or a
// framework whose caching allocator has already reserved the GPU's memory),
// or a plugin host that only lends buffers to the plugins it loads and
// budgets every byte.  fold3d_solve_noalloc serves them: it runs the same
// per-plane kernels as fold3d_solve, needs no context, and calls no
// cudaMalloc, cudaFree, graph or event routine.
//
// Its only scratch is g_sweep_maxd below, a file-scope device array of
// FOLD3D_NOALLOC_MAX_SWEEPS 8-byte slots (32 KiB) that every GPU which loads
// the library holds until the process exits.  Slot s receives the largest
// |T_after - T_before| of sweep s of the current call.  Calls share the array
// and it keeps the last call's values, so each sweep clears its own slot on
// the stream before its first plane; two calls whose work overlaps on the GPU
// (different streams, or different host threads, on one device) race on it.
//
// Host code cannot use g_sweep_maxd's name as a device address.  The first
// call on a device looks the address up with cudaGetSymbolAddress, with that
// device current, and keeps it for later calls; that first call should
// therefore come before any stream capture that involves this library.
#include <chrono>
#include <cstring>
#include <mutex>

#include "fold3d_fast.cuh"
#include "fold3d_internal.h"

namespace fold3d {

static __device__ __align__(256) unsigned long long g_sweep_maxd[FOLD3D_NOALLOC_MAX_SWEEPS];

namespace {
constexpr int kMaxDevices = 128;
std::mutex g_noalloc_mu;
unsigned long long *g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_sweep_maxd on the current device (set up once per device).
int noalloc_scratch(int dev, unsigned long long **out)
{
    if (dev < 0 || dev >= kMaxDevices) return set_error(FOLD3D_ERR_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sweep_maxd);
        if (e != cudaSuccess || !p) return cuda_error(e, "cudaGetSymbolAddress(g_sweep_maxd)");
        g_noalloc_ptr[dev] = (unsigned long long *)p;
    }
    *out = g_noalloc_ptr[dev];
    return FOLD3D_OK;
}
}  // namespace

}  // namespace fold3d

using namespace fold3d;

extern "C" int fold3d_solve_noalloc(const fold3d_grid *g, const fold3d_medium *m, double *T,
                                    const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    clear_error();
    if (!g || !m || !T || !o) return set_error(FOLD3D_ERR_INVALID, "NULL argument");
    if (g->nx < 2 || g->ny < 2 || g->nz < 2 || !(g->dx > 0 && g->dy > 0 && g->dz > 0))
        return set_error(FOLD3D_ERR_INVALID, "grid sizes must be >= 2 and spacings > 0");
    if (!(m->F > 0)) return set_error(FOLD3D_ERR_INVALID, "medium must have F > 0");
    if (o->max_sweeps < 1) return set_error(FOLD3D_ERR_INVALID, "max_sweeps must be >= 1");
    if (o->max_sweeps > FOLD3D_NOALLOC_MAX_SWEEPS)
        return set_error(FOLD3D_ERR_INVALID,
                         "fold3d_solve_noalloc: max_sweeps exceeds FOLD3D_NOALLOC_MAX_SWEEPS (4096), the size of "
                         "its static per-sweep scratch; use fold3d_solve for longer solves");
    if (!o->fixed && !(o->tol >= 0.0)) return set_error(FOLD3D_ERR_INVALID, "tol must be >= 0");
    if (o->variant != kVariantFast && o->variant != kVariantLiteral && o->variant != kVariantCompact)
        return set_error(FOLD3D_ERR_INVALID, "unknown solver variant");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    unsigned long long *slots = nullptr;
    int rc = noalloc_scratch(dev, &slots);
    if (rc) return rc;

    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = (cudaStream_t)stream;
    DirTable tab;  // one direction's constants at a time (4.6 KiB of host stack)
    int sweeps = 0;
    unsigned long long bits = 0;
    while (sweeps < o->max_sweeps) {
        unsigned long long *slot = slots + sweeps;
        if ((e = cudaMemsetAsync(slot, 0, sizeof *slot, s)) != cudaSuccess) return cuda_error(e, "cudaMemsetAsync");
        for (int d = 0; d < 6; ++d) {
            const PlaneGeom pg = make_geom(*g, d);
            const LocalFrameH L = make_frame(*g, *m, d);
            build_dir_table(L, tab, false);  // no search: it would allocate
            int src = pass_first(pg, d);
            for (int p = 0; p < pass_count(pg); ++p, src += kDirs[d].sg)
                if ((e = launch_plane(T, pg, L, &tab, o->variant, src, slot, s)) != cudaSuccess)
                    return cuda_error(e, "plane launch");
        }
        ++sweeps;
        if (!o->fixed) {
            if ((e = cudaMemcpyAsync(&bits, slot, sizeof bits, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
                return cuda_error(e, "cudaMemcpyAsync");
            if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "sweep");
            double delta;
            memcpy(&delta, &bits, sizeof delta);
            if (delta <= o->tol) break;
        }
    }
    if ((e = cudaMemcpyAsync(&bits, slots + sweeps - 1, sizeof bits, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_error(e, "cudaMemcpyAsync");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "solve");
    if (rep) {
        const uint64_t nx = g->nx, ny = g->ny, nz = g->nz;
        memcpy(&rep->max_delta, &bits, sizeof bits);
        rep->sweeps = sweeps;
        rep->elapsed_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        rep->nominal_updates = (uint64_t)sweeps * 2 * ((nx - 1) * ny * nz + (ny - 1) * nx * nz + (nz - 1) * nx * ny);
        rep->evaluated_updates = rep->nominal_updates;
        rep->engine = FOLD3D_ENGINE_PLANES;
    }
    return FOLD3D_OK;
}
