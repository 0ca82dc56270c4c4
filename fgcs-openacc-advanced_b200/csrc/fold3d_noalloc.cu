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
// Host code cannot use g_sweep_maxd's name as a device address.  Its address
// is looked up with cudaGetSymbolAddress, with the caller's device and
// context current, by the first call in each CUDA context, and kept for later
// calls in that context.  The cache is keyed on the context's unique id
// (cuCtxGetId), not on the device ordinal: after cudaDeviceReset, or when a
// caller makes another context current on the same device (an OpenACC
// runtime with its own context, say), the module is loaded again at another
// address and the next call looks it up afresh.  That first call in a
// context should come before any stream capture that involves this library.
#include <chrono>
#include <cstring>
#include <cuda.h>
#include <mutex>

#include "fold3d_fast.cuh"
#include "fold3d_internal.h"

namespace fold3d {

static __device__ __align__(256) unsigned long long g_sweep_maxd[FOLD3D_NOALLOC_MAX_SWEEPS];

namespace {
std::mutex g_noalloc_mu;

// Driver entry points, fetched through the runtime (the library does not
// link libcuda itself).
using CtxGetCurrentFn = CUresult(CUDAAPI *)(CUcontext *);
using CtxGetIdFn = CUresult(CUDAAPI *)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

// Contexts seen so far and g_sweep_maxd's address in each; a fixed table
// (no allocation), the oldest entry replaced when it is full.
constexpr int kCacheSlots = 64;
struct ScratchEntry {
    unsigned long long ctx_id;
    unsigned long long *ptr;
};
ScratchEntry g_cache[kCacheSlots];
int g_cache_used = 0, g_cache_next = 0;

int driver_entry_points()
{
    if (g_ctx_current && g_ctx_id) return FOLD3D_OK;
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
    if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDriverEntryPoint");
    if (!f1 || !f2 || q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess)
        return set_error(FOLD3D_ERR_UNSUPPORTED, "fold3d_solve_noalloc: the driver lacks cuCtxGetId");
    g_ctx_current = (CtxGetCurrentFn)f1;
    g_ctx_id = (CtxGetIdFn)f2;
    return FOLD3D_OK;
}

// Device address of g_sweep_maxd in the current context (looked up once per
// context).
int noalloc_scratch(unsigned long long **out)
{
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    int rc = driver_entry_points();
    if (rc) return rc;
    CUcontext ctx = nullptr;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS)
        return set_error(FOLD3D_ERR_CUDA, "fold3d_solve_noalloc: cuCtxGetCurrent failed");
    unsigned long long id = 0;
    void *p = nullptr;
    cudaError_t e;
    if (ctx) {
        if (g_ctx_id(ctx, &id) != CUDA_SUCCESS)
            return set_error(FOLD3D_ERR_CUDA, "fold3d_solve_noalloc: cuCtxGetId failed");
        for (int i = 0; i < g_cache_used; ++i)
            if (g_cache[i].ctx_id == id) {
                *out = g_cache[i].ptr;
                return FOLD3D_OK;
            }
    }
    // first call in this context (or no context bound yet: the lookup
    // initialises the runtime's primary context of the current device)
    if ((e = cudaGetSymbolAddress(&p, g_sweep_maxd)) != cudaSuccess || !p)
        return cuda_error(e, "cudaGetSymbolAddress(g_sweep_maxd)");
    if (!ctx) {
        if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx || g_ctx_id(ctx, &id) != CUDA_SUCCESS)
            return set_error(FOLD3D_ERR_CUDA, "fold3d_solve_noalloc: no current CUDA context");
    }
    const int slot = (g_cache_used < kCacheSlots) ? g_cache_used++ : g_cache_next++ % kCacheSlots;
    g_cache[slot] = ScratchEntry{id, (unsigned long long *)p};
    *out = (unsigned long long *)p;
    return FOLD3D_OK;
}
}  // namespace

}  // namespace fold3d

using namespace fold3d;

namespace {
int solve_noalloc(const fold3d_grid *g, const fold3d_medium *m, double *T, const fold3d_opts *o, void *stream,
                  fold3d_report *rep)
{
    if (!T || !o) return set_error(FOLD3D_ERR_INVALID, "NULL argument");
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_medium(m))) return rc;
    if (o->max_sweeps < 1) return set_error(FOLD3D_ERR_INVALID, "max_sweeps must be >= 1");
    if (o->max_sweeps > FOLD3D_NOALLOC_MAX_SWEEPS)
        return set_error(FOLD3D_ERR_INVALID,
                         "fold3d_solve_noalloc: max_sweeps exceeds FOLD3D_NOALLOC_MAX_SWEEPS (4096), the size of "
                         "its static per-sweep scratch; use fold3d_solve for longer solves");
    if (!o->fixed && !(o->tol >= 0.0)) return set_error(FOLD3D_ERR_INVALID, "tol must be >= 0");
    if (o->variant != kVariantFast && o->variant != kVariantLiteral && o->variant != kVariantCompact)
        return set_error(FOLD3D_ERR_INVALID, "unknown solver variant");
    unsigned long long *slots = nullptr;
    if ((rc = noalloc_scratch(&slots))) return rc;
    cudaError_t e;

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
}  // namespace

extern "C" int fold3d_solve_noalloc(const fold3d_grid *g, const fold3d_medium *m, double *T,
                                    const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    clear_error();
    return host_guard([&] { return solve_noalloc(g, m, T, o, stream, rep); });
}
