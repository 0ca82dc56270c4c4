// fold3d_wavefront.cu -- the WAVEFRONT engine: one persistent launch per
// directional pass, tile dataflow between consecutive planes, and tiles
// skipped when their inputs did not change.
//
// Work items are (plane step p, tile t) pairs of a pass, tiles being
// 32 x kWaveTV points of a plane, numbered plane-major.  Every CTA claims the next item
// from an atomic counter.  Item (p, t) reads the source plane written by
// step p-1 only within t's 1-point halo, i.e. from the 3 x 3 tiles around t,
// so it waits for exactly those items (their completion flags), not for the
// whole previous plane: consecutive planes overlap and no plane-wide barrier
// or launch separates them.  Items are claimed in increasing order, so every
// item an item waits for is held by a CTA that is already running; the
// waits always end.  They are bounded anyway: after a time limit the CTA
// raises the status word and every CTA leaves (FOLD3D_ERR_TIMEOUT).
//
// Skipping.  A point update is min(T_old, M(nine source values, side)) (see
// fold3d_fast.cuh), so re-evaluating a tile whose source neighbourhood has
// not changed since its previous evaluation in the same direction leaves
// every target value unchanged, bit for bit.  Each orientation (plane normal
// x, y or z) keeps a map with, per plane and tile, the last pass in which any
// of its points changed; a pass writes the maps of all three orientations for
// the points it changes.  From the second sweep of a solve on, item (p, t)
// of pass e is skipped when no tile of the 3 x 3 neighbourhood of its source
// plane changed in passes e-5 .. e (the previous evaluation of that tile in
// this direction was in pass e-6, after the source plane's update of that
// pass).
//
// The change marks of earlier passes are final when a pass starts; whether
// step p-1 of the current pass changed the source plane comes with its
// completion flags, which hold (pass << 1) | changed.
//
// Synchronisation: a CTA publishes an item with __syncthreads and a
// gpu-scope release store into the item's flag; in a waiting CTA, nine
// threads poll the nine neighbour flags in parallel with acquire loads and
// then release the block with __syncthreads.  Each CTA claims its next item
// while it works on the current one.  Field values written inside the launch are read with
// L2-cached loads (ld.global.cg), never through the non-coherent read-only
// path.
#include <cstring>

#include "fold3d_ellip.cuh"
#include "fold3d_fast.cuh"
#include "fold3d_internal.h"
#include "fold3d_sync.cuh"

namespace fold3d {

namespace {

__device__ __forceinline__ double ld_cg(const double *p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg(const float *p) { return __ldcg(p); }

// Whether a stored value changes (bit patterns, so -0 vs +0 counts).
__device__ __forceinline__ bool bits_differ(double a, double b) { return __double_as_longlong(a) != __double_as_longlong(b); }
__device__ __forceinline__ bool bits_differ(float a, float b) { return __float_as_int(a) != __float_as_int(b); }

}  // namespace

constexpr int kWaveThreads = 32 * kWaveTV;

template <int MED, class R, bool LARGE> constexpr int wave_min_blocks()
{
    return LARGE ? (MED == kMediumDrift   ? FOLD3D_WAVE_MINB_LARGE_DRIFT
                    : sizeof(R) == 8      ? FOLD3D_WAVE_MINB_LARGE_ELLIP
                                          : FOLD3D_WAVE_MINB_LARGE)
                 : MED == kMediumDrift ? FOLD3D_WAVE_MINB_DRIFT
                                       : (sizeof(R) == 8 ? FOLD3D_WAVE_MINB_ELLIP : FOLD3D_WAVE_MINB_ELLIP_F32);
}

// Medium-dependent launch parameters: the drift medium's constant table, or
// the elliptical medium's direction constants and metric arrays.
template <int MED> struct WaveMedium;
template <> struct WaveMedium<kMediumDrift> {
    using type = DirTable;
};
template <> struct WaveMedium<kMediumEllip> {
    using type = EllipParam;
};

// One work item (step p, tile t) of one grid, for all threads of the CTA:
// wait for the 3 x 3 tiles of step p-1, then skip or update the tile, then
// publish its flag.  Adds each changed point's |dT| into dmax and the
// evaluated points into evaluated.  Returns false if a wait gave up (the
// item is then left unpublished and the caller must leave).
template <int MED, class R, int TV = kWaveTV>
__device__ __forceinline__ bool wave_item(R *__restrict__ T, const WaveArgs &a,
                                          const typename WaveMedium<MED>::type &tab, int item, double &dmax,
                                          unsigned long long &evaluated)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const PlaneGeom &g = a.pg;
    const int ntiles = a.ntu * a.ntv;
    const unsigned want = a.epoch << 1;  // flags hold (pass << 1) | changed
    const bool may_skip = a.epoch >= a.skip_from;
    const int p = item / ntiles, t = item - p * ntiles;
    const int tu = t % a.ntu, tv = t / a.ntu;
    const int src = a.first_src + p * a.sg;
    const int tgt = src + a.sg;

    // Threads 0..8 each watch one tile of the 3 x 3 neighbourhood: its change
    // mark from earlier passes, and its step p-1 flag (which also says whether
    // that item changed the source plane).
    int timed_out = 0, recent = 0;
    if (tid < 9) {
        const int nu = tu + tid % 3 - 1, nv = tv + tid / 3 - 1;
        if (nu >= 0 && nu < a.ntu && nv >= 0 && nv < a.ntv) {
            const int nt = nv * a.ntu + nu;
            if (may_skip) recent = (__ldcg(a.mod[a.nrm] + (long long)src * ntiles + nt) + 5u >= a.epoch);
            if (p > 0) {
                const unsigned *fl = a.flags + (long long)(p - 1) * ntiles + nt;
                const unsigned long long t0 = global_ns();
                unsigned spins = 0, f;
                while ((f = ld_acquire(fl)) < want) {
                    if (++spins > (1u << 26) || global_ns() - t0 > a.timeout_ns ||
                        *(volatile unsigned *)a.status != 0) {
                        atomicCAS(a.status, 0u, 1u);  // FOLD3D_ERR_TIMEOUT
                        timed_out = 1;
                        break;
                    }
                    if (kPollNs) __nanosleep(kPollNs);
                }
                if (!timed_out) recent |= (int)(f & 1u);
            }
        }
    }
    if (__syncthreads_or(timed_out)) return false;
    const int skip = may_skip && !__syncthreads_or(recent);

    int changed = 0;
    if (!skip) {
        const int u = tu * 32 + lane + 1;
        const int v = tv * TV + warp + 1;
        if (u <= g.nu && v <= g.nv) {
            const long long s = (long long)src * g.s_nrm + (long long)u * g.su + (long long)v * g.sv;
            const long long d = s + g.sn;
            const R st = fabs(ld_cg(T + s));
            const R xt = fabs(ld_cg(T + s + g.sx));
            const R yt = fabs(ld_cg(T + s + g.sy));
            const R xnt = fabs(ld_cg(T + s - g.sx));
            const R ynt = fabs(ld_cg(T + s - g.sy));
            const R txm = fabs(ld_cg(T + s + g.sx - g.sy));
            const R txy = fabs(ld_cg(T + s + g.sx + g.sy));
            const R tym = fabs(ld_cg(T + s - g.sx + g.sy));
            const R txnyn = fabs(ld_cg(T + s - g.sx - g.sy));
            const R told = ld_cg(T + d);
            R tnew;
            if constexpr (MED == kMediumDrift) {
                static_assert(sizeof(R) == 8, "the drift medium is solved in double");
                tnew = point_update_fast(told, st, xt, yt, xnt, ynt, txy, txm, tym, txnyn, &tab);
            } else {
                const R nb[8] = {xt, txy, yt, tym, xnt, txnyn, ynt, txm};
                int win;
                tnew = point_update_ellip(told, st, nb, ell_local<R>(tab.med, tab.dir, d), win);
                if (a.winners && bits_differ(tnew, told))
                    a.winners[d] = (win < 0) ? (unsigned char)kNoWinner : (unsigned char)(a.dir * kEllipCands + win);
            }
            if (bits_differ(tnew, told)) {
                T[d] = tnew;
                changed = 1;
                dmax = fmax(dmax, (double)fabs(tnew - told));
                // mark the point's tile in the two other orientations
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int b = (q == 0) ? a.ua : a.va;
                    const int ub = (b == 0) ? 1 : 0, vb = (b == 2) ? 1 : 2;
                    const int cb = (q == 0) ? u : v;
                    const int cu = (ub == a.nrm) ? tgt : (ub == a.ua) ? u : v;
                    const int cv = (vb == a.nrm) ? tgt : (vb == a.ua) ? u : v;
                    const int tile = ((cv - 1) / TV) * a.mod_ntu[b] + ((cu - 1) >> 5);
                    a.mod[b][(long long)cb * a.mod_ntiles[b] + tile] = a.epoch;
                }
            }
            ++evaluated;
        }
        changed = __syncthreads_or(changed);
        if (changed && tid == 0) a.mod[a.nrm][(long long)tgt * ntiles + t] = a.epoch;
    }
    // publish: the barrier makes every thread's stores precede thread 0's
    // release store, which orders them (cumulatively) before the flag
    __syncthreads();
    if (tid == 0) st_release(a.flags + item, want | (unsigned)changed);
    return true;
}

// The same work item done by one warp alone: its 32 lanes take the tile's
// rows one after the other, lanes 0..8 watch the nine neighbour flags, and
// lane 0 publishes after a __syncwarp (which orders every lane's stores
// before lane 0's release store).  The warps of a CTA each own their items,
// so none waits at a CTA barrier for the slowest row of another's.
template <int MED, class R, int TV = kWaveTV>
__device__ __forceinline__ bool wave_item_warp(R *__restrict__ T, const WaveArgs &a,
                                               const typename WaveMedium<MED>::type &tab, int item, double &dmax,
                                               unsigned long long &evaluated)
{
    const int lane = threadIdx.x & 31;
    const PlaneGeom &g = a.pg;
    const int ntiles = a.ntu * a.ntv;
    const unsigned want = a.epoch << 1;  // flags hold (pass << 1) | changed
    const bool may_skip = a.epoch >= a.skip_from;
    const int p = item / ntiles, t = item - p * ntiles;
    const int tu = t % a.ntu, tv = t / a.ntu;
    const int src = a.first_src + p * a.sg;
    const int tgt = src + a.sg;

    int timed_out = 0, recent = 0;
    if (lane < 9) {
        const int nu = tu + lane % 3 - 1, nv = tv + lane / 3 - 1;
        if (nu >= 0 && nu < a.ntu && nv >= 0 && nv < a.ntv) {
            const int nt = nv * a.ntu + nu;
            if (may_skip) recent = (__ldcg(a.mod[a.nrm] + (long long)src * ntiles + nt) + 5u >= a.epoch);
            if (p > 0) {
                const unsigned *fl = a.flags + (long long)(p - 1) * ntiles + nt;
                const unsigned long long t0 = global_ns();
                unsigned spins = 0, f;
                while ((f = ld_acquire(fl)) < want) {
                    if (++spins > (1u << 26) || global_ns() - t0 > a.timeout_ns ||
                        *(volatile unsigned *)a.status != 0) {
                        atomicCAS(a.status, 0u, 1u);  // FOLD3D_ERR_TIMEOUT
                        timed_out = 1;
                        break;
                    }
                    if (kPollNs) __nanosleep(kPollNs);
                }
                if (!timed_out) recent |= (int)(f & 1u);
            }
        }
    }
    if (__any_sync(0xffffffffu, timed_out)) return false;
    const bool skip = may_skip && !__any_sync(0xffffffffu, recent);

    int changed = 0;
    if (!skip) {
        const int u = tu * 32 + lane + 1;
        for (int r = 0; r < TV; ++r) {
            const int v = tv * TV + r + 1;
            if (u <= g.nu && v <= g.nv) {
                const long long s = (long long)src * g.s_nrm + (long long)u * g.su + (long long)v * g.sv;
                const long long d = s + g.sn;
                const R st = fabs(ld_cg(T + s));
                const R xt = fabs(ld_cg(T + s + g.sx));
                const R yt = fabs(ld_cg(T + s + g.sy));
                const R xnt = fabs(ld_cg(T + s - g.sx));
                const R ynt = fabs(ld_cg(T + s - g.sy));
                const R txm = fabs(ld_cg(T + s + g.sx - g.sy));
                const R txy = fabs(ld_cg(T + s + g.sx + g.sy));
                const R tym = fabs(ld_cg(T + s - g.sx + g.sy));
                const R txnyn = fabs(ld_cg(T + s - g.sx - g.sy));
                const R told = ld_cg(T + d);
                R tnew;
                if constexpr (MED == kMediumDrift) {
                    tnew = point_update_fast(told, st, xt, yt, xnt, ynt, txy, txm, tym, txnyn, &tab);
                } else {
                    const R nb[8] = {xt, txy, yt, tym, xnt, txnyn, ynt, txm};
                    int win;
                    tnew = point_update_ellip(told, st, nb, ell_local<R>(tab.med, tab.dir, d), win);
                    if (a.winners && bits_differ(tnew, told))
                        a.winners[d] =
                            (win < 0) ? (unsigned char)kNoWinner : (unsigned char)(a.dir * kEllipCands + win);
                }
                if (bits_differ(tnew, told)) {
                    T[d] = tnew;
                    changed = 1;
                    dmax = fmax(dmax, (double)fabs(tnew - told));
#pragma unroll
                    for (int q = 0; q < 2; ++q) {  // the point's tile in the two other orientations
                        const int b = (q == 0) ? a.ua : a.va;
                        const int ub = (b == 0) ? 1 : 0, vb = (b == 2) ? 1 : 2;
                        const int cb = (q == 0) ? u : v;
                        const int cu = (ub == a.nrm) ? tgt : (ub == a.ua) ? u : v;
                        const int cv = (vb == a.nrm) ? tgt : (vb == a.ua) ? u : v;
                        const int tile = ((cv - 1) / TV) * a.mod_ntu[b] + ((cu - 1) >> 5);
                        a.mod[b][(long long)cb * a.mod_ntiles[b] + tile] = a.epoch;
                    }
                }
                ++evaluated;
            }
        }
        changed = __any_sync(0xffffffffu, changed);
        if (changed && lane == 0) a.mod[a.nrm][(long long)tgt * ntiles + t] = a.epoch;
    }
    __syncwarp();
    if (lane == 0) st_release(a.flags + item, want | (unsigned)changed);
    return true;
}

// Block-wide maximum of d into *out (IEEE bits) and sum of e into *sum.
template <int TV = kWaveTV>
__device__ __forceinline__ void wave_flush(double d, unsigned long long e, unsigned long long *out,
                                           unsigned long long *sum)
{
    __shared__ double wmax[TV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if (lane == 0) {
        wmax[warp] = d;
        if (e) atomicAdd(sum, e);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < TV; ++w) m = fmax(m, wmax[w]);
        if (m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
}

template <int MED, class R, bool LARGE>
__global__ void __launch_bounds__(kWaveThreads, (wave_min_blocks<MED, R, LARGE>()))
    wave_pass_kernel(R *__restrict__ T, WaveArgs a, const __grid_constant__ typename WaveMedium<MED>::type tab)
{
    __shared__ int s_next;
    const long long total = (long long)a.steps * a.ntu * a.ntv;
    double dmax = 0.0;
    unsigned long long evaluated = 0;
    if constexpr (kWaveWarpItems && LARGE && MED == kMediumDrift) {
        // drift medium, large planes: every warp claims and processes its own
        // items (wave_item_warp).  A plane then has enough tiles to keep all
        // warps busy, and no warp waits at a CTA barrier for another's row.
        // On smaller planes the plane-to-plane chain binds instead, and an
        // item shared by the CTA's warps (each one row) finishes sooner; the
        // elliptical medium's larger per-point state made warp items slower
        // on large planes too (measured).
        const int lane = threadIdx.x & 31;
        int item = -1;
        if (lane == 0) {
            const unsigned w = atomicAdd(a.work, 1u);
            item = (w < total) ? (int)w : -1;
        }
        item = __shfl_sync(0xffffffffu, item, 0);
        while (item >= 0) {
            int next = -1;  // claimed now, processed after this one
            if (lane == 0 && *(volatile unsigned *)a.status == 0) {
                const unsigned w = atomicAdd(a.work, 1u);
                if (w < total) next = (int)w;
            }
            next = __shfl_sync(0xffffffffu, next, 0);
            if (!wave_item_warp<MED, R>(T, a, tab, item, dmax, evaluated)) break;
            item = next;
        }
        wave_flush(dmax, evaluated, a.maxd, a.evaluated);
        return;
    }
    if (threadIdx.x == 0) {
        const unsigned w = atomicAdd(a.work, 1u);
        s_next = (w < total) ? (int)w : -1;
    }
    __syncthreads();
    for (;;) {
        const int item = s_next;
        if (item < 0) break;
        __syncthreads();  // every thread has read s_next
        if (threadIdx.x == 0) {  // claim the next item now; it is processed after this one
            int it = -1;
            if (*(volatile unsigned *)a.status == 0) {
                const unsigned w = atomicAdd(a.work, 1u);
                if (w < total) it = (int)w;
            }
            s_next = it;
        }
        if (!wave_item<MED, R>(T, a, tab, item, dmax, evaluated)) break;
    }
    wave_flush(dmax, evaluated, a.maxd, a.evaluated);
}

// ---------------------------------------------------------------------------
// Batched passes: the items of one pass of many independent grids (the
// elliptical medium) in one launch.  Items are ordered step-major across the
// instances (step p of every instance that has one, then step p+1), the
// instances sorted by their number of steps, so that the active instances of
// a step are a prefix of the list; every item's predecessors (step p-1 of the
// same instance) come earlier in that order, and the launch's claimed items
// spread over many instances at once.
// ---------------------------------------------------------------------------
// Resident CTAs per SM the batched kernel is compiled for, by tile height:
// the same register budget per thread (65536 / (128 * 8)) for every height.
template <int TV> constexpr int batch_min_blocks() { return FOLD3D_WAVE_MINB_BATCH * kWaveTV / TV; }

template <class R, int TV>
__global__ void __launch_bounds__(32 * TV, batch_min_blocks<TV>()) batch_pass_kernel(BatchArgs b)
{
    // A CTA claims kBatchChunk consecutive items at a time, and the first
    // lanes of warp 0 locate them in parallel (two binary searches each over
    // the launch's tables): consecutive items mostly belong to one instance
    // (its tiles of a step come together), so the instance is staged once for
    // several items, and the searches' dependent loads are paid once per
    // chunk.  Claims stay in increasing order and a chunk's items run in
    // order, so the lowest unfinished item always runs and every wait ends.
    __shared__ int s_next;  // first item of the CTA's next chunk, -1 for none
    __shared__ int s_loc[kBatchChunk][2];
    __shared__ int s_n;     // items of the current chunk
    __shared__ int s_cur;   // the active slot staged in s_inst, -1 for none
    __shared__ BatchInst s_inst;
    const unsigned total = *b.total;
    if (threadIdx.x == 0) {
        const unsigned w = atomicAdd(b.work, (unsigned)kBatchChunk);
        s_next = (w < total) ? (int)w : -1;
        s_n = 0;
        s_cur = -1;
    }
    __syncthreads();
    // The instance stays staged, and its largest change and evaluated points
    // are flushed only when the CTA moves to another one.
    double dmax = 0.0;
    unsigned long long evaluated = 0;
    for (int q = 0;; ++q) {
        if (q == s_n) {  // the same for every thread
            const int c0 = s_next;
            if (c0 < 0) break;
            __syncthreads();  // every thread has read s_n and s_next
            if (threadIdx.x < 32) {
                const int n = (int)min((unsigned)kBatchChunk, total - (unsigned)c0);
                if ((int)threadIdx.x < n)
                    batch_locate(b.step_off, b.step_k, b.tile_pre, b.max_steps, c0 + (int)threadIdx.x,
                                 s_loc[threadIdx.x][0], s_loc[threadIdx.x][1]);
                if (threadIdx.x == 0) {
                    int it = -1;
                    if (*(volatile unsigned *)b.status == 0) {
                        const unsigned w = atomicAdd(b.work, (unsigned)kBatchChunk);
                        if (w < total) it = (int)w;
                    }
                    s_next = it;
                    s_n = n;
                }
            }
            __syncthreads();
            q = 0;
        }
        const int slot = s_loc[q][0];
        if (slot != s_cur) {  // the same for every thread
            if (s_cur >= 0) {
                wave_flush<TV>(dmax, evaluated, s_inst.a.maxd, s_inst.a.evaluated);
                dmax = 0.0;
                evaluated = 0;
            }
            const unsigned *src = reinterpret_cast<const unsigned *>(b.inst + b.act[slot]);
            unsigned *dst = reinterpret_cast<unsigned *>(&s_inst);
            for (int w = threadIdx.x; w < (int)(sizeof(BatchInst) / 4); w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            if (threadIdx.x == 0) {  // the pass number is per launch, not per staged instance
                s_inst.a.epoch = *b.epoch_base + (unsigned)b.dir + 1u;
                s_inst.a.skip_from = b.skip_from;
                s_cur = slot;
            }
            __syncthreads();
        }
        if (!wave_item<kMediumEllip, R, TV>(static_cast<R *>(s_inst.T), s_inst.a, s_inst.p, s_loc[q][1], dmax,
                                            evaluated))
            break;
    }
    if (s_cur >= 0) wave_flush<TV>(dmax, evaluated, s_inst.a.maxd, s_inst.a.evaluated);
}

// The batch's state after a sweep and the next sweep's tables (BatchCtl).
// One block: the instances are folded in parallel, then one thread per
// direction rebuilds that direction's tables (a few thousand steps).
__global__ void __launch_bounds__(256) batch_restage_kernel(BatchCtl c, int first)
{
    __shared__ int s_left;
    if (threadIdx.x == 0) s_left = 0;
    __syncthreads();
    if (first) {
        for (int i = threadIdx.x; i < c.n; i += blockDim.x) {
            c.active[i] = 1;
            c.sweeps[i] = 0;
            c.delta[i] = 0.0;
            c.maxd[i] = 0ull;
        }
        if (threadIdx.x == 0) {
            *c.epoch_base = c.epoch0;
            c.sweep[0] = 0;
            c.sweep[1] = c.n;
        }
    } else {
        int left = 0;
        for (int i = threadIdx.x; i < c.n; i += blockDim.x) {
            if (c.active[i]) {
                c.sweeps[i] += 1;
                const double d = __longlong_as_double((long long)c.maxd[i]);
                c.delta[i] = d;
                if (!c.fixed && d <= c.tol) c.active[i] = 0;
                else ++left;
            }
            c.maxd[i] = 0ull;
        }
        atomicAdd(&s_left, left);
    }
    __syncthreads();
    if (!first && threadIdx.x == 0) {
        *c.epoch_base += 6u;
        c.sweep[0] += 1;
        c.sweep[1] = s_left;
    }
    if (threadIdx.x < 6) c.total[threadIdx.x] = batch_tables(c.dir[threadIdx.x], c.active, c.n, c.max_steps);
    if (!first && threadIdx.x == 0) {
        const int more = (*(volatile const unsigned *)c.status == 0) && c.sweep[0] < c.max_sweeps && s_left > 0;
        cudaGraphSetConditional((cudaGraphConditionalHandle)c.cond, more ? 1u : 0u);
    }
}

cudaError_t launch_batch_restage(const BatchCtl &ctl, bool first, cudaStream_t s)
{
    batch_restage_kernel<<<1, 256, 0, s>>>(ctl, first ? 1 : 0);
    return cudaGetLastError();
}

template <int TV> static cudaError_t launch_batch_tv(const BatchArgs &b, bool f32, int grid, cudaStream_t s)
{
    if (f32) batch_pass_kernel<float, TV><<<grid, 32 * TV, 0, s>>>(b);
    else batch_pass_kernel<double, TV><<<grid, 32 * TV, 0, s>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_batch_pass(const BatchArgs &b, bool f32, int tv, int grid, cudaStream_t s)
{
    switch (tv) {
    case 2: return launch_batch_tv<2>(b, f32, grid, s);
    case 4: return launch_batch_tv<4>(b, f32, grid, s);
    case 8: return launch_batch_tv<8>(b, f32, grid, s);
    default: return cudaErrorInvalidValue;
    }
}

template <int TV> static int batch_occupancy(bool f32)
{
    int n = 0;
    const cudaError_t e =
        f32 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_pass_kernel<float, TV>, 32 * TV, 0)
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_pass_kernel<double, TV>, 32 * TV, 0);
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

int batch_blocks_per_sm(bool f32, int tv)
{
    return tv == 2 ? batch_occupancy<2>(f32) : tv == 8 ? batch_occupancy<8>(f32) : batch_occupancy<4>(f32);
}

cudaError_t launch_wave_pass(double *T, const WaveArgs &a, const DirTable &tab, int grid, cudaStream_t s, bool large)
{
    if (large) wave_pass_kernel<kMediumDrift, double, true><<<grid, kWaveThreads, 0, s>>>(T, a, tab);
    else wave_pass_kernel<kMediumDrift, double, false><<<grid, kWaveThreads, 0, s>>>(T, a, tab);
    return cudaGetLastError();
}

cudaError_t launch_wave_pass_ellip(void *T, bool f32, const WaveArgs &a, const EllipParam &p, int grid, cudaStream_t s,
                                   bool large)
{
    float *tf = static_cast<float *>(T);
    double *td = static_cast<double *>(T);
    if (f32) {
        if (large) wave_pass_kernel<kMediumEllip, float, true><<<grid, kWaveThreads, 0, s>>>(tf, a, p);
        else wave_pass_kernel<kMediumEllip, float, false><<<grid, kWaveThreads, 0, s>>>(tf, a, p);
    } else {
        if (large) wave_pass_kernel<kMediumEllip, double, true><<<grid, kWaveThreads, 0, s>>>(td, a, p);
        else wave_pass_kernel<kMediumEllip, double, false><<<grid, kWaveThreads, 0, s>>>(td, a, p);
    }
    return cudaGetLastError();
}

template <class K> static int occupancy(K kernel)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kWaveThreads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

int wave_blocks_per_sm(int medium, bool f32, bool large)
{
    if (medium != kMediumEllip)
        return large ? occupancy(wave_pass_kernel<kMediumDrift, double, true>)
                     : occupancy(wave_pass_kernel<kMediumDrift, double, false>);
    if (f32)
        return large ? occupancy(wave_pass_kernel<kMediumEllip, float, true>)
                     : occupancy(wave_pass_kernel<kMediumEllip, float, false>);
    return large ? occupancy(wave_pass_kernel<kMediumEllip, double, true>)
                 : occupancy(wave_pass_kernel<kMediumEllip, double, false>);
}

}  // namespace fold3d
