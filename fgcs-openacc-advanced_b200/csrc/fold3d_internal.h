// fold3d_internal.h -- shared declarations of the library's translation units.
#pragma once

#include <functional>
#include <new>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "fold3dpmm.h"

namespace fold3d {

// One row per reference sweep function in the driver's order
// (AN_ISO_1_OpenACC.c:1195-1236).  nrm: axis normal to the planes; sg = +1
// when the target plane is src+1; (xa, xs) and (ya, ys): axis and sign of the
// local x and y neighbours (xt, yt).  The local drift is
// (xs*a[xa], ys*a[ya], sg*a[nrm]) and the spacings (h[nrm], h[xa], h[ya]).
struct DirSpec {
    int nrm, sg, xa, xs, ya, ys;
};
extern const DirSpec kDirs[6];

// In-plane geometry of one direction on one grid (all strides in elements).
struct PlaneGeom {
    long long sn;       // target = source + sn
    long long sx, sy;   // signed strides of the local x / y neighbours
    long long su, sv;   // strides of the two in-plane axes, u the faster one
    long long s_nrm;    // unsigned stride along the plane normal
    int nu, nv;         // interior extents along u and v
    int nplanes;        // extent along the normal
};

struct LocalFrameH {  // host mirror of fold3d::LocalFrame (same layout)
    double F, ax, ay, az, hz, hx, hy, hxy, hxz, hyz;
};

PlaneGeom make_geom(const fold3d_grid &g, int dir);
LocalFrameH make_frame(const fold3d_grid &g, const fold3d_medium &m, int dir);

// Source plane indices of a pass, in the reference's order.
inline int pass_first(const PlaneGeom &pg, int dir) { return kDirs[dir].sg > 0 ? 1 : pg.nplanes; }
inline int pass_count(const PlaneGeom &pg) { return pg.nplanes - 1; }

// Error recording (thread-local message readable by fold3d_last_error).
int set_error(int code, const char *msg);
int set_errorf(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int cuda_error(cudaError_t e, const char *what);
void clear_error();

// Runs an entry point's body: a host exception (an allocation that failed,
// a mutex that could not be locked) becomes a status code instead of
// crossing the C boundary.  Recording the error allocates nothing.
template <class Fn> int host_guard(Fn &&fn)
{
    try {
        return fn();
    } catch (const std::bad_alloc &) {
        return set_error(FOLD3D_ERR_NOMEM, "out of host memory");
    } catch (...) {
        return set_error(FOLD3D_ERR_INVALID, "unexpected host error");
    }
}

// Argument checks shared by the solve entry points (fold3d_api.cu): a grid
// with sizes >= 2, finite spacings > 0 and a bounded size; a finite drift
// medium with F > 0.  FOLD3D_OK, or FOLD3D_ERR_INVALID with the message set.
int check_grid(const fold3d_grid *g);
int check_medium(const fold3d_medium *m);

// Pitch of the reference's host helpers InitNode and updateVoxel, which take
// no size (the reference compiles HEIGHT in): the grid of
// fold3d_compat_set_grid if set, else the grid of the last
// ImplicitInitialiser call.  false (error message set) when neither is known.
void compat_note_host_grid(int nx, int ny, int nz);
bool compat_host_pitch(long long &sy, long long &sz);

struct DirTable;  // fold3d_fast.cuh

// Per-direction solver constants, evaluated on the host (fold3d_tables.cpp).
// The direction table of a frame.  search: prove the tight skip bounds (a
// host search, memoised per thread); false: closed-form bounds only, with
// no memory allocated (fold3d_solve_noalloc).
void build_dir_table(const LocalFrameH &L, DirTable &out, bool search = true);

// Solver variants of the plane kernel.
enum Variant {
    kVariantFast = 0,     // host-folded constants (fold3d_fast.cuh), the default
    kVariantLiteral = 1,  // the reference's expressions point by point (fold3d_solver.cuh)
    kVariantCompact = 2   // host-folded constants, solver calls compacted across the block
};

// WAVEFRONT tiles are 32 points along the plane's faster axis by
// FOLD3D_WAVE_TV rows; one CTA of 32*FOLD3D_WAVE_TV threads works on a tile.
// Pause between two polls of a dependency flag (ns; 0 polls back to back).
#ifndef FOLD3D_POLL_NS
#define FOLD3D_POLL_NS 32
#endif
constexpr unsigned kPollNs = FOLD3D_POLL_NS;

// Single-solve dataflow passes over large planes: each warp owns whole items
// (1), or the CTA's warps share each item's rows (0); build option.
#ifndef FOLD3D_WAVE_WARP_ITEMS
#define FOLD3D_WAVE_WARP_ITEMS 1
#endif
constexpr bool kWaveWarpItems = FOLD3D_WAVE_WARP_ITEMS != 0;

// Items a batched pass's CTA claims at a time (1..32); build option.
#ifndef FOLD3D_BATCH_CHUNK
#define FOLD3D_BATCH_CHUNK 4
#endif
constexpr int kBatchChunk = FOLD3D_BATCH_CHUNK;
static_assert(kBatchChunk >= 1 && kBatchChunk <= 32, "batch chunk");

#ifndef FOLD3D_WAVE_TV
#define FOLD3D_WAVE_TV 4
#endif
constexpr int kWaveTV = FOLD3D_WAVE_TV;

// Resident CTAs per SM the forward dataflow kernels are compiled for (their
// register budget is 65536 / (32 * kWaveTV * this)); build options, each the
// count that measured fastest with 32 x 4 tiles: drift 7 (512^3) and 7 on
// planes of kLargePlaneTiles tiles or more (1280^3, warp-owned items; 8:
// 2% slower, 6: 4% slower); the FP64 elliptical medium 6, and 7 on large
// planes; the float32 one 8; batched solves (many small instances) 8.
#ifndef FOLD3D_WAVE_MINB_DRIFT
#define FOLD3D_WAVE_MINB_DRIFT 7
#endif
#ifndef FOLD3D_WAVE_MINB_ELLIP
#define FOLD3D_WAVE_MINB_ELLIP 6
#endif
#ifndef FOLD3D_WAVE_MINB_ELLIP_F32
#define FOLD3D_WAVE_MINB_ELLIP_F32 8
#endif
#ifndef FOLD3D_WAVE_MINB_BATCH
#define FOLD3D_WAVE_MINB_BATCH 8
#endif
#ifndef FOLD3D_WAVE_MINB_LARGE
#define FOLD3D_WAVE_MINB_LARGE 8  // large planes, float32 elliptical medium
#endif
#ifndef FOLD3D_WAVE_MINB_LARGE_DRIFT
#define FOLD3D_WAVE_MINB_LARGE_DRIFT 7
#endif
#ifndef FOLD3D_WAVE_MINB_LARGE_ELLIP
#define FOLD3D_WAVE_MINB_LARGE_ELLIP 7
#endif
#ifndef FOLD3D_WAVE_LARGE_TILES
#define FOLD3D_WAVE_LARGE_TILES 8192
#endif
constexpr int kLargePlaneTiles = FOLD3D_WAVE_LARGE_TILES;
static_assert(kWaveTV == 1 || kWaveTV == 2 || kWaveTV == 4 || kWaveTV == 8, "tile rows");

// Arguments of one WAVEFRONT pass (fold3d_wavefront.cu).
struct WaveArgs {
    PlaneGeom pg;
    int nrm, ua, va, sg;         // normal axis, in-plane u / v axes, step direction
    int ntu, ntv;                // 32 x kWaveTV tiles per plane (this orientation)
    int steps, first_src;        // plane steps of the pass and the first source plane
    unsigned epoch;              // number of this pass (monotonic per context)
    unsigned skip_from;          // passes numbered below this never skip
    unsigned long long timeout_ns;
    unsigned *flags;             // [steps][tiles]: pass number when the item finished
    unsigned *mod[3];            // per orientation: [plane 0..n+1][tile]: last pass a point changed
    int mod_ntu[3], mod_ntiles[3];
    unsigned *work;              // item counter (zeroed before each pass)
    unsigned *status;            // 0, or 1 after a wait gave up
    unsigned long long *maxd;    // max |dT| (IEEE bits) of the sweep
    unsigned long long *evaluated;  // points evaluated
    unsigned char *winners;      // elliptical medium: winner records, or NULL
    int dir;                     // direction of the pass (for the winner records)
};
// Host sampling of the implicit surface (fold3d_init.cpp).  The tables hold
// the factors of Fold3dPMM.c:29-33 that do not depend on every coordinate:
// sin(x_i), cos(y_j + x_i) and, when the rounded sums x_i + y_j take few
// distinct values (equal or commensurate spacings), those values and each
// (i, j)'s index among them, so that each plane evaluates sin(x + y + z) once
// per distinct sum (the same arguments, so the same bits).
struct SurfaceTables {
    std::vector<double> sin_x;   // nx + 2 values
    std::vector<double> cos_yx;  // (ny + 2) rows of nx + 2
    std::vector<double> sums;    // distinct x_i + y_j, or empty
    std::vector<int> sum_of;     // index into sums of each (i, j), row-major like cos_yx
};
bool surface_tables(const fold3d_grid &g, SurfaceTables &t, int nth);  // false: out of memory
void surface_planes(double *IF, const fold3d_grid &g, int k0, int k1, const SurfaceTables &t, int nth);
int init_threads();
// fn(i) for lo <= i < hi on up to nthreads host threads (contiguous ranges).
void host_parallel_for(int lo, int hi, int nthreads, const std::function<void(int)> &fn);
// ImplicitInitialiser into device field T (fold3d_init_dev.cu): IF_dev a
// device scratch of one field, stage two pinned host buffers of stage_planes
// node planes each.
int init_implicit_device(const fold3d_grid &g, const fold3d_medium &m, double *T, double *IF_dev,
                         double *stage[2], size_t stage_planes, cudaStream_t s);

// Media of the local solver.
enum Medium { kMediumDrift = 0, kMediumEllip = 1 };

// Winner record of a cell (elliptical medium): direction * kEllipCands +
// candidate id (candidate ids 0..32 of the fan solver), kNoWinner if no
// candidate set the cell's time.  One byte per cell.
constexpr unsigned kEllipCands = 33;
constexpr unsigned kNoWinner = 0xffu;

struct EllipDir;     // fold3d_ellip.cuh
struct EllipParam;   // below, once EllipDir is complete

// large: the variant compiled for passes over large planes (kLargePlaneTiles).
cudaError_t launch_wave_pass(double *T, const WaveArgs &a, const DirTable &tab, int grid, cudaStream_t s,
                             bool large = false);
// The elliptical medium's field is double, or float when f32.
cudaError_t launch_wave_pass_ellip(void *T, bool f32, const WaveArgs &a, const EllipParam &p, int grid, cudaStream_t s,
                                   bool large = false);
int wave_blocks_per_sm(int medium, bool f32 = false, bool large = false);

}  // namespace fold3d
#include "fold3d_ellip.cuh"
namespace fold3d {

// One instance of a batched pass (fold3d_wavefront.cu): its pass arguments,
// elliptical-medium constants and field.
struct BatchInst {
    WaveArgs a;
    EllipParam p;
    void *T;  // double, or float in a float32 batch
};
static_assert(sizeof(BatchInst) % 4 == 0, "BatchInst is copied in words");

// One batched pass of direction dir.  inst holds every instance of the batch
// in this direction's order (step count descending); the active ones are
// listed by act (their positions in inst, in that order), so that the
// active instances of a step are a prefix of the list.  step_off: the first
// global item of each step; step_k: the number of active instances with a
// step p; tile_pre: prefix sums of the active instances' tiles per plane.
// Those tables, the pass's item count and the sweep's pass numbers live in
// device memory and are rewritten by the restage kernel after every sweep,
// so a captured graph runs the whole sweep loop.
struct BatchArgs {
    const BatchInst *inst;
    const int *act;               // [active]
    const long long *step_off;    // [max_steps + 1]
    const int *step_k;            // [max_steps]
    const long long *tile_pre;    // [active + 1]
    const unsigned *total;        // items of this pass
    const unsigned *epoch_base;   // this sweep's first pass number minus 1; the pass is epoch_base + dir + 1
    int max_steps, dir;
    unsigned *work, *status;
    unsigned skip_from;           // first pass that may skip
};
// tv: tile height of the batch (2, 4 or 8 rows; 32 * tv threads per CTA).
cudaError_t launch_batch_pass(const BatchArgs &b, bool f32, int tv, int grid, cudaStream_t s);
int batch_blocks_per_sm(bool f32, int tv);

// The sweep loop of a batched solve on the device (fold3d_wavefront.cu).
// After each sweep the restage kernel folds every active instance's largest
// change into its state (sweeps run, last change; converged instances drop
// out), rebuilds each direction's active list and item tables, advances the
// pass numbers, clears the per-sweep maxima, and sets the loop's condition:
// another sweep while some instance is active, the sweep limit is not
// reached and no dependency wait gave up.  With first set it only builds the
// tables (before the first sweep).
struct BatchDirTables {
    const int *order;             // [n] instance at each position of this direction's order
    const int *steps;             // [n] plane steps of the instance at each position
    const long long *tiles;       // [n] tiles per plane of the instance at each position
    int *act;                     // outputs, as in BatchArgs
    long long *step_off;
    int *step_k;
    long long *tile_pre;
};
struct BatchCtl {
    BatchDirTables dir[6];
    int n, max_steps, fixed, max_sweeps;
    double tol;
    unsigned epoch0;              // first pass number minus 1 (first call)
    unsigned *total;              // [6]
    unsigned *epoch_base;
    int *sweep;                   // [0] sweeps run, [1] instances still active
    int *active;                  // [n]
    int *sweeps;                  // [n]
    double *delta;                // [n] largest change of the instance's last sweep
    unsigned long long *maxd;     // [n] this sweep's largest change (IEEE bits), cleared here
    const unsigned *status;
    unsigned long long cond;      // cudaGraphConditionalHandle of the sweep loop
};
cudaError_t launch_batch_restage(const BatchCtl &ctl, bool first, cudaStream_t s);

// One direction's item tables for the active instances (active[i] != 0 for
// instance i): act, tile_pre, step_k and step_off; returns the pass's item
// count.  The active instances with a step p are a prefix of the list (steps
// descending), so step_k[p] shrinks from k as p grows, dropping from the end
// the instances with at most p steps.  Host and device (the restage kernel).
#ifdef __CUDACC__
__host__ __device__
#endif
inline unsigned batch_tables(const BatchDirTables &t, const int *active, int n, int max_steps)
{
    int k = 0;
    t.tile_pre[0] = 0;
    for (int q = 0; q < n; ++q)
        if (active[t.order[q]]) {
            t.act[k] = q;
            t.tile_pre[k + 1] = t.tile_pre[k] + t.tiles[q];
            ++k;
        }
    int kk = k;
    t.step_off[0] = 0;
    for (int p = 0; p < max_steps; ++p) {
        while (kk > 0 && t.steps[t.act[kk - 1]] <= p) --kk;
        t.step_k[p] = kk;
    }
    for (int p = 0; p < max_steps; ++p) t.step_off[p + 1] = t.step_off[p] + t.tile_pre[t.step_k[p]];
    return (unsigned)t.step_off[max_steps];
}

// Adjoint of the elliptical solver (fold3d_adjoint.cu).
struct AdjGeom {
    PlaneGeom pg[6];
    EllipDir d[6];
};
// One backward pass of direction a.dir: a.first_src holds the first target
// plane of the pass (the forward pass's last), a.steps the planes, a.maxd
// receives max |pushed amount|, a.epoch numbers the pass like a forward pass.
struct AdjWaveArgs {
    WaveArgs a;
    const void *T;           // double, or float in a float32 adjoint (as lam and pushed)
    void *lam, *pushed;
    const unsigned char *W;
    const unsigned char *has;  // [plane][tile] of this pass's orientation: 1 if a cell's winner is a.dir
};

// Work map of the adjoint: per direction d, one byte per (plane, tile) of d's
// orientation, 1 when a cell of the tile has its winner in direction d (set
// to 0 before launch_adj_tiles).  Backward items of tiles marked 0 push
// nothing, so they publish at once, without waiting.
struct AdjTiles {
    unsigned char *has[6];
    int nrm[6];              // normal axis of each direction
    int ntu[3], ntiles[3];   // tiles per orientation
};
cudaError_t launch_adj_tiles(const unsigned char *W, const fold3d_grid &g, const AdjTiles &t, cudaStream_t s);

// Batched backward passes: one instance's pass arguments and medium; the
// item tables are laid out as for BatchArgs.
struct BatchAdjInst {
    AdjWaveArgs b;
    EllipParam ep;
};
static_assert(sizeof(BatchAdjInst) % 4 == 0, "BatchAdjInst is copied in words");
struct BatchAdjArgs {
    const BatchAdjInst *inst;
    const unsigned long long *items;  // slot << 40 | item, tiles with work only, step-major
    unsigned total;                   // items in the list
    unsigned *work, *status;
    unsigned epoch;
};
cudaError_t launch_batch_adj_pass(const BatchAdjArgs &b, bool f32, int grid, cudaStream_t s);
// L2 bytes the instances of one launch of a batched x-normal backward pass
// may occupy together (0: one launch over every instance); build option.
#ifndef FOLD3D_ADJ_XGROUP_MB
#define FOLD3D_ADJ_XGROUP_MB 48
#endif
constexpr size_t kAdjXGroupBytes = (size_t)FOLD3D_ADJ_XGROUP_MB << 20;
// Item list of a backward pass over k instance slots: with off == NULL,
// cnt[p * k + q] <- tiles with work at step p of slot q; else items[] <- the
// list, off[p * k + q] being the exclusive prefix of cnt in that order.
cudaError_t launch_adj_list(const BatchAdjInst *inst, int k, int max_steps, int *cnt, const long long *off,
                            unsigned long long *items, cudaStream_t s);
int batch_adj_blocks_per_sm(bool f32);
cudaError_t launch_adj_grad(const void *T, const void *lam, const unsigned char *W, const AdjGeom &geo,
                            const EllipMedium &med, const fold3d_grid &g, void *dLdM, int accumulate, bool f32,
                            cudaStream_t s);

// Kernel launchers (fold3d_kernels.cu).  tab is required for kVariantFast.
cudaError_t launch_plane(double *T, const PlaneGeom &pg, const LocalFrameH &L, const DirTable *tab,
                         int variant, int src, unsigned long long *maxd, cudaStream_t s);

}  // namespace fold3d
