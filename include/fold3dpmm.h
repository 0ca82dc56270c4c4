/*
 * fold3dpmm.h -- C-ABI of the B200 Fold3dPMM library (libfold3dpmm.so).
 *
 * Fold3dPMM is the parallel marching method for the anisotropic ("folding")
 * 3-D eikonal equation of ezhilmathik/FGCS-OpenACC-Advanced: the travel-time
 * field is swept plane by plane in the six axis directions, every point of a
 * plane being updated from the already updated previous plane by a local
 * upwind solver, and the sweeps repeat until the field stops changing.
 *
 * Two layers are declared here.
 *
 * 1. Reference-compatible entry points, with the names, argument lists and
 *    semantics of the reference, so that the reference's C host driver
 *    (Stencil-OpenACC/AN_ISO_1_OpenACC.c:main) runs on this library
 *    unchanged.  They have no error channel (void, as in the reference);
 *    failures are recorded and readable with fold3d_last_error().
 *
 * 2. The native API (fold3d_*): run-time grid sizes (the three axes may
 *    differ), run-time medium, whole solves on the GPU with a convergence
 *    test, status codes, no exits and no traps.
 *
 * Array layout (both layers): a field of (nx+2)*(ny+2)*(nz+2) doubles with one
 * ghost layer per face, element (i,j,k) at T[i + (nx+2)*(j + (ny+2)*k)], interior
 * indices 1..n.  Axis i has spacing dx and drift ax, j: dy/ay, k: dz/az.  The
 * sign of T marks the side of the source surface; |T| is the travel time;
 * FOLD3D_MAXT marks unreached points.  Ghost cells are read, never written.
 */
#ifndef FOLD3DPMM_NATIVE_H
#define FOLD3DPMM_NATIVE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Only the declarations of this header are exported from the shared library
 * (it is built with -fvisibility=hidden). */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
#define FOLD3D_OK 0
#define FOLD3D_ERR_INVALID 1     /* bad argument (null pointer, bad size)  */
#define FOLD3D_ERR_NOMEM 2       /* host or device allocation failed       */
#define FOLD3D_ERR_CUDA 3        /* a CUDA runtime call failed             */
#define FOLD3D_ERR_TIMEOUT 4     /* a bounded device-side wait gave up      */
#define FOLD3D_ERR_UNSUPPORTED 5 /* valid request the library cannot serve */

/* Unreached time, Fold3dPMM.h:6 (MAXT). */
#define FOLD3D_MAXT (10e15 * 1.0)

/* Sweep directions, in the order the reference driver runs them each sweep
 * (AN_ISO_1_OpenACC.c:1195-1236). */
enum fold3d_dir {
    FOLD3D_X_DOWN = 0, /* target plane i+1 from i, i = 1..nx-1  (function_x_down) */
    FOLD3D_X_UP = 1,   /* target plane i-1 from i, i = nx..2    (function_x_up)   */
    FOLD3D_K_UP = 2,   /* target plane k+1 from k, k = 1..nz-1  (function_k_up)   */
    FOLD3D_K_DOWN = 3, /* target plane k-1 from k, k = nz..2    (function_k_down) */
    FOLD3D_Y_UP = 4,   /* target plane j-1 from j, j = ny..2    (function_y_up)   */
    FOLD3D_Y_DOWN = 5  /* target plane j+1 from j, j = 1..ny-1  (function_y_down) */
};

/* Execution engines for a whole solve. */
enum fold3d_engine {
    FOLD3D_ENGINE_AUTO = 0,      /* WAVEFRONT for variant 0, PLANES otherwise          */
    FOLD3D_ENGINE_PLANES = 1,    /* one kernel per plane, each sweep a CUDA graph    */
    FOLD3D_ENGINE_WAVEFRONT = 2  /* one persistent kernel per pass, tile dataflow     */
};

typedef struct {
    int nx, ny, nz;       /* interior points per axis (>= 2)          */
    double dx, dy, dz;    /* grid spacing per axis (> 0)              */
} fold3d_grid;

/* The reference's medium: isotropic speed F plus a constant drift
 * a = (ax, ay, az); the unit-time wavefront from a point is the sphere
 * |x - a| = F (Fold3dPMM.c:9-26).  Requires F*F > |a|^2. */
typedef struct {
    double F;
    double ax, ay, az;
} fold3d_medium;

typedef struct {
    int max_sweeps;   /* sweeps to run at most (>= 1)                          */
    int fixed;        /* non-zero: run exactly max_sweeps, no convergence test   */
                      /* (the reference driver runs a fixed 8, :1187)            */
    double tol;       /* else stop after the first sweep with max|dT| <= tol     */
    int engine;       /* enum fold3d_engine                                      */
    int skip;         /* non-zero: skip tiles whose inputs did not change since   */
                      /* their last update in that direction (result unchanged, */
                      /* bit for bit); wavefront engine only                     */
    int variant;      /* local-solver form, same results bit for bit:            */
                      /* 0 = per-direction constants folded on the host (fast),  */
                      /* 1 = the reference's expressions point by point (check), */
                      /* 2 = folded constants, calls compacted across the block  */
} fold3d_opts;

typedef struct {
    int sweeps;                  /* sweeps run                                 */
    double max_delta;            /* max |T_after - T_before| of the last sweep */
    double elapsed_ms;           /* device time of the sweeps (CUDA events)    */
    uint64_t nominal_updates;    /* point updates the reference would do       */
    uint64_t evaluated_updates;  /* point updates actually evaluated           */
    int engine;                  /* engine that ran                            */
} fold3d_report;

typedef struct fold3d_ctx fold3d_ctx;

/* ------------------------------------------------------------------------ */
/* Native API                                                                */
/* ------------------------------------------------------------------------ */

/* Message of the last failure on the calling host thread ("" if none). */
const char *fold3d_last_error(void);

/* Library version string. */
const char *fold3d_version(void);

/* Default options: fixed = 0, max_sweeps = 1000, tol = 0.0 (run until the
 * field stops changing), engine = AUTO, skip = 1, variant = 0. */
void fold3d_default_opts(fold3d_opts *o);

/* Context: owns device scratch, graphs and events for one device.  One
 * context per host thread, or externally synchronised. */
int fold3d_create(fold3d_ctx **ctx, int device);
void fold3d_destroy(fold3d_ctx *ctx);

/* Solve in place on a device field.  T_dev: device pointer to the
 * (nx+2)(ny+2)(nz+2) field.  stream: a cudaStream_t (NULL = legacy default
 * stream).  Returns when the solve has finished on the device.  rep may be
 * NULL. */
int fold3d_solve(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_medium *m,
                 double *T_dev, const fold3d_opts *o, void *stream, fold3d_report *rep);

/* Same, for fields in host memory: copies T_in to the device, solves, copies
 * the result to T_out (T_out may equal T_in).  Pinned host buffers make the
 * copies faster.  Device memory is allocated by the context and kept for
 * reuse. */
int fold3d_solve_host(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_medium *m,
                      const double *T_in, double *T_out, const fold3d_opts *o, void *stream,
                      fold3d_report *rep);

/* One plane step on a device field: update plane src+1 (down) or src-1 (up)
 * of direction dir from plane src.  Asynchronous on stream. */
int fold3d_plane(const fold3d_grid *g, const fold3d_medium *m, double *T_dev, int dir,
                 int src, void *stream);

/* A per-cell elliptical (tilted transversely isotropic) medium.  No
 * counterpart in the reference, whose solver only knows the drift medium.
 * The travel time along a short straight segment d is sqrt(d^T M d), M the
 * cell's symmetric positive definite metric (slowness squared); the six
 * arrays hold M's entries in the i, j, k axes, as float, in the field layout
 * ((nx+2)(ny+2)(nz+2), only interior cells are read), on the device. */
typedef struct {
    const float *mxx, *mxy, *mxz, *myy, *myz, *mzz;
} fold3d_ellip;

/* Metric of a tilted elliptical cell: vertical speed vz, Thomsen epsilon eps
 * (horizontal speed vz*sqrt(1+2*eps)) and symmetry axis (ax, ay, az) (need
 * not be normalised): M = a I + b n n^T with a = 1/(vz^2 (1+2 eps)),
 * b = 1/vz^2 - a.  out = {xx, xy, xz, yy, yz, zz}. */
void fold3d_ellip_metric(double vz, double eps, double ax, double ay, double az, float out[6]);

/* Solve in place on a device field with an elliptical medium (engine
 * WAVEFRONT; opts.variant must be 0).  Same sweep order, stopping rules and
 * report as fold3d_solve. */
int fold3d_solve_ellip(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_ellip *m, double *T_dev,
                       const fold3d_opts *o, void *stream, fold3d_report *rep);

/* fold3d_solve_ellip that also records, per cell, the candidate that last
 * set its time -- direction * 33 + candidate id (directions 0..5 as in
 * fold3d_dir, candidate ids 0..32 of the fan solver), or 0xff if none did --
 * into winners_dev (one byte per field cell, device memory; the call first
 * sets it to 0xff).  This record is the checkpoint of the
 * adjoint; it replaces the history of the field. */
int fold3d_solve_ellip_record(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_ellip *m, double *T_dev,
                              unsigned char *winners_dev, const fold3d_opts *o, void *stream,
                              fold3d_report *rep);

/* Adjoint of a converged elliptical solve.  No counterpart in the reference.
 * Given the converged field T_dev, its winner record and dLdT_dev = dL/dT
 * (device, field layout), writes lambda_dev = the total derivative dL/dT
 * (device, field layout) and dLdM_dev = dL/dM, six arrays of doubles in the
 * field layout, component-major (xx xy xz yy yz zz), every cell written (0 on
 * ghosts and on cells without a winner).  Backward sweeps repeat until one
 * pushes at most tol times the largest amount the first sweep pushed (tol 0:
 * until one pushes nothing), at most max_sweeps; rep->sweeps counts them and
 * rep->max_delta is the largest pushed amount of the last one.  The gradient
 * converges geometrically over the sweeps; tol 1e-12 typically leaves a
 * relative error of that order.
 * lambda is accumulated with floating-point atomics: results agree with the
 * FP64 CPU statement to rounding, not bit for bit. */
int fold3d_adjoint_ellip(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_ellip *m, const double *T_dev,
                         const unsigned char *winners_dev, const double *dLdT_dev, double *lambda_dev,
                         double *dLdM_dev, int max_sweeps, double tol, void *stream, fold3d_report *rep);

/* One instance of a batched solve: its grid, elliptical medium and device
 * field (in/out).  winners: NULL, or a device winner record of one byte per
 * field cell, filled as by fold3d_solve_ellip_record. */
typedef struct {
    fold3d_grid grid;
    fold3d_ellip medium;
    double *T;
    unsigned char *winners;
} fold3d_instance;

/* Solves n independent instances (grids of any sizes, elliptical media) at
 * once: every directional pass of all instances that are still running is
 * one launch, whose CTAs take tiles of all instances from one queue.  No
 * counterpart in the reference.  Unless opts.fixed, each instance stops
 * after its first sweep with max|dT| <= opts.tol, the others go on.  Results
 * are bit-identical to solving the instances one by one with
 * fold3d_solve_ellip.  reps: n reports, or NULL. */
int fold3d_solve_batch(fold3d_ctx *ctx, int n, const fold3d_instance *inst, const fold3d_opts *o,
                       void *stream, fold3d_report *reps);

/* One instance of a batched adjoint: the arguments of fold3d_adjoint_ellip
 * (device pointers, field layout; dLdM: six arrays, component-major). */
typedef struct {
    fold3d_grid grid;
    fold3d_ellip medium;
    const double *T;
    const unsigned char *winners;
    const double *dLdT;
    double *lambda;
    double *dLdM;
} fold3d_adjoint_instance;

/* The adjoints of n converged elliptical solves at once (no counterpart in
 * the reference): every backward pass of all instances still running is one
 * launch.  Each instance stops as fold3d_adjoint_ellip would with the same
 * max_sweeps and tol.  accumulate = 0: dLdM is written as by
 * fold3d_adjoint_ellip; accumulate != 0: dLdM += the instance's gradient, so
 * instances of one grid may share one dLdM (the sum over sources of a
 * tomography loss).  reps: n reports, or NULL. */
int fold3d_adjoint_batch(fold3d_ctx *ctx, int n, const fold3d_adjoint_instance *inst, int max_sweeps, double tol,
                         int accumulate, void *stream, fold3d_report *reps);

/* Float32 build of the elliptical medium (no counterpart in the reference):
 * the entry points above with float fields.  The local solver, the winner
 * records and the adjoint compute in float arithmetic throughout (the metric
 * arrays are float in both builds); dLdM is float too. */
typedef struct {
    fold3d_grid grid;
    fold3d_ellip medium;
    float *T;
    unsigned char *winners;
} fold3d_instance_f32;

typedef struct {
    fold3d_grid grid;
    fold3d_ellip medium;
    const float *T;
    const unsigned char *winners;
    const float *dLdT;
    float *lambda;
    float *dLdM;
} fold3d_adjoint_instance_f32;

int fold3d_solve_ellip_f32(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_ellip *m, float *T_dev,
                           const fold3d_opts *o, void *stream, fold3d_report *rep);
int fold3d_solve_ellip_record_f32(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_ellip *m, float *T_dev,
                                  unsigned char *winners_dev, const fold3d_opts *o, void *stream,
                                  fold3d_report *rep);
int fold3d_adjoint_ellip_f32(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_ellip *m, const float *T_dev,
                             const unsigned char *winners_dev, const float *dLdT_dev, float *lambda_dev,
                             float *dLdM_dev, int max_sweeps, double tol, void *stream, fold3d_report *rep);
int fold3d_solve_batch_f32(fold3d_ctx *ctx, int n, const fold3d_instance_f32 *inst, const fold3d_opts *o,
                           void *stream, fold3d_report *reps);
int fold3d_adjoint_batch_f32(fold3d_ctx *ctx, int n, const fold3d_adjoint_instance_f32 *inst, int max_sweeps,
                             double tol, int accumulate, void *stream, fold3d_report *reps);

/* Configuration of the batched solves (no counterpart in the reference):
 * tile height in rows of 32 points (2, 4 or 8; a CTA has 32 * rows threads)
 * and resident CTAs per SM (0 or above the occupancy limit: the limit).
 * tile_rows = 0 (the default) lets the context's autotuner choose: for each
 * size mix it has not seen (8 or more instances), it times one sweep of each
 * candidate on copies of a few median-size instances and keeps the fastest.
 * Every configuration gives the same results bit for bit. */
int fold3d_batch_set_config(fold3d_ctx *ctx, int tile_rows, int ctas_per_sm);
/* The configuration the last batched solve on ctx ran with. */
int fold3d_batch_get_config(fold3d_ctx *ctx, int *tile_rows, int *ctas_per_sm);

/* The tilted elliptical medium given by its FP64 parameters (no counterpart
 * in the reference).  Four double arrays in the field layout: slowness
 * s = 1/Vz, Thomsen epsilon, and the x and y components of the unit symmetry
 * axis n (its z component is sqrt(1 - nx^2 - ny^2) >= 0; n and -n are the
 * same axis).  The kernels form M = a I + b n n^T with a = s^2/(1 + 2 eps),
 * b = s^2 - a per cell in FP64, so nothing is rounded to float.  Fields are
 * float64; the solver, winner records, batches and the adjoint are those of
 * the six-array medium above.  32 bytes of medium per cell (1280^3: 67 GB). */
typedef struct {
    const double *s, *eps, *nx, *ny;
} fold3d_tti;

typedef struct {
    fold3d_grid grid;
    fold3d_tti medium;
    double *T;
    unsigned char *winners;  /* or NULL */
} fold3d_tti_instance;

typedef struct {
    fold3d_grid grid;
    fold3d_tti medium;
    const double *T;
    const unsigned char *winners;
    const double *dLdT;
    double *lambda;
    double *dLdP;  /* 4 x cells: dL/ds, dL/deps, dL/dnx, dL/dny */
} fold3d_tti_adjoint_instance;

int fold3d_solve_tti(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_tti *m, double *T_dev,
                     const fold3d_opts *o, void *stream, fold3d_report *rep);
int fold3d_solve_tti_record(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_tti *m, double *T_dev,
                            unsigned char *winners_dev, const fold3d_opts *o, void *stream,
                            fold3d_report *rep);
/* As fold3d_adjoint_ellip, but the gradient is with respect to the medium's
 * parameters: dLdP holds four arrays (dL/ds, dL/deps, dL/dnx, dL/dny; the
 * axis components at fixed unit length, nz following them; where nz = 0 only
 * the direct terms). */
int fold3d_adjoint_tti(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_tti *m, const double *T_dev,
                       const unsigned char *winners_dev, const double *dLdT_dev, double *lambda_dev,
                       double *dLdP_dev, int max_sweeps, double tol, void *stream, fold3d_report *rep);
int fold3d_solve_batch_tti(fold3d_ctx *ctx, int n, const fold3d_tti_instance *inst, const fold3d_opts *o,
                           void *stream, fold3d_report *reps);
int fold3d_adjoint_batch_tti(fold3d_ctx *ctx, int n, const fold3d_tti_adjoint_instance *inst, int max_sweeps,
                             double tol, int accumulate, void *stream, fold3d_report *reps);

/* Implicit-surface source initialisation of a host field (the reference's
 * ImplicitInitialiser, Fold3dPMM.c:129-389, with run-time sizes and medium).
 * Uses all host cores. */
int fold3d_init_implicit(double *T_host, const fold3d_grid *g, const fold3d_medium *m);

/* ImplicitInitialiser into a device field T_dev (no counterpart in the
 * reference, whose initialiser is host-only): the implicit surface is
 * sampled on the host (the reference's libm, for the same bits) and streamed
 * to the device in slabs; the crossings and node updates run on the GPU.
 * The result equals fold3d_init_implicit's bit for bit.  Keeps one field of
 * device scratch and two ~256 MB pinned host buffers in the context. */
int fold3d_init_implicit_device(fold3d_ctx *ctx, const fold3d_grid *g, const fold3d_medium *m, double *T_dev,
                                void *stream);

/* Output of a host field.
 * fold3d_write_text: the reference's error-checking dump
 * (AN_ISO_1_OpenACC.c:1244-1260): "%f\n" per value, i outermost, k innermost,
 * ghosts included -- the same bytes as the reference's file.
 * fold3d_write_vtk: a legacy VTK STRUCTURED_POINTS file of the travel times
 * (binary big-endian doubles, x fastest; ghosts = 0: the interior only), the
 * file the reference's Write_VTK_Structured_Grid (:1098-1135) leaves empty.
 * fold3d_write_raw: a 64-byte header ("FOLD3DRW", int32 version 1, nx, ny,
 * nz, double dx, dy, dz) and the whole field, little-endian doubles. */
int fold3d_write_text(const char *path, const double *T_host, const fold3d_grid *g);
int fold3d_write_vtk(const char *path, const double *T_host, const fold3d_grid *g, int ghosts);
int fold3d_write_raw(const char *path, const double *T_host, const fold3d_grid *g);

/* Point source: T = +MAXT everywhere, T[si,sj,sk] = 0 (host field). */
int fold3d_init_point(double *T_host, const fold3d_grid *g, int si, int sj, int sk);

/* Exact travel time of the homogeneous medium from the origin to (x,y,z),
 * FOLD3D_MAXT where undefined (InitFoldFromPoint, Fold3dPMM.c:9-26). */
double fold3d_exact_time(const fold3d_medium *m, double x, double y, double z);

/* Whole solve that allocates nothing.  No counterpart in the reference.
 *
 * For callers that must not have device memory allocated for them: host
 * programs whose device buffers all come from another runtime (an OpenACC
 * driver using acc_malloc, a framework whose caching allocator already holds
 * the GPU's memory) or plugin hosts that lend buffers and budget every byte.
 * It runs the same per-plane kernels as fold3d_solve (engine and skip are
 * ignored), needs no context, and calls no cudaMalloc, cudaFree or other
 * allocating routine.  The caller passes the device field T_dev (in/out).
 *
 * Scratch: a static device array of FOLD3D_NOALLOC_MAX_SWEEPS 8-byte slots
 * (32 KiB), one per sweep, that every GPU which loads the library holds until
 * the process exits; calls with max_sweeps above that limit are rejected with
 * FOLD3D_ERR_INVALID.  All calls share the array and it keeps the previous
 * call's values: each sweep clears its own slot first, and calls whose work
 * overlaps on the GPU race on it.  The first call in each CUDA context looks
 * up the array's device address (cudaGetSymbolAddress) with the caller's
 * device and context current, and later calls in that context reuse it; a
 * new context on the same device (after cudaDeviceReset, or another
 * runtime's context made current) gets its own lookup.  Make the first call
 * in a context before any stream capture.  Arguments are checked as by
 * fold3d_solve.  Synchronous like fold3d_solve; rep->elapsed_ms is the
 * call's host wall time. */
#define FOLD3D_NOALLOC_MAX_SWEEPS 4096
int fold3d_solve_noalloc(const fold3d_grid *g, const fold3d_medium *m, double *T_dev,
                         const fold3d_opts *o, void *stream, fold3d_report *rep);

/* The body of the six reference-compatible sweep functions below: one plane
 * step of direction dir with the reference's argument conventions.  Programs
 * that compile the reference's own sweep definitions (AN_ISO_1_OpenACC.c)
 * and want this library's instead link the forwarders in
 * fgcs-openacc-advanced_b200/dropin/fold3d_dropin.c, which call this. */
void fold3d_compat_plane(int dir, double *T, int plane, double dzz, double dxx, double dyy,
                         double dxy, double dxz, double dyz, double F, double ay, double ax,
                         double az);

/* Diagnostic: runs one WAVEFRONT pass on a small internal field whose first
 * plane step is never published, with the dependency-wait limit set to
 * timeout_ms, so every wait gives up.  Returns FOLD3D_ERR_TIMEOUT when the
 * bounded waits and the status word work (the context stays usable), any
 * other code otherwise.  Faults nothing and hangs nothing. */
int fold3d_selftest_wait_timeout(fold3d_ctx *ctx, double timeout_ms);

/* Grid size the reference-compatible sweep functions assume for a device
 * field (they have no size argument, AN_ISO_1_OpenACC.c:180).  If never set,
 * the size is taken from the allocation made by this library's acc_malloc. */
int fold3d_compat_set_grid(int nx, int ny, int nz);

/* ------------------------------------------------------------------------ */
/* Reference-compatible entry points                                         */
/* ------------------------------------------------------------------------ */

/* Fold3dPMM.h:58-75 / Fold3dPMM.c:9-126.  Host functions; T is a host field
 * of a cubic grid whose pitch is nx+2 (the reference's HEIGHT). */
double InitFoldFromPoint(double F, double ax, double ay, double az, double x, double y,
                         double z);
double ImpSurfF(double x, double y, double z);
/* Fold3dPMM.h:81-85 / Fold3dPMM.c:129-389: medium = the reference constants
 * F = 1.1, a = (-0.35, 0.4, 0.7).  Also remembers (nx, ny, nz) as the grid of
 * InitNode and updateVoxel. */
void ImplicitInitialiser(double *T, int nx, int ny, int nz, double dxx, double dyy,
                         double dzz);
/* Fold3dPMM.h:64 / Fold3dPMM.c:35-54: min-update of host node (i, j, k) with
 * the reference medium's exact time from the point (x, y, z) relative to it,
 * keeping the node's sign.  The reference indexes T with its compile-time
 * HEIGHT; here the pitch is nx+2 (and ny+2) of the grid set by
 * fold3d_compat_set_grid, else of the last ImplicitInitialiser call.  With
 * neither, nothing is written and fold3d_last_error says why. */
void InitNode(double x, double y, double z, int i, int j, int k, double *T);
/* Fold3dPMM.h:67-70 / Fold3dPMM.c:56-112: the 44 InitNode calls of one
 * seeding point at (xp, yp, zp) in voxel (i, j, k), in the reference's order
 * (same pitch rule as InitNode). */
void updateVoxel(double *T, int i, int j, int k, double xp, double yp, double zp, double dxx,
                 double dyy, double dzz);
/* Fold3dPMM.h:72-76 / Fold3dPMM.c:115-126: coordinate of node i, j or k
 * ((i - 1) * spacing + 0, the reference's domain starting at 0). */
double x(int i, double DX);
double y(int j, double dy);
double z(int k, double dz);

/* AN_ISO_1_OpenACC.c:180, 334, 485, 636, 790, 944.  T is a DEVICE pointer
 * (the reference's deviceptr(T), :189).  The plane index and the permuted
 * spacings and drift are those the reference driver passes (:1195-1236):
 * (dzz, dxx, dyy) = spacing normal to the plane, along the local x and y
 * neighbours; dxy, dxz, dyz the diagonals; (ax, ay, az) the drift in that
 * local frame.  Synchronous, like the reference's OpenACC regions. */
void function_x_down(double *T, int i, double dzz, double dxx, double dyy, double dxy,
                     double dxz, double dyz, double F, double ay, double ax, double az);
void function_x_up(double *T, int i, double dzz, double dxx, double dyy, double dxy,
                   double dxz, double dyz, double F, double ay, double ax, double az);
void function_y_up(double *T, int j, double dzz, double dxx, double dyy, double dxy,
                   double dxz, double dyz, double F, double ay, double ax, double az);
void function_y_down(double *T, int j, double dzz, double dxx, double dyy, double dxy,
                     double dxz, double dyz, double F, double ay, double ax, double az);
void function_k_up(double *T, int k, double dzz, double dxx, double dyy, double dxy,
                   double dxz, double dyz, double F, double ay, double ax, double az);
void function_k_down(double *T, int k, double dzz, double dxx, double dyy, double dxy,
                     double dxz, double dyz, double F, double ay, double ax, double az);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* FOLD3DPMM_NATIVE_H */
