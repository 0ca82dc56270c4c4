// fold3d_api.cu -- the C-ABI: contexts, whole solves, per-plane steps, the
// reference-compatible sweep entry points and the OpenACC runtime subset the
// reference driver calls.
#include <cmath>
#include <cstdio>
#include <cstdarg>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <vector>
#include <mutex>
#include <new>
#include <string>

#include "fold3d_acc.h"
#include "fold3d_ellip.cuh"
#include "fold3d_fast.cuh"
#include "fold3d_internal.h"

namespace fold3d {

const DirSpec kDirs[6] = {
    {0, +1, 2, +1, 1, +1},  // x_down  AN_ISO_1_OpenACC.c:180
    {0, -1, 2, -1, 1, -1},  // x_up    :334
    {2, +1, 1, +1, 0, +1},  // k_up    :790
    {2, -1, 1, -1, 0, -1},  // k_down  :944
    {1, -1, 0, -1, 2, -1},  // y_up    :485
    {1, +1, 0, +1, 2, +1},  // y_down  :636
};

// The last error message of this host thread.  A fixed buffer: recording an
// error allocates nothing, so no error path can throw.
static thread_local char t_err[512];

int set_error(int code, const char *msg)
{
    snprintf(t_err, sizeof t_err, "%s", msg ? msg : "");
    return code;
}
int set_errorf(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_err, sizeof t_err, fmt, ap);
    va_end(ap);
    return code;
}
int cuda_error(cudaError_t e, const char *what)
{
    return set_errorf(FOLD3D_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void clear_error() { t_err[0] = 0; }

static void strides(const fold3d_grid &g, long long st[3])
{
    st[0] = 1;
    st[1] = (long long)g.nx + 2;
    st[2] = ((long long)g.nx + 2) * ((long long)g.ny + 2);
}

PlaneGeom make_geom(const fold3d_grid &g, int dir)
{
    const DirSpec &d = kDirs[dir];
    const int n[3] = {g.nx, g.ny, g.nz};
    long long st[3];
    strides(g, st);
    const int u = (d.nrm == 0) ? 1 : 0;
    const int v = (d.nrm == 2) ? 1 : 2;
    PlaneGeom p;
    p.s_nrm = st[d.nrm];
    p.sn = d.sg * st[d.nrm];
    p.sx = d.xs * st[d.xa];
    p.sy = d.ys * st[d.ya];
    p.su = st[u];
    p.sv = st[v];
    p.nu = n[u];
    p.nv = n[v];
    p.nplanes = n[d.nrm];
    return p;
}

LocalFrameH make_frame(const fold3d_grid &g, const fold3d_medium &m, int dir)
{
    const DirSpec &d = kDirs[dir];
    const double h[3] = {g.dx, g.dy, g.dz};
    const double a[3] = {m.ax, m.ay, m.az};
    LocalFrameH L;
    L.F = m.F;
    L.ax = d.xs * a[d.xa];
    L.ay = d.ys * a[d.ya];
    L.az = d.sg * a[d.nrm];
    L.hz = h[d.nrm];
    L.hx = h[d.xa];
    L.hy = h[d.ya];
    // The reference driver's diagonals, e.g. DXYP = sqrt(DX*DX + dy*dy)
    // (AN_ISO_1_OpenACC.c:1158-1160); the sum is commutative in IEEE.
    L.hxy = std::sqrt(L.hx * L.hx + L.hy * L.hy);
    L.hxz = std::sqrt(L.hx * L.hx + L.hz * L.hz);
    L.hyz = std::sqrt(L.hy * L.hy + L.hz * L.hz);
    return L;
}

int check_grid(const fold3d_grid *g)
{
    if (!g) return set_error(FOLD3D_ERR_INVALID, "grid is NULL");
    if (g->nx < 2 || g->ny < 2 || g->nz < 2)
        return set_error(FOLD3D_ERR_INVALID, "grid sizes must be >= 2");
    if (!(g->dx > 0 && g->dy > 0 && g->dz > 0) || !std::isfinite(g->dx) ||
        !std::isfinite(g->dy) || !std::isfinite(g->dz))
        return set_error(FOLD3D_ERR_INVALID, "grid spacings must be finite and > 0");
    const double n3[3] = {(double)g->nx, (double)g->ny, (double)g->nz};
    const double cells = (n3[0] + 2) * (n3[1] + 2) * (n3[2] + 2);
    if (cells > 4.0e18 / 8) return set_error(FOLD3D_ERR_INVALID, "grid too large");
    // The (plane, tile) items of one pass are counted in int.  Tiles hold at
    // least 4 x 4 points in either orientation, so this bound is safe; it only
    // rejects grids whose FP64 field alone exceeds 270 GB.
    for (int a = 0; a < 3; ++a)
        if (n3[a] * std::ceil(n3[(a + 1) % 3] / 4) * std::ceil(n3[(a + 2) % 3] / 4) > 2147483647.0)
            return set_error(FOLD3D_ERR_INVALID, "grid too large");
    return FOLD3D_OK;
}

int check_medium(const fold3d_medium *m)
{
    if (!m) return set_error(FOLD3D_ERR_INVALID, "medium is NULL");
    if (!(m->F > 0) || !std::isfinite(m->F) || !std::isfinite(m->ax) || !std::isfinite(m->ay) ||
        !std::isfinite(m->az))
        return set_error(FOLD3D_ERR_INVALID, "medium must be finite with F > 0");
    return FOLD3D_OK;
}

static size_t field_cells(const fold3d_grid &g)
{
    return (size_t)(g.nx + 2) * (size_t)(g.ny + 2) * (size_t)(g.nz + 2);
}

static uint64_t nominal_per_sweep(const fold3d_grid &g)
{
    const uint64_t nx = g.nx, ny = g.ny, nz = g.nz;
    return 2 * ((nx - 1) * ny * nz + (ny - 1) * nx * nz + (nz - 1) * nx * ny);
}

}  // namespace fold3d

using namespace fold3d;

// ------------------------------------------------------------------------
// Context
// ------------------------------------------------------------------------
struct fold3d_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;  // blocking w.r.t. the legacy stream
    unsigned long long *d_maxd = nullptr;
    unsigned long long *h_maxd = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // PLANES engine: one sweep captured as a graph, cached per (T, grid, medium)
    cudaGraphExec_t sweep_exec = nullptr;
    double *key_T = nullptr;
    fold3d_grid key_g{};
    fold3d_medium key_m{};
    int key_variant = -1;
    // buffer for fold3d_solve_host
    double *d_field = nullptr;
    size_t d_field_cells = 0;
    // WAVEFRONT engine scratch, sized for the grid of key_wg
    fold3d_grid key_wg{};
    unsigned *w_flags = nullptr;
    unsigned *w_mod[3] = {nullptr, nullptr, nullptr};
    unsigned *w_counters = nullptr;          // [0] work, [1] status
    unsigned long long *w_evaluated = nullptr;
    unsigned epoch = 0;                      // passes run so far on this context (never decreases)
    int sms = 0, batch_adj_bps = 0;
    int batch_bps[2][9] = {};                // resident batched-pass CTAs per SM, [f32][tile height]
    int btv = kWaveTV;                       // tile height the batch scratch is laid out for
    int tune_tv = 0, tune_bps = 0;           // fold3d_batch_set_config (0: autotune)
    int last_tv = 0, last_bps = 0;           // configuration of the last batched solve
    std::map<std::vector<long long>, std::pair<int, int>> tuned;  // size mix -> (tile height, CTAs per SM)
    double *tune_T = nullptr;                // autotuner: copies of a few instances' fields
    size_t tune_cells = 0;
    int wave_bps[2][2][2] = {};              // [ellip][f32][large plane] resident CTAs per SM
    // batched solves: per-instance scratch and per-direction staging
    std::vector<int> bkey;                   // dims of the instances the scratch is sized for
    unsigned *b_scratch = nullptr;           // flags and change maps of all instances
    std::vector<size_t> b_flag_off, b_mod_off[3];
    unsigned long long *b_slots = nullptr;   // [2n]: max|dT| and evaluated points per instance
    unsigned *b_counters = nullptr;          // work, status
    double *adj_pushed = nullptr;            // adjoint: lambda already pushed, per cell
    size_t adj_cells = 0;
    unsigned char *adj_has = nullptr;        // adjoint work maps (AdjTiles)
    size_t adj_has_bytes = 0;
    unsigned long long *adj_items = nullptr; // adjoint item lists, six directions
    size_t adj_items_cap = 0;
    double *i_if = nullptr;                  // device initialiser: the surface on the device
    size_t i_if_cells = 0;
    double *i_stage[2] = {nullptr, nullptr}; // ... and two pinned slabs of it on the host
    size_t i_stage_bytes = 0;
    int *adj_cnt = nullptr;                  // per (step, slot) counts, then offsets
    long long *adj_off = nullptr;
    size_t adj_cnt_cap = 0;
    char *b_stage_d = nullptr, *b_stage_h = nullptr;
    size_t b_stage_bytes = 0;
    char *b_ctl = nullptr;                   // device state of the batched sweep loop (BatchCtl)
};

namespace {
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};
}  // namespace

extern "C" {

const char *fold3d_last_error(void) { return t_err; }

const char *fold3d_version(void) { return "fold3dpmm-b200 0.1 (sm_100a)"; }

void fold3d_default_opts(fold3d_opts *o)
{
    if (!o) return;
    o->max_sweeps = 1000;
    o->fixed = 0;
    o->tol = 0.0;
    o->engine = FOLD3D_ENGINE_AUTO;
    o->skip = 1;
    o->variant = 0;
}

int fold3d_create(fold3d_ctx **out, int device)
{
    clear_error();
    if (!out) return set_error(FOLD3D_ERR_INVALID, "ctx out-pointer is NULL");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) return set_error(FOLD3D_ERR_INVALID, "no such device");
    DeviceGuard dg(device);
    fold3d_ctx *c = new (std::nothrow) fold3d_ctx();
    if (!c) return set_error(FOLD3D_ERR_NOMEM, "host allocation failed");
    c->device = device;
    if ((e = cudaStreamCreate(&c->stream)) != cudaSuccess ||
        (e = cudaMalloc(&c->d_maxd, sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMallocHost(&c->h_maxd, sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaEventCreate(&c->ev0)) != cudaSuccess || (e = cudaEventCreate(&c->ev1)) != cudaSuccess) {
        fold3d_destroy(c);
        return cuda_error(e, "context setup");
    }
    *out = c;
    return FOLD3D_OK;
}

void fold3d_destroy(fold3d_ctx *c)
{
    if (!c) return;
    DeviceGuard dg(c->device);
    if (c->sweep_exec) cudaGraphExecDestroy(c->sweep_exec);
    if (c->d_field) cudaFree(c->d_field);
    if (c->w_flags) cudaFree(c->w_flags);
    for (int b = 0; b < 3; ++b)
        if (c->w_mod[b]) cudaFree(c->w_mod[b]);
    if (c->w_counters) cudaFree(c->w_counters);
    if (c->w_evaluated) cudaFree(c->w_evaluated);
    if (c->b_scratch) cudaFree(c->b_scratch);
    if (c->b_slots) cudaFree(c->b_slots);
    if (c->b_counters) cudaFree(c->b_counters);
    if (c->adj_pushed) cudaFree(c->adj_pushed);
    if (c->adj_has) cudaFree(c->adj_has);
    if (c->adj_items) cudaFree(c->adj_items);
    if (c->adj_cnt) cudaFree(c->adj_cnt);
    if (c->i_if) cudaFree(c->i_if);
    for (int b = 0; b < 2; ++b)
        if (c->i_stage[b]) cudaFreeHost(c->i_stage[b]);
    if (c->adj_off) cudaFree(c->adj_off);
    if (c->b_stage_d) cudaFree(c->b_stage_d);
    if (c->b_stage_h) cudaFreeHost(c->b_stage_h);
    if (c->b_ctl) cudaFree(c->b_ctl);
    if (c->tune_T) cudaFree(c->tune_T);
    if (c->d_maxd) cudaFree(c->d_maxd);
    if (c->h_maxd) cudaFreeHost(c->h_maxd);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // extern "C"

// One sweep (max-delta reset + the 6 passes) captured into a graph.
static int build_sweep_graph(fold3d_ctx *c, const fold3d_grid &g, const fold3d_medium &m, double *T,
                             int variant)
{
    if (c->sweep_exec && c->key_T == T && !memcmp(&c->key_g, &g, sizeof g) &&
        !memcmp(&c->key_m, &m, sizeof m) && c->key_variant == variant)
        return FOLD3D_OK;
    if (c->sweep_exec) {
        cudaGraphExecDestroy(c->sweep_exec);
        c->sweep_exec = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_error(e, "cudaStreamBeginCapture");
    cudaError_t le = cudaMemsetAsync(c->d_maxd, 0, sizeof(unsigned long long), c->stream);
    for (int dir = 0; dir < 6 && le == cudaSuccess; ++dir) {
        const PlaneGeom pg = make_geom(g, dir);
        const LocalFrameH L = make_frame(g, m, dir);
        DirTable tab;
        build_dir_table(L, tab);
        int src = pass_first(pg, dir);
        for (int p = 0; p < pass_count(pg) && le == cudaSuccess; ++p, src += kDirs[dir].sg)
            le = launch_plane(T, pg, L, &tab, variant, src, c->d_maxd, c->stream);
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(c->stream, &graph);
    if (le != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_error(le, "capturing the sweep");
    }
    if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&c->sweep_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        c->sweep_exec = nullptr;
        return cuda_error(e, "cudaGraphInstantiate");
    }
    c->key_T = T;
    c->key_g = g;
    c->key_m = m;
    c->key_variant = variant;
    return FOLD3D_OK;
}

static int solve_planes(fold3d_ctx *c, const fold3d_grid &g, const fold3d_medium &m, double *T,
                        const fold3d_opts &o, cudaStream_t s, fold3d_report *rep)
{
    int rc = build_sweep_graph(c, g, m, T, o.variant);
    if (rc) return rc;
    cudaError_t e;
    if ((e = cudaEventRecord(c->ev0, s)) != cudaSuccess) return cuda_error(e, "cudaEventRecord");
    int sweeps = 0;
    double delta = 0.0;
    while (sweeps < o.max_sweeps) {
        if ((e = cudaGraphLaunch(c->sweep_exec, s)) != cudaSuccess) return cuda_error(e, "cudaGraphLaunch");
        ++sweeps;
        if (!o.fixed) {
            if ((e = cudaMemcpyAsync(c->h_maxd, c->d_maxd, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
                return cuda_error(e, "cudaMemcpyAsync");
            if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "sweep");
            memcpy(&delta, c->h_maxd, 8);
            if (delta <= o.tol) break;
        }
    }
    if ((e = cudaEventRecord(c->ev1, s)) != cudaSuccess) return cuda_error(e, "cudaEventRecord");
    if ((e = cudaMemcpyAsync(c->h_maxd, c->d_maxd, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_error(e, "cudaMemcpyAsync");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "solve");
    memcpy(&delta, c->h_maxd, 8);
    if (rep) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        rep->sweeps = sweeps;
        rep->max_delta = delta;
        rep->elapsed_ms = ms;
        rep->nominal_updates = nominal_per_sweep(g) * (uint64_t)sweeps;
        rep->evaluated_updates = rep->nominal_updates;
        rep->engine = FOLD3D_ENGINE_PLANES;
    }
    return FOLD3D_OK;
}

// WAVEFRONT tiles (32 x kWaveTV) per plane of the orientation with normal axis b.
static void orient_tiles(const fold3d_grid &g, int b, int &ntu, int &ntv, int tv = kWaveTV)
{
    const int n[3] = {g.nx, g.ny, g.nz};
    const int ub = (b == 0) ? 1 : 0, vb = (b == 2) ? 1 : 2;
    ntu = (n[ub] + 31) / 32;
    ntv = (n[vb] + tv - 1) / tv;
}

// Pass numbers travel as (pass << 1) | changed in 32-bit flags.  Far before
// that overflows, every flag and change map is cleared and numbering restarts.
static int reserve_passes(fold3d_ctx *c, unsigned passes)
{
    if (c->epoch + passes < (1u << 30)) return FOLD3D_OK;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_error(e, "cudaDeviceSynchronize");
    if (c->w_flags) {
        c->key_wg = fold3d_grid{};
        cudaFree(c->w_flags);
        c->w_flags = nullptr;
    }
    if (c->b_scratch) {
        cudaFree(c->b_scratch);
        c->b_scratch = nullptr;
    }
    c->bkey.clear();
    c->epoch = 0;
    return FOLD3D_OK;
}

static int wave_scratch(fold3d_ctx *c, const fold3d_grid &g)
{
    if (c->w_flags && c->key_wg.nx == g.nx && c->key_wg.ny == g.ny && c->key_wg.nz == g.nz) return FOLD3D_OK;
    if (c->w_flags) cudaFree(c->w_flags);
    for (int b = 0; b < 3; ++b) {
        if (c->w_mod[b]) cudaFree(c->w_mod[b]);
        c->w_mod[b] = nullptr;
    }
    c->w_flags = nullptr;
    const int n[3] = {g.nx, g.ny, g.nz};
    size_t flag_words = 0;
    cudaError_t e;
    for (int b = 0; b < 3; ++b) {
        int ntu, ntv;
        orient_tiles(g, b, ntu, ntv);
        flag_words = std::max(flag_words, (size_t)(n[b] - 1) * ntu * ntv);
        const size_t words = (size_t)(n[b] + 2) * ntu * ntv;
        if ((e = cudaMalloc(&c->w_mod[b], words * 4)) != cudaSuccess ||
            (e = cudaMemset(c->w_mod[b], 0, words * 4)) != cudaSuccess)
            return set_errorf(FOLD3D_ERR_NOMEM, "wavefront scratch: %s", cudaGetErrorString(e));
    }
    if ((e = cudaMalloc(&c->w_flags, flag_words * 4)) != cudaSuccess ||
        (e = cudaMemset(c->w_flags, 0, flag_words * 4)) != cudaSuccess)
        return set_errorf(FOLD3D_ERR_NOMEM, "wavefront scratch: %s", cudaGetErrorString(e));
    if (!c->w_counters) {
        if ((e = cudaMalloc(&c->w_counters, 2 * sizeof(unsigned))) != cudaSuccess ||
            (e = cudaMalloc(&c->w_evaluated, sizeof(unsigned long long))) != cudaSuccess)
            return set_errorf(FOLD3D_ERR_NOMEM, "wavefront scratch: %s", cudaGetErrorString(e));
    }
    if (!c->sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev);
    }
    c->key_wg = g;  // fresh flags and maps are zero, below every pass number to come
    return FOLD3D_OK;
}

// Elliptical-medium constants of a sweep direction.
static EllipParam ellip_param(const fold3d_grid &g, const EllipMedium &m, int dir)
{
    const DirSpec &d = kDirs[dir];
    const double h[3] = {g.dx, g.dy, g.dz};
    static const int pair[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    EllipParam p;
    memset(&p, 0, sizeof p);
    p.dir.hx = h[d.xa];
    p.dir.hy = h[d.ya];
    p.dir.hz = h[d.nrm];
    p.dir.sxy = d.xs * d.ys;
    p.dir.sxz = d.xs * d.sg;
    p.dir.syz = d.ys * d.sg;
    p.dir.ixx = pair[d.xa][d.xa];
    p.dir.iyy = pair[d.ya][d.ya];
    p.dir.izz = pair[d.nrm][d.nrm];
    p.dir.ixy = pair[d.xa][d.ya];
    p.dir.ixz = pair[d.xa][d.nrm];
    p.dir.iyz = pair[d.ya][d.nrm];
    p.med = m;
    return p;
}

// T: double, or float when f32 (elliptical medium only).
static int solve_wavefront(fold3d_ctx *c, const fold3d_grid &g, const fold3d_medium *fm, const EllipMedium *em,
                           void *T, bool f32, const fold3d_opts &o, cudaStream_t s, fold3d_report *rep,
                           unsigned char *winners = nullptr)
{
    int rc = reserve_passes(c, 6u * (unsigned)std::min(o.max_sweeps, 1 << 20) + 12u);
    if (rc) return rc;
    if ((rc = wave_scratch(c, g))) return rc;
    cudaError_t e;
    if ((e = cudaMemsetAsync(c->w_counters, 0, 2 * sizeof(unsigned), s)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->w_evaluated, 0, sizeof(unsigned long long), s)) != cudaSuccess)
        return cuda_error(e, "cudaMemsetAsync");
    WaveArgs a;
    memset(&a, 0, sizeof a);
    for (int b = 0; b < 3; ++b) {
        int ntu, ntv;
        orient_tiles(g, b, ntu, ntv);
        a.mod[b] = c->w_mod[b];
        a.mod_ntu[b] = ntu;
        a.mod_ntiles[b] = ntu * ntv;
    }
    a.flags = c->w_flags;
    a.work = c->w_counters;
    a.status = c->w_counters + 1;
    a.maxd = c->d_maxd;
    a.evaluated = c->w_evaluated;
    a.timeout_ns = 4000000000ull;
    const unsigned e0 = c->epoch + 1;
    a.skip_from = o.skip ? e0 + 6 : 0xffffffffu;
    if ((e = cudaEventRecord(c->ev0, s)) != cudaSuccess) return cuda_error(e, "cudaEventRecord");
    int sweeps = 0;
    double delta = 0.0;
    unsigned hstat[2] = {0, 0};
    DirTable tab;
    while (sweeps < o.max_sweeps) {
        if ((e = cudaMemsetAsync(c->d_maxd, 0, sizeof(unsigned long long), s)) != cudaSuccess)
            return cuda_error(e, "cudaMemsetAsync");
        for (int dir = 0; dir < 6; ++dir) {
            const DirSpec &d = kDirs[dir];
            a.pg = make_geom(g, dir);
            a.nrm = d.nrm;
            a.ua = (d.nrm == 0) ? 1 : 0;
            a.va = (d.nrm == 2) ? 1 : 2;
            a.sg = d.sg;
            orient_tiles(g, d.nrm, a.ntu, a.ntv);
            a.steps = pass_count(a.pg);
            a.first_src = pass_first(a.pg, dir);
            a.epoch = ++c->epoch;
            a.dir = dir;
            a.winners = winners;
            const long long items = (long long)a.steps * a.ntu * a.ntv;
            const bool large = (long long)a.ntu * a.ntv >= kLargePlaneTiles;
            int &bps = c->wave_bps[em ? 1 : 0][f32 ? 1 : 0][large ? 1 : 0];
            if (!bps) bps = wave_blocks_per_sm(em ? kMediumEllip : kMediumDrift, f32, large);
            const int grid = (int)std::min<long long>(items, (long long)c->sms * bps);
            if ((e = cudaMemsetAsync(a.work, 0, sizeof(unsigned), s)) != cudaSuccess)
                return cuda_error(e, "cudaMemsetAsync");
            if (em) {
                e = launch_wave_pass_ellip(T, f32, a, ellip_param(g, *em, dir), grid, s, large);
            } else {
                build_dir_table(make_frame(g, *fm, dir), tab);
                e = launch_wave_pass(static_cast<double *>(T), a, tab, grid, s, large);
            }
            if (e != cudaSuccess) return cuda_error(e, "wavefront pass");
        }
        ++sweeps;
        if (!o.fixed) {
            if ((e = cudaMemcpyAsync(c->h_maxd, c->d_maxd, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaMemcpyAsync(hstat, c->w_counters, sizeof hstat, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
                return cuda_error(e, "cudaMemcpyAsync");
            if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "sweep");
            if (hstat[1]) return set_error(FOLD3D_ERR_TIMEOUT, "wavefront: a dependency wait gave up");
            memcpy(&delta, c->h_maxd, 8);
            if (delta <= o.tol) break;
        }
    }
    if ((e = cudaEventRecord(c->ev1, s)) != cudaSuccess) return cuda_error(e, "cudaEventRecord");
    unsigned long long evald = 0;
    if ((e = cudaMemcpyAsync(c->h_maxd, c->d_maxd, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hstat, c->w_counters, sizeof hstat, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&evald, c->w_evaluated, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_error(e, "cudaMemcpyAsync");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "solve");
    if (hstat[1]) return set_error(FOLD3D_ERR_TIMEOUT, "wavefront: a dependency wait gave up");
    memcpy(&delta, c->h_maxd, 8);
    if (rep) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        rep->sweeps = sweeps;
        rep->max_delta = delta;
        rep->elapsed_ms = ms;
        rep->nominal_updates = nominal_per_sweep(g) * (uint64_t)sweeps;
        rep->evaluated_updates = evald;
        rep->engine = FOLD3D_ENGINE_WAVEFRONT;
    }
    return FOLD3D_OK;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
static constexpr size_t kStageInst = sizeof(BatchInst) > sizeof(BatchAdjInst) ? sizeof(BatchInst) : sizeof(BatchAdjInst);

// Device state of the batched sweep loop: total[6], epoch_base, sweep[2],
// then active[n], sweeps[n] and delta[n].
static size_t batch_ctl_bytes(int n) { return 64 + align_up((size_t)n * 4, 256) * 2 + (size_t)n * 8; }
struct BatchCtlMem {
    unsigned *total, *epoch_base;
    int *sweep, *active, *sweeps;
    double *delta;
};
static BatchCtlMem batch_ctl_mem(char *base, int n)
{
    BatchCtlMem m;
    m.total = reinterpret_cast<unsigned *>(base);
    m.epoch_base = m.total + 6;
    m.sweep = reinterpret_cast<int *>(base + 32);
    m.active = reinterpret_cast<int *>(base + 64);
    m.sweeps = reinterpret_cast<int *>(base + 64 + align_up((size_t)n * 4, 256));
    m.delta = reinterpret_cast<double *>(base + 64 + 2 * align_up((size_t)n * 4, 256));
    return m;
}

static int batch_scratch(fold3d_ctx *c, const std::vector<fold3d_grid> &grids, int tv = kWaveTV)
{
    const int n = (int)grids.size();
    std::vector<int> key(3 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        key[3 * i] = grids[i].nx;
        key[3 * i + 1] = grids[i].ny;
        key[3 * i + 2] = grids[i].nz;
    }
    if (c->b_scratch && key == c->bkey && tv == c->btv) return FOLD3D_OK;
    if (c->b_scratch) cudaFree(c->b_scratch);
    if (c->b_slots) cudaFree(c->b_slots);
    if (c->b_stage_d) cudaFree(c->b_stage_d);
    if (c->b_stage_h) cudaFreeHost(c->b_stage_h);
    if (c->b_ctl) cudaFree(c->b_ctl);
    c->b_scratch = nullptr;
    c->b_slots = nullptr;
    c->b_stage_d = c->b_stage_h = nullptr;
    c->b_ctl = nullptr;
    c->bkey.clear();
    size_t words = 0;
    int max_steps = 0;
    c->b_flag_off.assign(n, 0);
    for (int b = 0; b < 3; ++b) c->b_mod_off[b].assign(n, 0);
    for (int i = 0; i < n; ++i) {
        const fold3d_grid &g = grids[i];
        const int dims[3] = {g.nx, g.ny, g.nz};
        size_t fw = 0;
        for (int b = 0; b < 3; ++b) {
            int ntu, ntv;
            orient_tiles(g, b, ntu, ntv, tv);
            fw = std::max(fw, (size_t)(dims[b] - 1) * ntu * ntv);
            c->b_mod_off[b][i] = words;
            words += (size_t)(dims[b] + 2) * ntu * ntv;
            max_steps = std::max(max_steps, dims[b] - 1);
        }
        c->b_flag_off[i] = words;
        words += fw;
    }
    cudaError_t e;
    if ((e = cudaMalloc(&c->b_scratch, words * 4)) != cudaSuccess ||
        (e = cudaMemset(c->b_scratch, 0, words * 4)) != cudaSuccess ||
        (e = cudaMalloc(&c->b_slots, 2 * (size_t)n * 8)) != cudaSuccess)
        return set_errorf(FOLD3D_ERR_NOMEM, "batch scratch: %s", cudaGetErrorString(e));
    if (!c->b_counters && (e = cudaMalloc(&c->b_counters, 2 * sizeof(unsigned))) != cudaSuccess)
        return set_errorf(FOLD3D_ERR_NOMEM, "batch scratch: %s", cudaGetErrorString(e));
    // per direction: inst[n], step_off[max_steps+1], step_k[max_steps], tile_pre[n+1], then the
    // device loop's order[n], steps[n], tiles[n] and act[n]
    const size_t per = align_up((size_t)n * kStageInst, 256) + align_up((max_steps + 1) * 8, 256) +
                       align_up((size_t)max_steps * 4, 256) + align_up(((size_t)n + 1) * 8, 256) +
                       2 * align_up((size_t)n * 4, 256) + align_up((size_t)n * 8, 256) + align_up((size_t)n * 4, 256);
    c->b_stage_bytes = per;
    if ((e = cudaMalloc(&c->b_stage_d, 6 * per)) != cudaSuccess ||
        (e = cudaMallocHost(&c->b_stage_h, 6 * per)) != cudaSuccess ||
        (e = cudaMalloc(&c->b_ctl, batch_ctl_bytes(n))) != cudaSuccess)
        return set_errorf(FOLD3D_ERR_NOMEM, "batch staging: %s", cudaGetErrorString(e));
    if (!c->sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev);
    }
    if (!c->batch_adj_bps) c->batch_adj_bps = batch_adj_blocks_per_sm(false);
    c->bkey = key;
    c->btv = tv;
    return FOLD3D_OK;
}

// Staging layout of direction dir: pointers into the host or device copy.
// The instance table holds BatchInst (forward) or BatchAdjInst (adjoint).
struct BatchStage {
    void *inst;
    long long *step_off;
    int *step_k;
    long long *tile_pre;
    int *order, *steps;
    long long *tiles;
    int *act;
};
static BatchStage batch_stage(fold3d_ctx *c, char *base, int dir, int n)
{
    int max_steps = 0;
    for (size_t i = 0; i < c->bkey.size(); ++i) max_steps = std::max(max_steps, c->bkey[i] - 1);
    char *p = base + (size_t)dir * c->b_stage_bytes;
    BatchStage s;
    s.inst = p;
    p += align_up((size_t)n * kStageInst, 256);
    s.step_off = reinterpret_cast<long long *>(p);
    p += align_up((max_steps + 1) * 8, 256);
    s.step_k = reinterpret_cast<int *>(p);
    p += align_up((size_t)max_steps * 4, 256);
    s.tile_pre = reinterpret_cast<long long *>(p);
    p += align_up(((size_t)n + 1) * 8, 256);
    s.order = reinterpret_cast<int *>(p);
    p += align_up((size_t)n * 4, 256);
    s.steps = reinterpret_cast<int *>(p);
    p += align_up((size_t)n * 4, 256);
    s.tiles = reinterpret_cast<long long *>(p);
    p += align_up((size_t)n * 8, 256);
    s.act = reinterpret_cast<int *>(p);
    return s;
}

// Instances of the batched drivers: fields of doubles, or of floats (f32).
// Internal medium of the elliptical solvers from the public structs.
static EllipMedium medium_of(const fold3d_ellip &m)
{
    EllipMedium e;
    const float *arr[6] = {m.mxx, m.mxy, m.mxz, m.myy, m.myz, m.mzz};
    for (int k = 0; k < 6; ++k) e.m[k] = arr[k];
    e.kind = kMetricF32;
    return e;
}
static EllipMedium medium_of(const fold3d_tti &m)
{
    EllipMedium e;
    const double *arr[4] = {m.s, m.eps, m.nx, m.ny};
    for (int k = 0; k < 4; ++k) e.m[k] = arr[k];
    e.m[4] = e.m[5] = nullptr;
    e.kind = kParamF64;
    return e;
}

struct SolveInst {
    fold3d_grid grid;
    EllipMedium medium;
    void *T;
    unsigned char *winners;
};
struct AdjInst {
    fold3d_grid grid;
    EllipMedium medium;
    const void *T;
    const unsigned char *winners;
    const void *dLdT;
    void *lambda;
    void *dLdM;
};

// Batched solve: the whole sweep loop runs on the device as one CUDA graph.
// Its prologue builds the item tables; a conditional while-node repeats the
// body -- the six directions' batched passes, then the restage kernel, which
// folds each instance's change into its state, drops converged instances,
// rebuilds the tables and decides whether to loop again -- so the host
// neither waits nor re-stages between sweeps.  The host only writes the
// per-direction instance tables once (every instance, in the direction's
// order) and reads the per-instance results at the end.  tv, bps: tile
// height and resident CTAs per SM.
static int solve_batch_cfg(fold3d_ctx *c, int n, const SolveInst *in, bool f32, const fold3d_opts &o, cudaStream_t s,
                           fold3d_report *reps, int tv, int bps)
{
    int rc = reserve_passes(c, 6u * (unsigned)std::min(o.max_sweeps, 1 << 20) + 12u);
    if (rc) return rc;
    std::vector<fold3d_grid> grids(n);
    for (int i = 0; i < n; ++i) grids[i] = in[i].grid;
    if ((rc = batch_scratch(c, grids, tv))) return rc;
    cudaError_t e;
    const unsigned e0 = c->epoch + 1;
    const unsigned skip_from = o.skip ? e0 + 6 : 0xffffffffu;
    int max_steps = 0;
    for (int v : c->bkey) max_steps = std::max(max_steps, v - 1);
    const BatchCtlMem cm = batch_ctl_mem(c->b_ctl, n);
    BatchArgs args[6];
    BatchCtl ctl;
    memset(&ctl, 0, sizeof ctl);
    long long max_total = 0;
    for (int dir = 0; dir < 6; ++dir) {
        const DirSpec &d = kDirs[dir];
        BatchStage h = batch_stage(c, c->b_stage_h, dir, n);
        BatchStage dv = batch_stage(c, c->b_stage_d, dir, n);
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        auto steps_of = [&](int i) {
            const int dims[3] = {in[i].grid.nx, in[i].grid.ny, in[i].grid.nz};
            return dims[d.nrm] - 1;
        };
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return steps_of(x) > steps_of(y); });
        long long items = 0;
        for (int q = 0; q < n; ++q) {
            const int i = order[q];
            const fold3d_grid &g = in[i].grid;
            BatchInst &bi = static_cast<BatchInst *>(h.inst)[q];
            memset(&bi, 0, sizeof bi);
            WaveArgs &a = bi.a;
            a.pg = make_geom(g, dir);
            a.nrm = d.nrm;
            a.ua = (d.nrm == 0) ? 1 : 0;
            a.va = (d.nrm == 2) ? 1 : 2;
            a.sg = d.sg;
            orient_tiles(g, d.nrm, a.ntu, a.ntv, tv);
            a.steps = pass_count(a.pg);
            a.first_src = pass_first(a.pg, dir);
            a.timeout_ns = 4000000000ull;
            a.flags = c->b_scratch + c->b_flag_off[i];
            for (int b = 0; b < 3; ++b) {
                int ntu, ntv;
                orient_tiles(g, b, ntu, ntv, tv);
                a.mod[b] = c->b_scratch + c->b_mod_off[b][i];
                a.mod_ntu[b] = ntu;
                a.mod_ntiles[b] = ntu * ntv;
            }
            a.work = c->b_counters;
            a.status = c->b_counters + 1;
            a.maxd = c->b_slots + i;
            a.evaluated = c->b_slots + n + i;
            a.dir = dir;
            a.winners = in[i].winners;
            bi.p = ellip_param(g, in[i].medium, dir);
            bi.T = in[i].T;
            h.order[q] = i;
            h.steps[q] = a.steps;
            h.tiles[q] = (long long)a.ntu * a.ntv;
            items += h.tiles[q] * a.steps;
        }
        if (items >= (1ll << 31)) return set_error(FOLD3D_ERR_UNSUPPORTED, "batch too large");
        max_total = std::max(max_total, items);
        BatchDirTables &t = ctl.dir[dir];
        t.order = dv.order;
        t.steps = dv.steps;
        t.tiles = dv.tiles;
        t.act = dv.act;
        t.step_off = dv.step_off;
        t.step_k = dv.step_k;
        t.tile_pre = dv.tile_pre;
        args[dir].inst = static_cast<const BatchInst *>(dv.inst);
        args[dir].act = dv.act;
        args[dir].step_off = dv.step_off;
        args[dir].step_k = dv.step_k;
        args[dir].tile_pre = dv.tile_pre;
        args[dir].total = cm.total + dir;
        args[dir].epoch_base = cm.epoch_base;
        args[dir].max_steps = max_steps;
        args[dir].dir = dir;
        args[dir].work = c->b_counters;
        args[dir].status = c->b_counters + 1;
        args[dir].skip_from = skip_from;
    }
    ctl.n = n;
    ctl.max_steps = max_steps;
    ctl.fixed = o.fixed ? 1 : 0;
    ctl.max_sweeps = o.max_sweeps;
    ctl.tol = o.tol;
    ctl.epoch0 = e0 - 1;
    ctl.total = cm.total;
    ctl.epoch_base = cm.epoch_base;
    ctl.sweep = cm.sweep;
    ctl.active = cm.active;
    ctl.sweeps = cm.sweeps;
    ctl.delta = cm.delta;
    ctl.maxd = c->b_slots;
    ctl.status = c->b_counters + 1;
    // a grid as large as the biggest pass can use (instances drop out later)
    const int grid = (int)std::min<long long>(max_total, (long long)c->sms * bps);

    // the graph: prologue (tables), then while (more) { six passes; restage }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto fail = [&](cudaError_t err, const char *what) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        return cuda_error(err, what);
    };
    if ((e = cudaMemcpyAsync(c->b_stage_d, c->b_stage_h, 6 * c->b_stage_bytes, cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemsetAsync(c->b_counters, 0, 2 * sizeof(unsigned), s)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->b_slots + n, 0, (size_t)n * 8, s)) != cudaSuccess)
        return cuda_error(e, "batch setup");
    if ((e = cudaGraphCreate(&graph, 0)) != cudaSuccess) return cuda_error(e, "cudaGraphCreate");
    cudaGraphConditionalHandle cond;
    if ((e = cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess)
        return fail(e, "cudaGraphConditionalHandleCreate");
    ctl.cond = (unsigned long long)cond;
    cudaStream_t cs = c->stream;  // the context's own stream captures; the graph runs on s
    cudaError_t le = cudaSuccess;
    if ((e = cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return fail(e, "cudaStreamBeginCaptureToGraph");
    le = launch_batch_restage(ctl, true, cs);
    if ((e = cudaStreamEndCapture(cs, &graph)) != cudaSuccess || le != cudaSuccess)
        return fail(le != cudaSuccess ? le : e, "capturing the batch prologue");
    cudaGraphNode_t pro = nullptr;
    size_t nn = 1;
    if ((e = cudaGraphGetNodes(graph, &pro, &nn)) != cudaSuccess || nn != 1)
        return fail(e != cudaSuccess ? e : cudaErrorUnknown, "batch prologue");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop = nullptr;
    if ((e = cudaGraphAddNode(&loop, graph, &pro, 1, &cp)) != cudaSuccess) return fail(e, "conditional node");
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess)
        return fail(e, "cudaStreamBeginCaptureToGraph");
    for (int dir = 0; dir < 6 && le == cudaSuccess; ++dir) {
        le = cudaMemsetAsync(c->b_counters, 0, sizeof(unsigned), cs);
        if (le == cudaSuccess && grid > 0) le = launch_batch_pass(args[dir], f32, tv, grid, cs);
    }
    if (le == cudaSuccess) le = launch_batch_restage(ctl, false, cs);
    if ((e = cudaStreamEndCapture(cs, &body)) != cudaSuccess || le != cudaSuccess)
        return fail(le != cudaSuccess ? le : e, "capturing the batch sweep");
    if ((e = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess) return fail(e, "cudaGraphInstantiate");
    if ((e = cudaEventRecord(c->ev0, s)) != cudaSuccess || (e = cudaGraphLaunch(exec, s)) != cudaSuccess ||
        (e = cudaEventRecord(c->ev1, s)) != cudaSuccess)
        return fail(e, "batch graph");
    std::vector<unsigned long long> evald(n);
    std::vector<int> sweeps(n);
    std::vector<double> delta(n);
    int loop_state[2] = {0, 0};
    unsigned hstat[2] = {0, 0};
    if ((e = cudaMemcpyAsync(evald.data(), c->b_slots + n, (size_t)n * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(sweeps.data(), cm.sweeps, (size_t)n * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(delta.data(), cm.delta, (size_t)n * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(loop_state, cm.sweep, sizeof loop_state, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hstat, c->b_counters, sizeof hstat, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fail(e, "batch");
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    c->epoch = e0 - 1 + 6u * (unsigned)loop_state[0];  // passes the loop numbered
    if (hstat[1]) return set_error(FOLD3D_ERR_TIMEOUT, "batch: a dependency wait gave up");
    if (reps) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        for (int i = 0; i < n; ++i) {
            reps[i].sweeps = sweeps[i];
            reps[i].max_delta = delta[i];
            reps[i].elapsed_ms = ms;
            reps[i].nominal_updates = nominal_per_sweep(in[i].grid) * (uint64_t)sweeps[i];
            reps[i].evaluated_updates = evald[i];
            reps[i].engine = FOLD3D_ENGINE_WAVEFRONT;
        }
    }
    return FOLD3D_OK;
}

// Resident batched-pass CTAs per SM at tile height tv (the occupancy limit).
static int batch_occupancy_of(fold3d_ctx *c, bool f32, int tv)
{
    int &v = c->batch_bps[f32 ? 1 : 0][tv];
    if (!v) v = batch_blocks_per_sm(f32, tv);
    return v;
}

// The batch autotuner.  For a size mix it has not seen (number of instances,
// total and largest extent, field type), it times one full sweep of each
// candidate tile height -- 2, 4 and 8 rows (64, 128 and 256 threads per CTA),
// each at its occupancy limit of resident CTAs per SM -- on copies of
// instances of median size, as many as it takes to give every resident CTA
// work (at least kTuneCells cells; the caller's fields are not touched), and
// keeps the fastest for the size mix.  Every configuration gives the same
// results bit for bit; they differ only in speed.  (Fewer resident CTAs than
// the limit were candidates too, but on a sample they won where the whole
// batch then ran slower, and they never won on a whole batch.)
static int batch_config(fold3d_ctx *c, int n, const SolveInst *in, bool f32, cudaStream_t s, int &tv, int &bps)
{
    if (!c->sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev);
    }
    if (c->tune_tv > 0) {  // fixed by fold3d_batch_set_config
        tv = c->tune_tv;
        const int occ = batch_occupancy_of(c, f32, tv);
        bps = c->tune_bps > 0 ? std::min(c->tune_bps, occ) : occ;
        return FOLD3D_OK;
    }
    if (n < 8) {  // too few instances to be worth a tuning run
        tv = kWaveTV;
        bps = batch_occupancy_of(c, f32, tv);
        return FOLD3D_OK;
    }
    long long total = 0, big = 0;
    std::vector<std::pair<size_t, int>> by_size(n);
    for (int i = 0; i < n; ++i) {
        const fold3d_grid &g = in[i].grid;
        total += (long long)g.nx * g.ny * g.nz;
        big = std::max<long long>(big, std::max(g.nx, std::max(g.ny, g.nz)));
        by_size[i] = {field_cells(g), i};
    }
    const std::vector<long long> key = {n, f32 ? 1 : 0, (long long)std::llround(4.0 * std::log2((double)total)),
                                        (long long)std::llround(4.0 * std::log2((double)big))};
    auto hit = c->tuned.find(key);
    if (hit != c->tuned.end()) {
        tv = hit->second.first;
        bps = hit->second.second;
        return FOLD3D_OK;
    }
    // instances around the median size, enough to fill the GPU, on copies of their fields
    std::sort(by_size.begin(), by_size.end());
    constexpr size_t kTuneCells = (size_t)64 << 20;
    int lo = n / 2, hi = n / 2;  // the sample: sorted positions [lo, hi), grown around the median
    size_t cells = 0;
    while (hi - lo < n && cells < kTuneCells) {
        if (hi < n && ((hi - lo) % 2 == 0 || lo == 0)) cells += by_size[hi++].first;
        else cells += by_size[--lo].first;
    }
    const int k = hi - lo, first = lo;
    const size_t esz = f32 ? sizeof(float) : sizeof(double);
    cudaError_t e;
    if (c->tune_cells * sizeof(double) < cells * esz) {
        if (c->tune_T) cudaFree(c->tune_T);
        c->tune_T = nullptr;
        c->tune_cells = 0;
        if ((e = cudaMalloc(&c->tune_T, cells * esz)) != cudaSuccess)
            return set_error(FOLD3D_ERR_NOMEM, "batch autotuner scratch");
        c->tune_cells = (cells * esz + sizeof(double) - 1) / sizeof(double);
    }
    std::vector<SolveInst> sub(k);
    size_t off = 0;
    for (int q = 0; q < k; ++q) {
        const SolveInst &src = in[by_size[first + q].second];
        sub[q] = src;
        sub[q].T = reinterpret_cast<char *>(c->tune_T) + off * esz;
        sub[q].winners = nullptr;
        off += field_cells(src.grid);
    }
    fold3d_opts one;
    fold3d_default_opts(&one);
    one.max_sweeps = 1;
    one.fixed = 1;
    one.skip = 0;
    std::vector<fold3d_report> r(k);
    double best = 1e300;
    tv = kWaveTV;
    bps = batch_occupancy_of(c, f32, tv);
    for (int ctv : {2, 4, 8}) {
        const int cb = batch_occupancy_of(c, f32, ctv);
        for (int q = 0; q < k; ++q) {
            const SolveInst &src = in[by_size[first + q].second];
            const size_t bytes = field_cells(src.grid) * esz;
            if ((e = cudaMemcpyAsync(sub[q].T, src.T, bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
                return cuda_error(e, "batch autotuner");
        }
        int rc = solve_batch_cfg(c, k, sub.data(), f32, one, s, r.data(), ctv, cb);
        if (rc) return rc;
        if (r[0].elapsed_ms < best) {
            best = r[0].elapsed_ms;
            tv = ctv;
            bps = cb;
        }
    }
    c->tuned[key] = {tv, bps};
    return FOLD3D_OK;
}

static int solve_batch(fold3d_ctx *c, int n, const SolveInst *in, bool f32, const fold3d_opts &o, cudaStream_t s,
                       fold3d_report *reps)
{
    int tv = kWaveTV, bps = 1;
    int rc = batch_config(c, n, in, f32, s, tv, bps);
    if (rc) return rc;
    c->last_tv = tv;
    c->last_bps = bps;
    return solve_batch_cfg(c, n, in, f32, o, s, reps, tv, bps);
}

// Adjoint scratch (lambda already pushed) for `cells` cells.
static int adj_scratch(fold3d_ctx *c, size_t cells)
{
    if (c->adj_cells >= cells) return FOLD3D_OK;
    if (c->adj_pushed) cudaFree(c->adj_pushed);
    c->adj_pushed = nullptr;
    c->adj_cells = 0;
    if (cudaMalloc(&c->adj_pushed, cells * sizeof(double)) != cudaSuccess)
        return set_error(FOLD3D_ERR_NOMEM, "adjoint scratch");
    c->adj_cells = cells;
    return FOLD3D_OK;
}

// Bytes of one grid's adjoint work maps (six directions).
static size_t adj_tiles_bytes(const fold3d_grid &g)
{
    const int n[3] = {g.nx, g.ny, g.nz};
    size_t bytes = 0;
    for (int d = 0; d < 6; ++d) {
        int ntu, ntv;
        orient_tiles(g, kDirs[d].nrm, ntu, ntv);
        bytes += (size_t)(n[kDirs[d].nrm] + 2) * ntu * ntv;
    }
    return bytes;
}

// Lays out one grid's work maps at base, clears them and fills them from its
// winner record.
static int adj_tiles(const fold3d_grid &g, const unsigned char *W, unsigned char *base, AdjTiles &t, cudaStream_t s)
{
    const int n[3] = {g.nx, g.ny, g.nz};
    for (int b = 0; b < 3; ++b) {
        int ntv;
        orient_tiles(g, b, t.ntu[b], ntv);
        t.ntiles[b] = t.ntu[b] * ntv;
    }
    size_t at = 0;
    for (int d = 0; d < 6; ++d) {
        t.nrm[d] = kDirs[d].nrm;
        t.has[d] = base + at;
        at += (size_t)(n[t.nrm[d]] + 2) * t.ntiles[t.nrm[d]];
    }
    cudaError_t e;
    if ((e = cudaMemsetAsync(base, 0, at, s)) != cudaSuccess ||
        (e = launch_adj_tiles(W, g, t, s)) != cudaSuccess)
        return cuda_error(e, "adjoint work map");
    return FOLD3D_OK;
}

static int adj_has_scratch(fold3d_ctx *c, size_t bytes)
{
    if (c->adj_has_bytes >= bytes) return FOLD3D_OK;
    if (c->adj_has) cudaFree(c->adj_has);
    c->adj_has = nullptr;
    c->adj_has_bytes = 0;
    if (cudaMalloc(&c->adj_has, bytes) != cudaSuccess) return set_error(FOLD3D_ERR_NOMEM, "adjoint work maps");
    c->adj_has_bytes = bytes;
    return FOLD3D_OK;
}

static int adj_list_scratch(fold3d_ctx *c, size_t items, size_t counts)
{
    if (c->adj_items_cap < items) {
        if (c->adj_items) cudaFree(c->adj_items);
        c->adj_items = nullptr;
        c->adj_items_cap = 0;
        if (cudaMalloc(&c->adj_items, items * 8) != cudaSuccess)
            return set_error(FOLD3D_ERR_NOMEM, "adjoint item lists");
        c->adj_items_cap = items;
    }
    if (c->adj_cnt_cap < counts) {
        if (c->adj_cnt) cudaFree(c->adj_cnt);
        if (c->adj_off) cudaFree(c->adj_off);
        c->adj_cnt = nullptr;
        c->adj_off = nullptr;
        c->adj_cnt_cap = 0;
        if (cudaMalloc(&c->adj_cnt, counts * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&c->adj_off, counts * sizeof(long long)) != cudaSuccess)
            return set_error(FOLD3D_ERR_NOMEM, "adjoint item lists");
        c->adj_cnt_cap = counts;
    }
    return FOLD3D_OK;
}

static int adjoint_batch(fold3d_ctx *c, int n, const AdjInst *in, bool f32, int max_sweeps, double tol,
                         int accumulate, cudaStream_t s, fold3d_report *reps)
{
    int rc = reserve_passes(c, 6u * (unsigned)std::min(max_sweeps, 1 << 20) + 12u);
    if (rc) return rc;
    std::vector<fold3d_grid> grids(n);
    for (int i = 0; i < n; ++i) grids[i] = in[i].grid;
    if ((rc = batch_scratch(c, grids))) return rc;
    std::vector<size_t> off(n + 1, 0);
    for (int i = 0; i < n; ++i) off[i + 1] = off[i] + field_cells(in[i].grid);
    if ((rc = adj_scratch(c, off[n]))) return rc;  // doubles: room for floats too
    const size_t esz = f32 ? sizeof(float) : sizeof(double);
    std::vector<size_t> hoff(n + 1, 0);
    for (int i = 0; i < n; ++i) hoff[i + 1] = hoff[i] + adj_tiles_bytes(in[i].grid);
    if ((rc = adj_has_scratch(c, hoff[n]))) return rc;
    std::vector<AdjTiles> tiles(n);
    for (int i = 0; i < n; ++i)
        if ((rc = adj_tiles(in[i].grid, in[i].winners, c->adj_has + hoff[i], tiles[i], s))) return rc;
    // item lists: direction dir's at item_off[dir], at most every (step, tile) of every instance
    size_t item_off[7] = {0};
    for (int dir = 0; dir < 6; ++dir) {
        size_t cap = 0;
        for (int i = 0; i < n; ++i) {
            const int dims[3] = {in[i].grid.nx, in[i].grid.ny, in[i].grid.nz};
            int ntu, ntv;
            orient_tiles(in[i].grid, kDirs[dir].nrm, ntu, ntv);
            cap += (size_t)(dims[kDirs[dir].nrm] - 1) * ntu * ntv;
        }
        item_off[dir + 1] = item_off[dir] + cap;
    }
    cudaError_t e;
    for (int i = 0; i < n; ++i)
        if ((e = cudaMemcpyAsync(in[i].lambda, in[i].dLdT, field_cells(in[i].grid) * esz, cudaMemcpyDeviceToDevice,
                                 s)) != cudaSuccess)
            return cuda_error(e, "adjoint setup");
    if ((e = cudaMemsetAsync(c->adj_pushed, 0, off[n] * esz, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->b_counters, 0, 2 * sizeof(unsigned), s)) != cudaSuccess)
        return cuda_error(e, "adjoint setup");
    std::vector<char> active(n, 1);
    std::vector<int> sweeps(n, 0);
    std::vector<double> delta(n, 0.0), first(n, 0.0);
    std::vector<unsigned long long> slots(n);
    int max_steps = 0;
    for (int v : c->bkey) max_steps = std::max(max_steps, v - 1);
    if ((rc = adj_list_scratch(c, item_off[6], (size_t)max_steps * n + 1))) return rc;
    std::vector<int> cnt((size_t)max_steps * n);
    std::vector<long long> offs((size_t)max_steps * n + 1);
    BatchAdjArgs args[6];
    // The launches of each direction's backward pass: one over every active
    // instance, except for the x-normal passes, whose planes have no
    // contiguous axis: there every cell of an instance's plane sits in its
    // own 32-byte sectors of the field, lambda, pushed amounts and winner
    // record, which later plane steps reuse only while they stay in L2.  Those
    // passes run over groups of instances whose sectors fit in kAdjXGroupBytes
    // of L2 together, one launch per group.
    std::vector<BatchAdjArgs> launches[6];
    int slots_k[6] = {0, 0, 0, 0, 0, 0};
    auto stage = [&]() -> int {
        for (int dir = 0; dir < 6; ++dir) {
            const DirSpec &d = kDirs[dir];
            BatchStage h = batch_stage(c, c->b_stage_h, dir, n);
            BatchStage dv = batch_stage(c, c->b_stage_d, dir, n);
            std::vector<int> order;  // the active instances (the item lists order steps across them)
            for (int i = 0; i < n; ++i)
                if (active[i]) order.push_back(i);
            const int k = (int)order.size();
            for (int q = 0; q < k; ++q) {
                const int i = order[q];
                const fold3d_grid &g = in[i].grid;
                BatchAdjInst &bi = static_cast<BatchAdjInst *>(h.inst)[q];
                memset(&bi, 0, sizeof bi);
                WaveArgs &a = bi.b.a;
                a.pg = make_geom(g, dir);
                a.nrm = d.nrm;
                a.sg = d.sg;
                orient_tiles(g, d.nrm, a.ntu, a.ntv);
                a.steps = pass_count(a.pg);
                a.first_src = pass_first(a.pg, dir) + d.sg * pass_count(a.pg);  // the forward pass's last target
                a.timeout_ns = 4000000000ull;
                a.flags = c->b_scratch + c->b_flag_off[i];
                a.work = c->b_counters;
                a.status = c->b_counters + 1;
                a.maxd = c->b_slots + i;
                a.dir = dir;
                bi.b.T = in[i].T;
                bi.b.lam = in[i].lambda;
                bi.b.pushed = reinterpret_cast<char *>(c->adj_pushed) + off[i] * esz;
                bi.b.W = in[i].winners;
                bi.b.has = tiles[i].has[dir];
                bi.ep = ellip_param(g, in[i].medium, dir);
            }
            args[dir].inst = static_cast<const BatchAdjInst *>(dv.inst);
            args[dir].items = c->adj_items + item_off[dir];
            args[dir].total = 0;
            args[dir].work = c->b_counters;
            args[dir].status = c->b_counters + 1;
            slots_k[dir] = k;
        }
        cudaError_t ce = cudaMemcpyAsync(c->b_stage_d, c->b_stage_h, 6 * c->b_stage_bytes, cudaMemcpyHostToDevice, s);
        if (ce != cudaSuccess) return cuda_error(ce, "batch staging upload");
        // the item lists, one per launch: counts, exclusive scan (step-major, slot-minor), fill
        for (int dir = 0; dir < 6; ++dir) {
            launches[dir].clear();
            const int k = slots_k[dir];
            if (k == 0) continue;
            int group = k;
            if (kDirs[dir].nrm == 0 && kAdjXGroupBytes > 0) {
                size_t per = 0;  // the largest instance's plane: 4 sectors of 32 bytes per cell
                for (int i = 0; i < n; ++i)
                    if (active[i]) per = std::max(per, (size_t)(in[i].grid.ny + 2) * (in[i].grid.nz + 2) * 128);
                group = (int)std::max<size_t>(1, std::min<size_t>(k, kAdjXGroupBytes / std::max<size_t>(per, 1)));
            }
            unsigned long long *items = const_cast<unsigned long long *>(args[dir].items);
            for (int g0 = 0; g0 < k; g0 += group) {
                const int kg = std::min(group, k - g0);
                BatchAdjArgs ga = args[dir];
                ga.inst = args[dir].inst + g0;
                ga.items = items;
                if ((ce = launch_adj_list(ga.inst, kg, max_steps, c->adj_cnt, nullptr, nullptr, s)) != cudaSuccess ||
                    (ce = cudaMemcpyAsync(cnt.data(), c->adj_cnt, (size_t)max_steps * kg * sizeof(int),
                                          cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                    (ce = cudaStreamSynchronize(s)) != cudaSuccess)
                    return cuda_error(ce, "adjoint item counts");
                offs[0] = 0;
                for (size_t q = 0; q < (size_t)max_steps * kg; ++q) offs[q + 1] = offs[q] + cnt[q];
                if (offs[(size_t)max_steps * kg] >= (1ll << 32))
                    return set_error(FOLD3D_ERR_UNSUPPORTED, "batch too large");
                ga.total = (unsigned)offs[(size_t)max_steps * kg];
                if ((ce = cudaMemcpyAsync(c->adj_off, offs.data(), ((size_t)max_steps * kg + 1) * sizeof(long long),
                                          cudaMemcpyHostToDevice, s)) != cudaSuccess ||
                    (ce = launch_adj_list(ga.inst, kg, max_steps, nullptr, c->adj_off, items, s)) != cudaSuccess ||
                    (ce = cudaStreamSynchronize(s)) != cudaSuccess)  // offs is reused by the next list
                    return cuda_error(ce, "adjoint item lists");
                items += ga.total;
                launches[dir].push_back(ga);
            }
        }
        return FOLD3D_OK;
    };
    if ((rc = stage())) return rc;
    if ((e = cudaEventRecord(c->ev0, s)) != cudaSuccess) return cuda_error(e, "cudaEventRecord");
    int sweep = 0, left = n;
    unsigned hstat[2] = {0, 0};
    while (sweep < max_sweeps && left > 0) {
        if ((e = cudaMemsetAsync(c->b_slots, 0, (size_t)n * 8, s)) != cudaSuccess) return cuda_error(e, "memset");
        for (int dir = 5; dir >= 0; --dir) {  // the forward order reversed
            const unsigned epoch = ++c->epoch;
            for (BatchAdjArgs &ga : launches[dir]) {
                ga.epoch = epoch;  // the groups of a pass share its number (their flags are their own)
                const int grid = (int)std::min<long long>(ga.total, (long long)c->sms * c->batch_adj_bps);
                if ((e = cudaMemsetAsync(c->b_counters, 0, sizeof(unsigned), s)) != cudaSuccess)
                    return cuda_error(e, "memset");
                if (grid > 0 && (e = launch_batch_adj_pass(ga, f32, grid, s)) != cudaSuccess)
                    return cuda_error(e, "batched adjoint pass");
            }
        }
        ++sweep;
        if ((e = cudaMemcpyAsync(slots.data(), c->b_slots, (size_t)n * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(hstat, c->b_counters, sizeof hstat, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_error(e, "batched adjoint sweep");
        if (hstat[1]) return set_error(FOLD3D_ERR_TIMEOUT, "batched adjoint: a dependency wait gave up");
        bool changed = false;
        for (int i = 0; i < n; ++i) {
            if (!active[i]) continue;
            ++sweeps[i];
            memcpy(&delta[i], &slots[i], 8);
            if (sweeps[i] == 1) first[i] = delta[i];
            if (delta[i] <= tol * first[i]) {
                active[i] = 0;
                --left;
                changed = true;
            }
        }
        if (changed && left > 0 && (rc = stage())) return rc;
    }
    for (int i = 0; i < n; ++i) {
        AdjGeom geo;
        memset(&geo, 0, sizeof geo);
        for (int d = 0; d < 6; ++d) {
            geo.pg[d] = make_geom(in[i].grid, d);
            geo.d[d] = ellip_param(in[i].grid, in[i].medium, d).dir;
        }
        if ((e = launch_adj_grad(in[i].T, in[i].lambda, in[i].winners, geo, in[i].medium, in[i].grid, in[i].dLdM,
                                 accumulate,
                                 f32, s)) != cudaSuccess)
            return cuda_error(e, "gradient");
    }
    if ((e = cudaEventRecord(c->ev1, s)) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_error(e, "batched adjoint");
    if (reps) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        for (int i = 0; i < n; ++i) {
            reps[i].sweeps = sweeps[i];
            reps[i].max_delta = delta[i];
            reps[i].elapsed_ms = ms;
            reps[i].nominal_updates = nominal_per_sweep(in[i].grid) * (uint64_t)sweeps[i];
            reps[i].evaluated_updates = 0;
            reps[i].engine = FOLD3D_ENGINE_WAVEFRONT;
        }
    }
    return FOLD3D_OK;
}

// Every array of the medium present; the FP64 parameter medium only with
// float64 fields.
static bool metric_ok(const EllipMedium &m)
{
    const int n = (m.kind == kParamF64) ? 4 : 6;
    for (int k = 0; k < n; ++k)
        if (!m.m[k]) return false;
    return true;
}
static int medium_ok(const EllipMedium &m, bool f32)
{
    if (!metric_ok(m)) return set_error(FOLD3D_ERR_INVALID, "medium array is NULL");
    if (f32 && m.kind == kParamF64)
        return set_error(FOLD3D_ERR_UNSUPPORTED, "the FP64 parameter medium runs with float64 fields");
    return FOLD3D_OK;
}

static int ellip_opts_ok(const fold3d_opts *o)
{
    if (o->max_sweeps < 1) return set_error(FOLD3D_ERR_INVALID, "max_sweeps must be >= 1");
    if (!o->fixed && !(o->tol >= 0.0)) return set_error(FOLD3D_ERR_INVALID, "tol must be >= 0");
    if (o->engine == FOLD3D_ENGINE_PLANES || o->variant != kVariantFast)
        return set_error(FOLD3D_ERR_UNSUPPORTED, "the elliptical medium runs on the wavefront engine, variant 0");
    return FOLD3D_OK;
}

// fold3d_solve_ellip(_record)(_f32): W == NULL for no record.
static int ellip_entry(fold3d_ctx *c, const fold3d_grid *g, const EllipMedium *m, void *T, bool f32,
                       unsigned char *W, bool record, const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    clear_error();
    if (!c) return set_error(FOLD3D_ERR_INVALID, "ctx is NULL");
    if (record && !W) return set_error(FOLD3D_ERR_INVALID, "winner array is NULL");
    if (!T || !o || !m) return set_error(FOLD3D_ERR_INVALID, "NULL argument");
    int rc = medium_ok(*m, f32);
    if (rc) return rc;
    rc = check_grid(g);
    if (rc || (rc = ellip_opts_ok(o))) return rc;
    DeviceGuard dg(c->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    if (record) {
        const cudaError_t e = cudaMemsetAsync(W, 0xff, field_cells(*g), s);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemsetAsync");
    }
    return solve_wavefront(c, *g, nullptr, m, T, f32, *o, s, rep, record ? W : nullptr);
}

static int adjoint_entry(fold3d_ctx *c, int n, const AdjInst *in, bool f32, int max_sweeps, double tol,
                         int accumulate, void *stream, fold3d_report *reps)
{
    clear_error();
    if (!c || !in) return set_error(FOLD3D_ERR_INVALID, "NULL argument");
    if (n < 1) return set_error(FOLD3D_ERR_INVALID, "n must be >= 1");
    if (max_sweeps < 1) return set_error(FOLD3D_ERR_INVALID, "max_sweeps must be >= 1");
    if (!(tol >= 0.0)) return set_error(FOLD3D_ERR_INVALID, "tol must be >= 0");
    for (int i = 0; i < n; ++i) {
        int rc = check_grid(&in[i].grid);
        if (rc) return rc;
        if (!in[i].T || !in[i].winners || !in[i].dLdT || !in[i].lambda || !in[i].dLdM || !metric_ok(in[i].medium))
            return set_error(FOLD3D_ERR_INVALID, n == 1 ? "NULL argument" : "instance with a NULL array");
        if ((rc = medium_ok(in[i].medium, f32))) return rc;
    }
    DeviceGuard dg(c->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    return adjoint_batch(c, n, in, f32, max_sweeps, tol, accumulate, s, reps);
}

static int batch_entry(fold3d_ctx *c, int n, const SolveInst *in, bool f32, const fold3d_opts *o, void *stream,
                       fold3d_report *reps)
{
    clear_error();
    if (!c || !in || !o) return set_error(FOLD3D_ERR_INVALID, "NULL argument");
    if (n < 1) return set_error(FOLD3D_ERR_INVALID, "n must be >= 1");
    for (int i = 0; i < n; ++i) {
        int rc = check_grid(&in[i].grid);
        if (rc) return rc;
        if (!in[i].T || !metric_ok(in[i].medium)) return set_error(FOLD3D_ERR_INVALID, "instance with a NULL array");
        if ((rc = medium_ok(in[i].medium, f32))) return rc;
    }
    int rc = ellip_opts_ok(o);
    if (rc) {
        if (rc == FOLD3D_ERR_UNSUPPORTED)
            return set_error(rc, "batched solves run on the wavefront engine, variant 0");
        return rc;
    }
    DeviceGuard dg(c->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    for (int i = 0; i < n; ++i)
        if (in[i].winners) {
            cudaError_t e = cudaMemsetAsync(in[i].winners, 0xff, field_cells(in[i].grid), s);
            if (e != cudaSuccess) return cuda_error(e, "cudaMemsetAsync");
        }
    return solve_batch(c, n, in, f32, *o, s, reps);
}

extern "C" {

int fold3d_solve_batch(fold3d_ctx *c, int n, const fold3d_instance *in, const fold3d_opts *o, void *stream,
                       fold3d_report *reps)
{
    if (!in || n < 1) return clear_error(), set_error(FOLD3D_ERR_INVALID, in ? "n must be >= 1" : "NULL argument");
    return host_guard([&] {
        std::vector<SolveInst> v(n);
        for (int i = 0; i < n; ++i) v[i] = {in[i].grid, medium_of(in[i].medium), in[i].T, in[i].winners};
        return batch_entry(c, n, v.data(), false, o, stream, reps);
    });
}

int fold3d_solve_batch_f32(fold3d_ctx *c, int n, const fold3d_instance_f32 *in, const fold3d_opts *o, void *stream,
                           fold3d_report *reps)
{
    if (!in || n < 1) return clear_error(), set_error(FOLD3D_ERR_INVALID, in ? "n must be >= 1" : "NULL argument");
    return host_guard([&] {
        std::vector<SolveInst> v(n);
        for (int i = 0; i < n; ++i) v[i] = {in[i].grid, medium_of(in[i].medium), in[i].T, in[i].winners};
        return batch_entry(c, n, v.data(), true, o, stream, reps);
    });
}

int fold3d_init_implicit_device(fold3d_ctx *c, const fold3d_grid *g, const fold3d_medium *m, double *T,
                                void *stream)
{
    clear_error();
    if (!c || !g || !m || !T) return set_error(FOLD3D_ERR_INVALID, "NULL argument");
    int rc = check_grid(g);
    if (rc) return rc;
    if (g->nx < 2 || g->ny < 2 || g->nz < 2) return set_error(FOLD3D_ERR_INVALID, "grid needs >= 2 points per axis");
    DeviceGuard dg(c->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    const size_t cells = field_cells(*g), plane = (size_t)(g->nx + 2) * (g->ny + 2) * sizeof(double);
    if (c->i_if_cells < cells) {
        if (c->i_if) cudaFree(c->i_if);
        c->i_if = nullptr;
        c->i_if_cells = 0;
        if (cudaMalloc(&c->i_if, cells * sizeof(double)) != cudaSuccess)
            return set_error(FOLD3D_ERR_NOMEM, "device initialiser scratch");
        c->i_if_cells = cells;
    }
    // two slabs of about 256 MB of node planes (at least one plane, at most the field)
    const size_t bytes = std::min(std::max((size_t)256 << 20, plane) / plane * plane, cells * sizeof(double));
    if (c->i_stage_bytes < bytes) {
        for (int b = 0; b < 2; ++b) {
            if (c->i_stage[b]) cudaFreeHost(c->i_stage[b]);
            c->i_stage[b] = nullptr;
        }
        c->i_stage_bytes = 0;
        for (int b = 0; b < 2; ++b)
            if (cudaMallocHost(&c->i_stage[b], bytes) != cudaSuccess)
                return set_error(FOLD3D_ERR_NOMEM, "device initialiser staging");
        c->i_stage_bytes = bytes;
    }
    return host_guard([&] { return init_implicit_device(*g, *m, T, c->i_if, c->i_stage, c->i_stage_bytes / plane, s); });
}

int fold3d_adjoint_batch(fold3d_ctx *c, int n, const fold3d_adjoint_instance *in, int max_sweeps, double tol,
                         int accumulate, void *stream, fold3d_report *reps)
{
    if (!in || n < 1) return clear_error(), set_error(FOLD3D_ERR_INVALID, in ? "n must be >= 1" : "NULL argument");
    return host_guard([&] {
        std::vector<AdjInst> v(n);
        for (int i = 0; i < n; ++i)
            v[i] = {in[i].grid, medium_of(in[i].medium), in[i].T, in[i].winners, in[i].dLdT, in[i].lambda,
                    in[i].dLdM};
        return adjoint_entry(c, n, v.data(), false, max_sweeps, tol, accumulate, stream, reps);
    });
}

int fold3d_adjoint_batch_f32(fold3d_ctx *c, int n, const fold3d_adjoint_instance_f32 *in, int max_sweeps,
                             double tol, int accumulate, void *stream, fold3d_report *reps)
{
    if (!in || n < 1) return clear_error(), set_error(FOLD3D_ERR_INVALID, in ? "n must be >= 1" : "NULL argument");
    return host_guard([&] {
        std::vector<AdjInst> v(n);
        for (int i = 0; i < n; ++i)
            v[i] = {in[i].grid, medium_of(in[i].medium), in[i].T, in[i].winners, in[i].dLdT, in[i].lambda,
                    in[i].dLdM};
        return adjoint_entry(c, n, v.data(), true, max_sweeps, tol, accumulate, stream, reps);
    });
}

int fold3d_solve(fold3d_ctx *c, const fold3d_grid *g, const fold3d_medium *m, double *T,
                 const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    clear_error();
    if (!c) return set_error(FOLD3D_ERR_INVALID, "ctx is NULL");
    if (!T) return set_error(FOLD3D_ERR_INVALID, "field is NULL");
    if (!o) return set_error(FOLD3D_ERR_INVALID, "opts is NULL");
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_medium(m))) return rc;
    if (o->max_sweeps < 1) return set_error(FOLD3D_ERR_INVALID, "max_sweeps must be >= 1");
    if (o->engine < 0 || o->engine > FOLD3D_ENGINE_WAVEFRONT)
        return set_error(FOLD3D_ERR_INVALID, "unknown engine");
    if (!o->fixed && !(o->tol >= 0.0)) return set_error(FOLD3D_ERR_INVALID, "tol must be >= 0");
    if (o->variant != kVariantFast && o->variant != kVariantLiteral && o->variant != kVariantCompact)
        return set_error(FOLD3D_ERR_INVALID, "unknown solver variant");
    DeviceGuard dg(c->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    // AUTO: the wavefront engine for the default solver form, the per-plane
    // engine for the cross-check forms.
    const int engine = (o->engine == FOLD3D_ENGINE_AUTO)
                           ? (o->variant == kVariantFast ? FOLD3D_ENGINE_WAVEFRONT : FOLD3D_ENGINE_PLANES)
                           : o->engine;
    if (engine == FOLD3D_ENGINE_WAVEFRONT) {
        if (o->variant != kVariantFast)
            return set_error(FOLD3D_ERR_UNSUPPORTED, "the wavefront engine runs the default solver variant only");
        return solve_wavefront(c, *g, m, nullptr, T, false, *o, s, rep);
    }
    return solve_planes(c, *g, *m, T, *o, s, rep);
}

int fold3d_selftest_wait_timeout(fold3d_ctx *c, double timeout_ms)
{
    clear_error();
    if (!c) return set_error(FOLD3D_ERR_INVALID, "ctx is NULL");
    if (!(timeout_ms > 0 && timeout_ms < 1000)) return set_error(FOLD3D_ERR_INVALID, "timeout_ms in (0, 1000)");
    DeviceGuard dg(c->device);
    const fold3d_grid g = {16, 16, 16, 1.0, 1.0, 1.0};
    const fold3d_medium m = {1.1, -0.35, 0.4, 0.7};
    int rc = wave_scratch(c, g);
    if (rc) return rc;
    cudaError_t e;
    const size_t cells = field_cells(g);
    if (c->d_field_cells < cells) {
        if (c->d_field) cudaFree(c->d_field);
        c->d_field = nullptr;
        c->d_field_cells = 0;
        c->key_T = nullptr;
        if ((e = cudaMalloc(&c->d_field, cells * sizeof(double))) != cudaSuccess)
            return set_error(FOLD3D_ERR_NOMEM, "cudaMalloc");
        c->d_field_cells = cells;
    }
    cudaStream_t s = c->stream;
    WaveArgs a;
    memset(&a, 0, sizeof a);
    for (int b = 0; b < 3; ++b) {
        int ntu, ntv;
        orient_tiles(g, b, ntu, ntv);
        a.mod[b] = c->w_mod[b];
        a.mod_ntu[b] = ntu;
        a.mod_ntiles[b] = ntu * ntv;
    }
    a.flags = c->w_flags;
    a.work = c->w_counters;
    a.status = c->w_counters + 1;
    a.maxd = c->d_maxd;
    a.evaluated = c->w_evaluated;
    a.timeout_ns = (unsigned long long)(timeout_ms * 1e6);
    a.skip_from = 0xffffffffu;
    a.pg = make_geom(g, FOLD3D_K_UP);
    a.nrm = 2;
    a.ua = 0;
    a.va = 1;
    a.sg = 1;
    orient_tiles(g, 2, a.ntu, a.ntv);
    a.steps = pass_count(a.pg);
    a.first_src = 1;
    a.epoch = ++c->epoch;
    DirTable tab;
    build_dir_table(make_frame(g, m, FOLD3D_K_UP), tab);
    // start the item counter after step 0: step 1 then waits for flags nothing sets
    const unsigned start[2] = {(unsigned)(a.ntu * a.ntv), 0u};
    unsigned hstat[2] = {0, 0};
    if ((e = cudaMemcpyAsync(c->w_counters, start, sizeof start, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = launch_wave_pass(c->d_field, a, tab, 4, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hstat, c->w_counters, sizeof hstat, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_error(e, "selftest");
    if (hstat[1] == 1) return set_error(FOLD3D_ERR_TIMEOUT, "wavefront: a dependency wait gave up (as intended)");
    return set_error(FOLD3D_ERR_CUDA, "selftest: the waits did not give up");
}

void fold3d_ellip_metric(double vz, double eps, double ax, double ay, double az, float out[6])
{
    if (!out) return;
    const double nn = std::sqrt(ax * ax + ay * ay + az * az);
    const double nx = ax / nn, ny = ay / nn, nz = az / nn;
    const double a = 1.0 / (vz * vz * (1.0 + 2.0 * eps));
    const double b = 1.0 / (vz * vz) - a;
    const double m[6] = {a + b * nx * nx, b * nx * ny, b * nx * nz, a + b * ny * ny, b * ny * nz, a + b * nz * nz};
    for (int k = 0; k < 6; ++k) out[k] = (float)m[k];
}

int fold3d_solve_ellip(fold3d_ctx *c, const fold3d_grid *g, const fold3d_ellip *m, double *T, const fold3d_opts *o,
                       void *stream, fold3d_report *rep)
{
    if (!m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const EllipMedium em = medium_of(*m);
    return ellip_entry(c, g, &em, T, false, nullptr, false, o, stream, rep);
}

int fold3d_solve_ellip_f32(fold3d_ctx *c, const fold3d_grid *g, const fold3d_ellip *m, float *T,
                           const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    if (!m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const EllipMedium em = medium_of(*m);
    return ellip_entry(c, g, &em, T, true, nullptr, false, o, stream, rep);
}

int fold3d_solve_ellip_record(fold3d_ctx *c, const fold3d_grid *g, const fold3d_ellip *m, double *T,
                              unsigned char *W, const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    if (!m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const EllipMedium em = medium_of(*m);
    return ellip_entry(c, g, &em, T, false, W, true, o, stream, rep);
}

int fold3d_solve_ellip_record_f32(fold3d_ctx *c, const fold3d_grid *g, const fold3d_ellip *m, float *T,
                                  unsigned char *W, const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    if (!m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const EllipMedium em = medium_of(*m);
    return ellip_entry(c, g, &em, T, true, W, true, o, stream, rep);
}

int fold3d_adjoint_ellip(fold3d_ctx *c, const fold3d_grid *g, const fold3d_ellip *m, const double *T,
                         const unsigned char *W, const double *dLdT, double *lam, double *dLdM, int max_sweeps,
                         double tol, void *stream, fold3d_report *rep)
{
    if (!g || !m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const AdjInst one = {*g, medium_of(*m), T, W, dLdT, lam, dLdM};
    return adjoint_entry(c, 1, &one, false, max_sweeps, tol, 0, stream, rep);
}

int fold3d_adjoint_ellip_f32(fold3d_ctx *c, const fold3d_grid *g, const fold3d_ellip *m, const float *T,
                             const unsigned char *W, const float *dLdT, float *lam, float *dLdM, int max_sweeps,
                             double tol, void *stream, fold3d_report *rep)
{
    if (!g || !m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const AdjInst one = {*g, medium_of(*m), T, W, dLdT, lam, dLdM};
    return adjoint_entry(c, 1, &one, true, max_sweeps, tol, 0, stream, rep);
}

int fold3d_batch_set_config(fold3d_ctx *c, int tile_rows, int ctas_per_sm)
{
    clear_error();
    if (!c) return set_error(FOLD3D_ERR_INVALID, "ctx is NULL");
    if (tile_rows != 0 && tile_rows != 2 && tile_rows != 4 && tile_rows != 8)
        return set_error(FOLD3D_ERR_INVALID, "tile_rows must be 0 (autotune), 2, 4 or 8");
    if (ctas_per_sm < 0) return set_error(FOLD3D_ERR_INVALID, "ctas_per_sm must be >= 0");
    c->tune_tv = tile_rows;
    c->tune_bps = tile_rows ? ctas_per_sm : 0;
    return FOLD3D_OK;
}

int fold3d_batch_get_config(fold3d_ctx *c, int *tile_rows, int *ctas_per_sm)
{
    clear_error();
    if (!c || !tile_rows || !ctas_per_sm) return set_error(FOLD3D_ERR_INVALID, "NULL argument");
    *tile_rows = c->last_tv;
    *ctas_per_sm = c->last_bps;
    return FOLD3D_OK;
}

int fold3d_solve_tti(fold3d_ctx *c, const fold3d_grid *g, const fold3d_tti *m, double *T, const fold3d_opts *o,
                     void *stream, fold3d_report *rep)
{
    if (!m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const EllipMedium em = medium_of(*m);
    return ellip_entry(c, g, &em, T, false, nullptr, false, o, stream, rep);
}

int fold3d_solve_tti_record(fold3d_ctx *c, const fold3d_grid *g, const fold3d_tti *m, double *T, unsigned char *W,
                            const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    if (!m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const EllipMedium em = medium_of(*m);
    return ellip_entry(c, g, &em, T, false, W, true, o, stream, rep);
}

int fold3d_adjoint_tti(fold3d_ctx *c, const fold3d_grid *g, const fold3d_tti *m, const double *T,
                       const unsigned char *W, const double *dLdT, double *lam, double *dLdP, int max_sweeps,
                       double tol, void *stream, fold3d_report *rep)
{
    if (!g || !m) return clear_error(), set_error(FOLD3D_ERR_INVALID, "NULL argument");
    const AdjInst one = {*g, medium_of(*m), T, W, dLdT, lam, dLdP};
    return adjoint_entry(c, 1, &one, false, max_sweeps, tol, 0, stream, rep);
}

int fold3d_solve_batch_tti(fold3d_ctx *c, int n, const fold3d_tti_instance *in, const fold3d_opts *o, void *stream,
                           fold3d_report *reps)
{
    if (!in || n < 1) return clear_error(), set_error(FOLD3D_ERR_INVALID, in ? "n must be >= 1" : "NULL argument");
    return host_guard([&] {
        std::vector<SolveInst> v(n);
        for (int i = 0; i < n; ++i) v[i] = {in[i].grid, medium_of(in[i].medium), in[i].T, in[i].winners};
        return batch_entry(c, n, v.data(), false, o, stream, reps);
    });
}

int fold3d_adjoint_batch_tti(fold3d_ctx *c, int n, const fold3d_tti_adjoint_instance *in, int max_sweeps, double tol,
                             int accumulate, void *stream, fold3d_report *reps)
{
    if (!in || n < 1) return clear_error(), set_error(FOLD3D_ERR_INVALID, in ? "n must be >= 1" : "NULL argument");
    return host_guard([&] {
        std::vector<AdjInst> v(n);
        for (int i = 0; i < n; ++i)
            v[i] = {in[i].grid, medium_of(in[i].medium), in[i].T, in[i].winners, in[i].dLdT, in[i].lambda,
                    in[i].dLdP};
        return adjoint_entry(c, n, v.data(), false, max_sweeps, tol, accumulate, stream, reps);
    });
}

int fold3d_solve_host(fold3d_ctx *c, const fold3d_grid *g, const fold3d_medium *m, const double *T_in,
                      double *T_out, const fold3d_opts *o, void *stream, fold3d_report *rep)
{
    clear_error();
    if (!c) return set_error(FOLD3D_ERR_INVALID, "ctx is NULL");
    if (!T_in || !T_out) return set_error(FOLD3D_ERR_INVALID, "field is NULL");
    int rc = check_grid(g);
    if (rc) return rc;
    DeviceGuard dg(c->device);
    const size_t cells = field_cells(*g);
    cudaError_t e;
    if (c->d_field_cells < cells) {
        if (c->d_field) cudaFree(c->d_field);
        c->d_field = nullptr;
        c->d_field_cells = 0;
        if (c->sweep_exec && c->key_T) c->key_T = nullptr;  // force a re-capture
        if ((e = cudaMalloc(&c->d_field, cells * sizeof(double))) != cudaSuccess)
            return set_errorf(FOLD3D_ERR_NOMEM, "cudaMalloc: %s", cudaGetErrorString(e));
        c->d_field_cells = cells;
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    if ((e = cudaMemcpyAsync(c->d_field, T_in, cells * sizeof(double), cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
        return cuda_error(e, "host-to-device copy");
    rc = fold3d_solve(c, g, m, c->d_field, o, s, rep);
    if (rc) return rc;
    if ((e = cudaMemcpyAsync(T_out, c->d_field, cells * sizeof(double), cudaMemcpyDeviceToHost, s)) !=
        cudaSuccess)
        return cuda_error(e, "device-to-host copy");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "device-to-host copy");
    return FOLD3D_OK;
}

int fold3d_plane(const fold3d_grid *g, const fold3d_medium *m, double *T, int dir, int src, void *stream)
{
    clear_error();
    int rc = check_grid(g);
    if (rc) return rc;
    if ((rc = check_medium(m))) return rc;
    if (!T) return set_error(FOLD3D_ERR_INVALID, "field is NULL");
    if (dir < 0 || dir > 5) return set_error(FOLD3D_ERR_INVALID, "dir must be 0..5");
    const PlaneGeom pg = make_geom(*g, dir);
    const int tgt = src + kDirs[dir].sg;
    if (src < 1 || src > pg.nplanes || tgt < 1 || tgt > pg.nplanes)
        return set_error(FOLD3D_ERR_INVALID, "plane index out of range");
    const LocalFrameH L = make_frame(*g, *m, dir);
    DirTable tab;
    build_dir_table(L, tab);
    cudaError_t e = launch_plane(T, pg, L, &tab, kVariantFast, src, nullptr, (cudaStream_t)stream);
    return e == cudaSuccess ? FOLD3D_OK : cuda_error(e, "plane launch");
}

}  // extern "C"

// ------------------------------------------------------------------------
// Reference-compatible sweep entry points and OpenACC runtime subset
// ------------------------------------------------------------------------
namespace {
std::mutex g_compat_mu;
std::map<uintptr_t, size_t> g_acc_allocs;  // base -> bytes, from acc_malloc
int g_compat_n[3] = {0, 0, 0};

// Grid of a compat call: the size set by fold3d_compat_set_grid, else the
// cube whose field fills the acc_malloc allocation that starts at T.  When T
// lies inside an acc_malloc allocation, the field must also fit between T
// and the allocation's end.  NULL, or the reason the call is rejected.
const char *compat_grid(const double *T, fold3d_grid &g)
{
    std::lock_guard<std::mutex> lk(g_compat_mu);
    // the acc_malloc allocation T points into, if any
    auto it = g_acc_allocs.upper_bound((uintptr_t)T);
    bool inside = false;
    if (it != g_acc_allocs.begin()) {
        --it;
        inside = (uintptr_t)T < it->first + it->second;
    }
    if (g_compat_n[0] > 0) {
        g.nx = g_compat_n[0];
        g.ny = g_compat_n[1];
        g.nz = g_compat_n[2];
        if (inside) {
            const double need = ((double)g.nx + 2) * ((double)g.ny + 2) * ((double)g.nz + 2) * sizeof(double);
            if (need > (double)(it->first + it->second - (uintptr_t)T))
                return "function_*: the field of the grid set by fold3d_compat_set_grid does not fit in the "
                       "acc_malloc allocation from T on";
        }
    } else {
        if (!inside)
            return "function_*: grid size unknown (call fold3d_compat_set_grid or allocate with acc_malloc)";
        if ((uintptr_t)T != it->first)
            return "function_*: T points inside an acc_malloc allocation, not at its start; call "
                   "fold3d_compat_set_grid to give the grid size";
        const size_t cells = it->second / sizeof(double);
        long long p = (long long)std::llround(std::cbrt((double)cells));
        while (p * p * p > (long long)cells) --p;
        while ((p + 1) * (p + 1) * (p + 1) <= (long long)cells) ++p;
        if (p * p * p != (long long)cells || p < 4)
            return "function_*: the acc_malloc allocation at T is not a cubic field; call fold3d_compat_set_grid";
        g.nx = g.ny = g.nz = (int)(p - 2);
    }
    g.dx = g.dy = g.dz = 1.0;  // geometry only; spacings come from the call
    return nullptr;
}

void compat_plane_body(int dir, double *T, int src, double dzz, double dxx, double dyy, double dxy, double dxz,
                       double dyz, double F, double ay, double ax, double az)
{
    fold3d_grid g;
    const char *why = T ? compat_grid(T, g) : "function_*: T is NULL";
    if (why) {
        set_error(FOLD3D_ERR_INVALID, why);
        return;
    }
    const PlaneGeom pg = make_geom(g, dir);
    const int tgt = src + kDirs[dir].sg;
    if (src < 1 || src > pg.nplanes || tgt < 1 || tgt > pg.nplanes) {
        set_error(FOLD3D_ERR_INVALID, "function_*: plane index out of range");
        return;
    }
    // The caller's arguments are already in the direction's local frame
    // (the reference driver permutes them, AN_ISO_1_OpenACC.c:1198-1235).
    const LocalFrameH L = {F, ax, ay, az, dzz, dxx, dyy, dxy, dxz, dyz};
    DirTable tab;
    build_dir_table(L, tab);
    cudaError_t e = launch_plane(T, pg, L, &tab, kVariantFast, src, nullptr, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) cuda_error(e, "function_*");
}

int g_host_n[3] = {0, 0, 0};  // grid of the last ImplicitInitialiser call
}  // namespace

void fold3d::compat_note_host_grid(int nx, int ny, int nz)
{
    host_guard([&] {
        std::lock_guard<std::mutex> lk(g_compat_mu);
        g_host_n[0] = nx;
        g_host_n[1] = ny;
        g_host_n[2] = nz;
        return FOLD3D_OK;
    });
}

bool fold3d::compat_host_pitch(long long &sy, long long &sz)
{
    int n[3] = {0, 0, 0};
    const int rc = host_guard([&] {
        std::lock_guard<std::mutex> lk(g_compat_mu);
        const int *src = (g_compat_n[0] > 0) ? g_compat_n : g_host_n;
        n[0] = src[0];
        n[1] = src[1];
        n[2] = src[2];
        return FOLD3D_OK;
    });
    if (rc) return false;
    if (n[0] < 2 || n[1] < 2) {
        set_error(FOLD3D_ERR_INVALID, "InitNode/updateVoxel: grid size unknown (call fold3d_compat_set_grid or "
                                      "ImplicitInitialiser first)");
        return false;
    }
    clear_error();
    sy = (long long)n[0] + 2;
    sz = sy * ((long long)n[1] + 2);
    return true;
}

namespace {
// The reference's sweep functions return nothing; errors are left in
// fold3d_last_error, and no host exception leaves the library.
void compat_plane(int dir, double *T, int src, double dzz, double dxx, double dyy, double dxy, double dxz,
                  double dyz, double F, double ay, double ax, double az)
{
    clear_error();
    host_guard([&] {
        compat_plane_body(dir, T, src, dzz, dxx, dyy, dxy, dxz, dyz, F, ay, ax, az);
        return FOLD3D_OK;
    });
}
}  // namespace

extern "C" {

int fold3d_compat_set_grid(int nx, int ny, int nz)
{
    clear_error();
    if ((nx | ny | nz) != 0 && (nx < 2 || ny < 2 || nz < 2))
        return set_error(FOLD3D_ERR_INVALID, "grid sizes must be >= 2 (or all 0 to unset)");
    return host_guard([&] {
        std::lock_guard<std::mutex> lk(g_compat_mu);
        g_compat_n[0] = nx;
        g_compat_n[1] = ny;
        g_compat_n[2] = nz;
        return FOLD3D_OK;
    });
}

void fold3d_compat_plane(int dir, double *T, int p, double dzz, double dxx, double dyy, double dxy, double dxz,
                         double dyz, double F, double ay, double ax, double az)
{
    if (dir < 0 || dir > 5) {
        set_error(FOLD3D_ERR_INVALID, "fold3d_compat_plane: dir must be 0..5");
        return;
    }
    compat_plane(dir, T, p, dzz, dxx, dyy, dxy, dxz, dyz, F, ay, ax, az);
}

#define FOLD3D_COMPAT(name, dir)                                                                    \
    void name(double *T, int p, double dzz, double dxx, double dyy, double dxy, double dxz, double dyz, \
              double F, double ay, double ax, double az)                                            \
    {                                                                                               \
        compat_plane(dir, T, p, dzz, dxx, dyy, dxy, dxz, dyz, F, ay, ax, az);                       \
    }
FOLD3D_COMPAT(function_x_down, FOLD3D_X_DOWN)
FOLD3D_COMPAT(function_x_up, FOLD3D_X_UP)
FOLD3D_COMPAT(function_k_up, FOLD3D_K_UP)
FOLD3D_COMPAT(function_k_down, FOLD3D_K_DOWN)
FOLD3D_COMPAT(function_y_up, FOLD3D_Y_UP)
FOLD3D_COMPAT(function_y_down, FOLD3D_Y_DOWN)
#undef FOLD3D_COMPAT

// The OpenACC runtime calls of the reference driver (AN_ISO_1_OpenACC.c:
// 1184-1186, 1241), over the CUDA runtime.  acc_malloc also records the
// allocation so the sweep entry points can recover the grid size.
void *acc_malloc(size_t bytes)
{
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        set_error(FOLD3D_ERR_NOMEM, "acc_malloc: cudaMalloc failed");
        return nullptr;
    }
    try {
        std::lock_guard<std::mutex> lk(g_compat_mu);
        g_acc_allocs[(uintptr_t)p] = bytes;
    } catch (...) {  // no host memory for the record: give the device block back
        cudaFree(p);
        set_error(FOLD3D_ERR_NOMEM, "acc_malloc: out of host memory");
        return nullptr;
    }
    return p;
}

void acc_free(void *p)
{
    if (!p) return;
    host_guard([&] {
        std::lock_guard<std::mutex> lk(g_compat_mu);
        g_acc_allocs.erase((uintptr_t)p);
        return FOLD3D_OK;
    });
    cudaFree(p);
}

void acc_memcpy_to_device(void *dst, void *src, size_t bytes)
{
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) cuda_error(e, "acc_memcpy_to_device");
}

void acc_memcpy_from_device(void *dst, void *src, size_t bytes)
{
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) cuda_error(e, "acc_memcpy_from_device");
}

}  // extern "C"
