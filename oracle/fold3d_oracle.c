/*
 * fold3d_oracle.c -- CPU oracle for the Fold3dPMM plane sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg use it, to check results or to time the CPU path.
 *
 * It is a plain-C restatement of the reference's single-device path
 * (ezhilmathik/FGCS-OpenACC-Advanced, Stencil-OpenACC/AN_ISO_1_OpenACC.c and
 * Stencil-OpenACC/Fold3dPMM.c) with three generalisations that do not change
 * the arithmetic of any cubic reference case:
 *   - grid sizes are run-time values and the three axes may differ
 *     (the reference fixes _nx=_ny=_nz and one pitch HEIGHT, Fold3dPMM.h:27-30);
 *   - the medium (F, ax, ay, az) is a run-time value (the reference hard-codes
 *     _Fc, _axx, _ayy, _azz, Fold3dPMM.h:49-52, AN_ISO_1_OpenACC.c:50-53);
 *   - the six copy-pasted sweep functions are one table-driven routine.
 *
 * Parity: pinned.  tests/golden/ holds outputs of the reference's own code
 * (compiled from its sources by oracle/build.py into oracle/_ref/) and the
 * tests check this file against them bit for bit.
 *
 * Every floating-point expression keeps the reference's operand order; the
 * file must be compiled with -ffp-contract=off (no FMA contraction), as the
 * reference's host build is.
 *
 * Array layout (AN_ISO_1_OpenACC.c:195, Fold3dPMM.c:143): T[i + Px*(j + Py*k)]
 * with Px = nx+2, Py = ny+2, one ghost layer on every face; interior indices
 * run 1..n per axis.  Axis 0 = i (spacing dx), 1 = j (dy), 2 = k (dz).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXT (10e15 * 1.0) /* Fold3dPMM.h:6 */

/* The reference overrides fmin with a ternary macro (AN_ISO_1_OpenACC.c:32-34). */
static inline double omin(double a, double b) { return (a < b) ? a : b; }
/* sign(a) maps 0 to -1 (AN_ISO_1_OpenACC.c:36-38). */
static inline double osign(double a) { return (a > 0) ? 1.0 : -1.0; }

/* ------------------------------------------------------------------------ */
/* Local solvers                                                             */
/* ------------------------------------------------------------------------ */

/* Edge (two-point) candidate from segment s0-s1 of the previous plane.
 * Follows FoldEdge2Points, AN_ISO_1_OpenACC.c:59-114 (OPTTEST off). */
static void orc_edge(double *tn, double s0, double s1, double F, double ax,
                     double ay, double az, double hx, double hz)
{
    if (*tn < omin(s1, s0) || (ax > 0.0 && s1 > s0))
        return;
    double g = F * F - ay * ay;
    double d = (s1 - s0) / hx;
    double c = (1.0 - d * ax);
    double q = g * (c * c - d * d * (g - az * az));
    if (0.0 < q) {
        c = (-az * c + sqrt(q)) / (g - az * az);
        q = s0 + hz * c;
        if (q < *tn && q > omin(s0, s1)) {
            g = sqrt((d * d + c * c) * F * F / g);
            /* :90 computes a first footpoint that :92 overwrites; dead. */
            double xe = -hz * (d + ax * g) / (c + az * g);
            if (0.0 < xe && xe < hx)
                *tn = q;
        }
    }
    if (*tn > s1) { /* fall-back from s1 alone, :99-113 */
        c = (-hx * ax + hz * az);
        g = hx * hx + hz * hz;
        q = (F * F - ax * ax - ay * ay - az * az) * g + c * c;
        if (q > 0.0) {
            c = c + sqrt(q);
            if (c > 0.0)
                *tn = omin(*tn, s1 + g / c);
        }
    }
}

/* Triangle (three-point) candidate from s0-s1-s2, then the nested edge on
 * s1-s2 with a rotated drift.  Follows FoldSurf3Points,
 * AN_ISO_1_OpenACC.c:119-175 (UNROLLED on, OPTTEST off). */
static void orc_surf(double *tn, double s0, double s1, double s2, double F,
                     double ax, double ay, double az, double hx, double hy,
                     double hz, double hxz)
{
    if (*tn < omin(s0, omin(s1, s2)) || (ax > 0.0 && s1 > s0) ||
        (ay > 0.0 && s2 > s1))
        return;
    double dx = (s1 - s0) / hx;
    double dy = (s2 - s1) / hy;
    double dd = dx * dx + dy * dy;
    double g = F * F - az * az;
    double al = 1.0 - ax * dx - ay * dy;
    double q = al * al - dd * g;
    if (q > 0.0) {
        al = (-az * al + F * sqrt(q)) / g;
        g = s0 + hz * al;
        if (g < *tn && g > omin(omin(s0, s1), s2)) {
            q = sqrt(dd + al * al);
            dd = -hz / (F * al + az * q);
            double xe = dd * (F * dx + ax * q);
            double ye = dd * (F * dy + ay * q);
            if (0.0 <= omin(xe, ye) && ye * hx <= xe * hy && xe <= hx)
                *tn = g;
        }
    }
    if (*tn > omin(s1, s2) && (!(ax * hz + az * hx > 0.0 && s1 > s2)))
        orc_edge(tn, s1, s2, F, ay, (ax * hz + az * hx) / hxz,
                 (-ax * hx + az * hz) / hxz, hy, hxz);
}

/* ------------------------------------------------------------------------ */
/* Sweep directions                                                          */
/* ------------------------------------------------------------------------ */

/* One row per reference sweep function, in the driver's order
 * (AN_ISO_1_OpenACC.c:1195-1236): x_down, x_up, k_up, k_down, y_up, y_down.
 *   nrm  : axis normal to the planes; sg: +1 if the target is src+1
 *   xa,xs: axis and sign of the local "x" neighbour (xt)
 *   ya,ys: axis and sign of the local "y" neighbour (yt)
 * The neighbour offsets of every function (e.g. :195-204 for x_down) are
 * xt=+x, yt=+y, xnt=-x, ynt=-y, txy=+x+y, txm=+x-y, tym=-x+y, txnyn=-x-y in
 * that local frame, and the local drift is (xs*a[xa], ys*a[ya], sg*a[nrm])
 * (:206, :359, :816, :971, :511, :663). */
typedef struct { int nrm, sg, xa, xs, ya, ys; } orc_dir;
static const orc_dir ORC_DIRS[6] = {
    {0, +1, 2, +1, 1, +1}, /* function_x_down :180 */
    {0, -1, 2, -1, 1, -1}, /* function_x_up   :334 */
    {2, +1, 1, +1, 0, +1}, /* function_k_up   :790 */
    {2, -1, 1, -1, 0, -1}, /* function_k_down :944 */
    {1, -1, 0, -1, 2, -1}, /* function_y_up   :485 */
    {1, +1, 0, +1, 2, +1}, /* function_y_down :636 */
};

typedef struct {
    int n[3];
    int64_t stride[3];
} orc_grid;

static orc_grid orc_make_grid(int nx, int ny, int nz)
{
    orc_grid g;
    g.n[0] = nx; g.n[1] = ny; g.n[2] = nz;
    g.stride[0] = 1;
    g.stride[1] = (int64_t)(nx + 2);
    g.stride[2] = (int64_t)(nx + 2) * (ny + 2);
    return g;
}

/* Update of one target point from the source plane; body of every
 * function_* (e.g. :195-326).  Returns nothing; writes T[tgt]. */
static void orc_point(double *T, int64_t tgt, int64_t src, int64_t sx,
                      int64_t sy, double F, double ax, double ay, double az,
                      double hz, double hx, double hy, double hxy, double hxz,
                      double hyz)
{
    double tnew = fabs(T[tgt]);
    double st = fabs(T[src]);
    double xt = fabs(T[src + sx]);
    double yt = fabs(T[src + sy]);
    double xnt = fabs(T[src - sx]);
    double ynt = fabs(T[src - sy]);
    double txm = fabs(T[src + sx - sy]);
    double txy = fabs(T[src + sx + sy]);
    double tym = fabs(T[src - sx + sy]);
    double txnyn = fabs(T[src - sx - sy]);

    if (T[tgt] < 0) { /* negative side: drift reversed, :207-212 */
        ax *= -1;
        ay *= -1;
        az *= -1;
    }
    if (st < tnew) { /* one-dimensional normal candidate, :214-228 */
        double q = (F * F - (ax * ax + ay * ay)) * hz * hz;
        if (q > 0.0) {
            q = az * hz + sqrt(q);
            if (q > 0.0)
                tnew = omin(tnew, st + hz * hz / q);
        }
    }
    /* early exit and the fixed 16-call order, :231-253 */
    if (!(tnew < st && tnew < omin(xt, yt) && tnew < omin(txy, txm) &&
          tnew < omin(txnyn, tym))) {
        orc_surf(&tnew, st, xt, txy, F, ax, ay, az, hx, hy, hz, hxz);
        orc_surf(&tnew, st, xt, txm, F, ax, -ay, az, hx, hy, hz, hxz);
        orc_surf(&tnew, st, xnt, txnyn, F, -ax, -ay, az, hx, hy, hz, hxz);
        orc_surf(&tnew, st, xnt, tym, F, -ax, ay, az, hx, hy, hz, hxz);
        orc_surf(&tnew, st, ynt, txnyn, F, -ay, -ax, az, hy, hx, hz, hyz);
        orc_surf(&tnew, st, ynt, txm, F, -ay, ax, az, hy, hx, hz, hyz);
        orc_surf(&tnew, st, yt, txy, F, ay, ax, az, hy, hx, hz, hyz);
        orc_surf(&tnew, st, yt, tym, F, ay, -ax, az, hy, hx, hz, hyz);

        orc_edge(&tnew, st, xt, F, ax, ay, az, hx, hz);
        orc_edge(&tnew, st, txy, F, (ax * hx + ay * hy) / hxy,
                 (-ax * hy + ay * hx) / hxy, az, hxy, hz);
        orc_edge(&tnew, st, yt, F, ay, ax, az, hy, hz);
        orc_edge(&tnew, st, tym, F, -(ax * hx - ay * hy) / hxy,
                 (ax * hy + ay * hx) / hxy, az, hxy, hz);
        orc_edge(&tnew, st, xnt, F, -ax, ay, az, hx, hz);
        orc_edge(&tnew, st, txnyn, F, -(ax * hx + ay * hy) / hxy,
                 (-ax * hy + ay * hx) / hxy, az, hxy, hz);
        orc_edge(&tnew, st, ynt, F, -ay, ax, az, hy, hz);
        orc_edge(&tnew, st, txm, F, (ax * hx - ay * hy) / hxy,
                 (ax * hy + ay * hx) / hxy, az, hxy, hz);
    }
    T[tgt] = (osign(T[tgt]) * 1.0) * tnew; /* :326 */
}

/* One plane step: update plane (src + sg) from plane src in direction dir.
 * Equivalent to one call of the matching function_* with the driver's
 * argument permutation (:1198, :1205, :1212, :1219, :1227, :1234). */
void orc_plane(double *T, int nx, int ny, int nz, double dx, double dy,
               double dz, double F, double a0, double a1, double a2, int dir,
               int src)
{
    const orc_grid g = orc_make_grid(nx, ny, nz);
    const orc_dir d = ORC_DIRS[dir];
    const double h[3] = {dx, dy, dz};
    const double a[3] = {a0, a1, a2};
    const double hz = h[d.nrm], hx = h[d.xa], hy = h[d.ya];
    const double hxy = sqrt(hx * hx + hy * hy);
    const double hxz = sqrt(hx * hx + hz * hz);
    const double hyz = sqrt(hy * hy + hz * hz);
    const double ax = d.xs * a[d.xa], ay = d.ys * a[d.ya], az = d.sg * a[d.nrm];
    const int64_t sx = d.xs * g.stride[d.xa], sy = d.ys * g.stride[d.ya];
    const int64_t sn = g.stride[d.nrm];
    /* the two in-plane axes, in increasing axis order */
    int u = (d.nrm == 0) ? 1 : 0;
    int v = (d.nrm == 2) ? 1 : 2;
    const int nu = g.n[u], nv = g.n[v];
    const int64_t su = g.stride[u], sv = g.stride[v];
#pragma omp parallel for schedule(static)
    for (int b = 1; b <= nv; ++b)
        for (int c = 1; c <= nu; ++c) {
            int64_t srci = (int64_t)src * sn + (int64_t)c * su + (int64_t)b * sv;
            orc_point(T, srci + d.sg * sn, srci, sx, sy, F, ax, ay, az, hz,
                      hx, hy, hxy, hxz, hyz);
        }
}

/* One directional pass: all planes of direction dir in the driver's order. */
void orc_pass(double *T, int nx, int ny, int nz, double dx, double dy,
              double dz, double F, double a0, double a1, double a2, int dir)
{
    const int n[3] = {nx, ny, nz};
    const orc_dir d = ORC_DIRS[dir];
    const int nn = n[d.nrm];
    if (d.sg > 0)
        for (int s = 1; s < nn; ++s)
            orc_plane(T, nx, ny, nz, dx, dy, dz, F, a0, a1, a2, dir, s);
    else
        for (int s = nn; s > 1; --s)
            orc_plane(T, nx, ny, nz, dx, dy, dz, F, a0, a1, a2, dir, s);
}

/* Sweeps in the reference order (:1192-1237).  Runs exactly nsweeps sweeps
 * when tol < 0; otherwise stops after the first sweep whose max|dT| <= tol
 * (or at nsweeps).  Returns the number of sweeps run; *last_delta receives
 * the max |T_after - T_before| over all cells of the last sweep. */
int orc_solve(double *T, int nx, int ny, int nz, double dx, double dy,
              double dz, double F, double a0, double a1, double a2,
              int nsweeps, double tol, double *last_delta)
{
    const size_t cells = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    double *prev = (double *)malloc(cells * sizeof(double));
    if (!prev)
        return -1;
    int s = 0;
    double delta = 0.0;
    for (s = 0; s < nsweeps;) {
        memcpy(prev, T, cells * sizeof(double));
        for (int dir = 0; dir < 6; ++dir)
            orc_pass(T, nx, ny, nz, dx, dy, dz, F, a0, a1, a2, dir);
        ++s;
        delta = 0.0;
        for (size_t c = 0; c < cells; ++c) {
            double e = fabs(T[c] - prev[c]);
            if (e > delta)
                delta = e;
        }
        if (tol >= 0.0 && delta <= tol)
            break;
    }
    free(prev);
    if (last_delta)
        *last_delta = delta;
    return s;
}

/* ------------------------------------------------------------------------ */
/* Source initialisation                                                     */
/* ------------------------------------------------------------------------ */

/* Exact point-source time of the homogeneous drift medium,
 * Fold3dPMM.c:9-26. */
double orc_fold_from_point(double F, double ax, double ay, double az, double x,
                           double y, double z)
{
    double xsq = x * x + y * y + z * z;
    double adotx = ax * x + ay * y + az * z;
    double q = (F * F - (ax * ax + ay * ay + az * az)) * xsq + adotx * adotx;
    if (q > 0.0) {
        q = adotx + sqrt(q);
        if (q > 0.0)
            return xsq / q;
    }
    return 1.0 * ORC_MAXT;
}

/* Implicit surface whose zero level set is the source, Fold3dPMM.c:29-33. */
double orc_surface(double x, double y, double z)
{
    return 5.0 + (sin(x) + cos(y + x) + sin(x + y + z)) * 0.4 - z +
           (x - 5.0) * (y - 5.0) * (z - 5) / 55.0;
}

typedef struct {
    double *T;
    orc_grid g;
    double F, a[3];
} orc_seed_ctx;

/* Fold3dPMM.c:35-54: min-update of one node from a surface point at
 * (x, y, z) relative to it, sign preserved, drift reversed on the negative
 * side. */
static void orc_node(const orc_seed_ctx *s, double x, double y, double z,
                     int i, int j, int k)
{
    double *T = s->T;
    int64_t id = i + s->g.stride[1] * j + s->g.stride[2] * k;
    double ax = s->a[0], ay = s->a[1], az = s->a[2], F = s->F;
    if (T[id] < 0.0) {
        ax *= -1;
        ay *= -1;
        az *= -1;
    }
    double tnew = orc_fold_from_point(F, ax, ay, az, -x, -y, -z);
    if (tnew < fabs(T[id]))
        T[id] = (osign(T[id]) * 1.0) * tnew;
}

/* The 44 node updates of updateVoxel (Fold3dPMM.c:62-110), in order.  Each
 * row: multiples (of dxx,dyy,dzz) added to the surface point's position, and
 * the node index offset.  Rows 17 and 21 (0-based) keep the reference's position/index
 * mismatches (:82 and :86). */
#define ORC_NVOXEL 44
static const signed char ORC_VOXEL[ORC_NVOXEL][6] = {
    {0, 0, 0, 0, 0, 0},    {-1, 0, 0, 1, 0, 0},   {0, -1, 0, 0, 1, 0},
    {0, 0, -1, 0, 0, 1},   {-1, -1, 0, 1, 1, 0},  {-1, 0, -1, 1, 0, 1},
    {0, -1, -1, 0, 1, 1},  {-1, -1, -1, 1, 1, 1}, {1, 0, 0, -1, 0, 0},
    {1, -1, 0, -1, 1, 0},  {1, 0, -1, -1, 0, 1},  {1, -1, -1, -1, 1, 1},
    {-2, 0, 0, 2, 0, 0},   {-2, -1, 0, 2, 1, 0},  {-2, 0, -1, 2, 0, 1},
    {-2, -1, -1, 2, 1, 1}, {0, 1, 0, 0, -1, 0},   {-1, 1, 0, 1, 0, 0},
    {0, 1, -1, 0, -1, 1},  {-1, 1, -1, 1, -1, 1}, {0, -2, 0, 0, 2, 0},
    {-1, -2, 0, 2, 0, 0},  {0, -2, -1, 0, 2, 1},  {-1, -2, -1, 1, 2, 1},
    {0, 0, 1, 0, 0, -1},   {-1, 0, 1, 1, 0, -1},  {0, -1, 1, 0, 1, -1},
    {-1, -1, 1, 1, 1, -1}, {0, 0, -2, 0, 0, 2},   {-1, 0, -2, 1, 0, 2},
    {0, -1, -2, 0, 1, 2},  {-1, -1, -2, 1, 1, 2}, {0, 1, 1, 0, -1, -1},
    {1, 0, 1, -1, 0, -1},  {1, 1, 0, -1, -1, 0},  {0, -2, -2, 0, 2, 2},
    {-2, 0, -2, 2, 0, 2},  {-2, -2, 0, 2, 2, 0},  {-1, 1, 1, 1, -1, -1},
    {1, -1, 1, -1, 1, -1}, {1, 1, -1, -1, -1, 1}, {-1, -2, -2, 1, 2, 2},
    {-2, -1, -2, 2, 1, 2}, {-2, -2, -1, 2, 2, 1},
};

static inline double orc_shift(double p, int m, double h)
{
    /* p, p+h, p-h, p-2*h exactly as the reference spells them */
    if (m == 0) return p;
    if (m == 1) return p + h;
    if (m == -1) return p - h;
    return p - 2 * h;
}

/* Fold3dPMM.c:56-112 */
static void orc_voxel(const orc_seed_ctx *s, int i, int j, int k, double xp,
                      double yp, double zp, double hx, double hy, double hz)
{
    for (int r = 0; r < ORC_NVOXEL; ++r) {
        const signed char *e = ORC_VOXEL[r];
        orc_node(s, orc_shift(xp, e[0], hx), orc_shift(yp, e[1], hy),
                 orc_shift(zp, e[2], hz), i + e[3], j + e[4], k + e[5]);
    }
}

/* Number of voxels in the last orc_init_implicit call with more than eight
 * edge crossings (the reference's 8-entry buffers would overflow there). */
static long orc_overfull_voxels = 0;
long orc_last_overfull(void) { return orc_overfull_voxels; }

/* Implicit-surface initialisation, ImplicitInitialiser (Fold3dPMM.c:129-389)
 * with run-time sizes and medium.  T must hold (nx+2)(ny+2)(nz+2) doubles. */
int orc_init_implicit(double *T, int nx, int ny, int nz, double hx, double hy,
                      double hz, double F, double a0, double a1, double a2)
{
    orc_seed_ctx s;
    s.T = T;
    s.g = orc_make_grid(nx, ny, nz);
    s.F = F;
    s.a[0] = a0; s.a[1] = a1; s.a[2] = a2;
    const int64_t sy = s.g.stride[1], sz = s.g.stride[2];
    const size_t cells = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    double *IF = (double *)malloc(cells * sizeof(double));
    if (!IF)
        return -1;
    /* :137-147; the coordinate helpers x/y/z are :115-126 */
    for (int i = 0; i < nx + 2; i++)
        for (int j = 0; j < ny + 2; j++)
            for (int k = 0; k < nz + 2; k++) {
                int64_t id = i + sy * j + sz * k;
                IF[id] = orc_surface((i - 1) * hx + 0., (j - 1) * hy + 0.,
                                     (k - 1) * hz + 0.);
                T[id] = (osign(IF[id]) * 1.0) * ORC_MAXT;
            }
    orc_overfull_voxels = 0;
    for (int i = 1; i < nx; i++)
        for (int j = 1; j < ny; j++)
            for (int k = 1; k < nz; k++) {
                const int64_t id = i + sy * j + sz * k;
                const double f = IF[id], fx = IF[id + 1], fy = IF[id + sy],
                             fz = IF[id + sz], fxy = IF[id + 1 + sy],
                             fzx = IF[id + 1 + sz], fzy = IF[id + sy + sz],
                             fxyz = IF[id + 1 + sy + sz];
                double X[12], Y[12], Z[12];
                int np = 0;
                double p;
#define ORC_CROSS(expr, H, px, py, pz)                                         \
    p = (expr);                                                                \
    if (0.0 <= p && p <= H) {                                                  \
        X[np] = (px); Y[np] = (py); Z[np] = (pz); np += 1;                     \
    }
                /* edge crossings, :173-269, in the reference's order */
                ORC_CROSS(hx * f / (f - fx), hx, p, 0.0, 0.0);
                ORC_CROSS(hx * fz / (fz - fzx), hx, p, 0.0, hz);
                ORC_CROSS(hx * fy / (fy - fxy), hx, p, hy, 0.0);
                ORC_CROSS(hx * fzy / (fzy - fxyz), hx, p, hy, hz);
                ORC_CROSS(hy * f / (f - fy), hy, 0.0, p, 0.0);
                ORC_CROSS(hy * fz / (fz - fzy), hy, 0., p, hz);
                ORC_CROSS(hy * fx / (fx - fxy), hy, hx, p, 0.0);
                ORC_CROSS(hy * fzx / (fzx - fxyz), hy, hx, p, hz);
                ORC_CROSS(hz * f / (f - fz), hz, 0.0, 0.0, p);
                ORC_CROSS(hz * fxy / (fxy - fxyz), hz, hx, hy, p);
                ORC_CROSS(hz * fx / (fx - fzx), hz, hx, 0.0, p);
                ORC_CROSS(hz * fy / (fy - fzy), hz, 0.0, hy, p);
#undef ORC_CROSS
                if (np > 8)
                    ++orc_overfull_voxels;
                /* :271-383: every crossing, plus blends with earlier ones.
                 * The blends' z coordinates take Y[l-2] / Y[l-3] where the
                 * reference does (:309-379). */
                for (int l = 0; l < np; l += 1) {
                    orc_voxel(&s, i, j, k, X[l], Y[l], Z[l], hx, hy, hz);
                    for (int b = 1; b <= 5 && b <= l; ++b) {
                        orc_voxel(&s, i, j, k, (2 * X[l] + X[l - b]) / 3,
                                  (2 * Y[l] + Y[l - b]) / 3,
                                  (2 * Z[l] + Z[l - b]) / 3, hx, hy, hz);
                        orc_voxel(&s, i, j, k, (X[l] + 2 * X[l - b]) / 3,
                                  (Y[l] + 2 * Y[l - b]) / 3,
                                  (Z[l] + 2 * Z[l - b]) / 3, hx, hy, hz);
                        if (b == 3) { /* :307-322 */
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 2] + X[l - 3]) / 3,
                                      (Y[l] + Y[l - 2] + Y[l - 3]) / 3,
                                      (Z[l] + Y[l - 2] + Z[l - 3]) / 3, hx, hy,
                                      hz);
                            orc_voxel(&s, i, j, k,
                                      (2 * X[l] + X[l - 2] + X[l - 3]) / 4,
                                      (2 * Y[l] + Y[l - 2] + Y[l - 3]) / 4,
                                      (2 * Z[l] + Y[l - 2] + Z[l - 3]) / 4, hx,
                                      hy, hz);
                            orc_voxel(&s, i, j, k,
                                      (X[l] + 2 * X[l - 2] + X[l - 3]) / 4,
                                      (Y[l] + 2 * Y[l - 2] + Y[l - 3]) / 4,
                                      (Z[l] + 2 * Y[l - 2] + Z[l - 3]) / 4, hx,
                                      hy, hz);
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 2] + 2 * X[l - 3]) / 4,
                                      (Y[l] + Y[l - 2] + 2 * Y[l - 3]) / 4,
                                      (Z[l] + Y[l - 2] + 2 * Z[l - 3]) / 4, hx,
                                      hy, hz);
                        }
                        if (b == 4) { /* :336-347 */
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 2] + X[l - 3]) / 3,
                                      (Y[l] + Y[l - 2] + Y[l - 3]) / 3,
                                      (Z[l] + Y[l - 2] + Z[l - 3]) / 3, hx, hy,
                                      hz);
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 2] + X[l - 4]) / 3,
                                      (Y[l] + Y[l - 2] + Y[l - 4]) / 3,
                                      (Z[l] + Y[l - 2] + Z[l - 4]) / 3, hx, hy,
                                      hz);
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 3] + X[l - 4]) / 3,
                                      (Y[l] + Y[l - 3] + Y[l - 4]) / 3,
                                      (Z[l] + Y[l - 3] + Z[l - 4]) / 3, hx, hy,
                                      hz);
                        }
                        if (b == 5) { /* :361-380 */
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 2] + X[l - 3]) / 3,
                                      (Y[l] + Y[l - 2] + Y[l - 3]) / 3,
                                      (Z[l] + Y[l - 2] + Z[l - 3]) / 3, hx, hy,
                                      hz);
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 2] + X[l - 4]) / 3,
                                      (Y[l] + Y[l - 2] + Y[l - 4]) / 3,
                                      (Z[l] + Y[l - 2] + Z[l - 4]) / 3, hx, hy,
                                      hz);
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 2] + X[l - 5]) / 3,
                                      (Y[l] + Y[l - 2] + Y[l - 5]) / 3,
                                      (Z[l] + Y[l - 2] + Z[l - 5]) / 3, hx, hy,
                                      hz);
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 3] + X[l - 5]) / 3,
                                      (Y[l] + Y[l - 3] + Y[l - 5]) / 3,
                                      (Z[l] + Y[l - 3] + Z[l - 5]) / 3, hx, hy,
                                      hz);
                            orc_voxel(&s, i, j, k,
                                      (X[l] + X[l - 3] + X[l - 4]) / 3,
                                      (Y[l] + Y[l - 3] + Y[l - 4]) / 3,
                                      (Z[l] + Y[l - 3] + Z[l - 4]) / 3, hx, hy,
                                      hz);
                        }
                    }
                }
            }
    free(IF);
    return 0;
}

/* Point source: T = +MAXT everywhere, T[src] = 0. */
void orc_init_point(double *T, int nx, int ny, int nz, int si, int sj, int sk)
{
    const size_t cells = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    for (size_t c = 0; c < cells; ++c)
        T[c] = ORC_MAXT;
    T[si + (int64_t)(nx + 2) * (sj + (int64_t)(ny + 2) * sk)] = 0.0;
}

/* ------------------------------------------------------------------------ */
/* Elliptical (tilted) medium                                                */
/* ------------------------------------------------------------------------ */
/*
 * No counterpart in the reference (its local solver only knows the drift
 * medium).  This is the CPU statement of this repository's own solver for a
 * per-cell Riemannian metric M (travel time of a short straight segment d is
 * sqrt(d^T M d)); the GPU kernel (csrc/fold3d_ellip.cuh) follows it operation
 * by operation, so the two agree bit for bit.
 *
 * In a sweep direction's local frame (x, y in the source plane, z towards
 * the target; unit vectors xs*e[xa], ys*e[ya], sg*e[nrm]) the target X sits
 * at (0, 0, hz) above the source point st, and the eight neighbours at
 * (i*hx, j*hy, 0), i, j in {-1, 0, 1}.  With t linear on each vertex, edge
 * and triangle of that 3 x 3 fan, the new time is
 *     min over the fan of  t(p) + ||X - p||_M,
 * found as: the 9 vertex values, the interior stationary points of the 16
 * edges (8 spokes st-P, 8 rim edges between adjacent neighbours) and of the
 * 8 triangles (st, neighbour, next neighbour), in closed form.  Each
 * candidate exceeds the smallest time it is built from, so a candidate is
 * only computed while the running time is above that smallest time.
 */

/* The metric in a direction's local frame, scaled by the spacings:
 * Axx = M'xx hx hx, Axy = M'xy hx hy, Axz = M'xz hx hz, and so on. */
typedef struct { double xx, yy, zz, xy, xz, yz; } orc_aq;

/* u^T M' v for u = (ui hx, uj hy, uk hz), v likewise (integer coefficients). */
static double orc_bf(const orc_aq *A, int ui, int uj, int uk, int vi, int vj, int vk)
{
    return (double)(ui * vi) * A->xx + (double)(uj * vj) * A->yy + (double)(uk * vk) * A->zz +
           (double)(ui * vj + uj * vi) * A->xy + (double)(ui * vk + uk * vi) * A->xz +
           (double)(uj * vk + uk * vj) * A->yz;
}

/* neighbour offsets in the local frame, st first, then the rim in order */
static const int ORC_RIM[8][2] = {{1, 0}, {1, 1}, {0, 1}, {-1, 1}, {-1, 0}, {-1, -1}, {0, -1}, {1, -1}};

/* Each candidate routine sets *win to its id (see the adjoint below) when it
 * lowers the time, so *win ends as the id of the candidate that set it. */
static void orc_ell_vertex(double *tn, int *win, int id, const orc_aq *A, double tp, int i, int j)
{
    if (!(*tn > tp)) return;
    double c = orc_bf(A, -i, -j, 1, -i, -j, 1);
    if (c > 0.0) {
        double cand = tp + sqrt(c);
        if (cand < *tn) { *tn = cand; *win = id; }
    }
}

/* edge from P (pi,pj) with time tp to Q (qi,qj) with time tq */
static void orc_ell_edge(double *tn, int *win, int id, const orc_aq *A, double tp, double tq, int pi, int pj,
                         int qi, int qj)
{
    if (!(*tn > omin(tp, tq))) return;
    const int ei = qi - pi, ej = qj - pj;
    double a = orc_bf(A, ei, ej, 0, ei, ej, 0);
    double b = orc_bf(A, ei, ej, 0, -pi, -pj, 1);
    double c = orc_bf(A, -pi, -pj, 1, -pi, -pj, 1);
    double d = tq - tp;
    double den = a - d * d;
    double disc = a * c - b * b;
    if (den > 0.0 && disc > 0.0) {
        double n = sqrt(disc / den);
        double lam = (b - d * n) / a;
        if (lam > 0.0 && lam < 1.0) {
            double cand = tp + lam * d + n;
            if (cand < *tn) { *tn = cand; *win = id; }
        }
    }
}

/* triangle st (origin, time t0) - A (ai,aj, time ta) - B (bi,bj, time tb) */
static void orc_ell_tri(double *tn, int *win, int id, const orc_aq *A, double t0, double ta, double tb, int ai,
                        int aj, int bi, int bj)
{
    if (!(*tn > omin(t0, omin(ta, tb)))) return;
    double p11 = orc_bf(A, ai, aj, 0, ai, aj, 0);
    double p12 = orc_bf(A, ai, aj, 0, bi, bj, 0);
    double p22 = orc_bf(A, bi, bj, 0, bi, bj, 0);
    double q1 = orc_bf(A, ai, aj, 0, 0, 0, 1);
    double q2 = orc_bf(A, bi, bj, 0, 0, 0, 1);
    double c = A->zz;
    double d1 = ta - t0, d2 = tb - t0;
    double det = p11 * p22 - p12 * p12;
    if (!(det > 0.0)) return;
    double u1 = p22 * d1 - p12 * d2, u2 = p11 * d2 - p12 * d1;
    double w1 = p22 * q1 - p12 * q2, w2 = p11 * q2 - p12 * q1;
    double s = (d1 * u1 + d2 * u2) / det;
    double r = c - (q1 * w1 + q2 * w2) / det;
    if (s < 1.0 && r > 0.0) {
        double n = sqrt(r / (1.0 - s));
        double l1 = (w1 - n * u1) / det, l2 = (w2 - n * u2) / det;
        if (l1 > 0.0 && l2 > 0.0 && l1 + l2 < 1.0) {
            double cand = t0 + (l1 * d1 + l2 * d2) + n;
            if (cand < *tn) { *tn = cand; *win = id; }
        }
    }
}

/* New signed value of a target from st and the rim values nb[8] (ORC_RIM
 * order); *win: id of the candidate that set it, -1 if none did. */
static double orc_ell_point(double told, double st, const double nb[8], const orc_aq *A, int *win)
{
    double tn = fabs(told);
    *win = -1;
    orc_ell_vertex(&tn, win, 0, A, st, 0, 0);
    double m = st;
    for (int r = 0; r < 8; ++r) m = omin(m, nb[r]);
    if (tn > m) {
        for (int r = 0; r < 8; ++r) orc_ell_vertex(&tn, win, 1 + r, A, nb[r], ORC_RIM[r][0], ORC_RIM[r][1]);
        for (int r = 0; r < 8; ++r) orc_ell_edge(&tn, win, 9 + r, A, st, nb[r], 0, 0, ORC_RIM[r][0], ORC_RIM[r][1]);
        for (int r = 0; r < 8; ++r) {
            const int s = (r + 1) & 7;
            orc_ell_edge(&tn, win, 17 + r, A, nb[r], nb[s], ORC_RIM[r][0], ORC_RIM[r][1], ORC_RIM[s][0],
                         ORC_RIM[s][1]);
        }
        for (int r = 0; r < 8; ++r) {
            const int s = (r + 1) & 7;
            orc_ell_tri(&tn, win, 25 + r, A, st, nb[r], nb[s], ORC_RIM[r][0], ORC_RIM[r][1], ORC_RIM[s][0],
                        ORC_RIM[s][1]);
        }
    }
    return ((told > 0) ? 1.0 : -1.0) * tn;
}

/* Winner record of a cell, one byte: direction * ORC_NCAND + candidate id;
 * ORC_NOWIN when no candidate set its value (a source, or never reached). */
#define ORC_NCAND 33
#define ORC_NOWIN 0xffu

/* The per-cell metric of the FP64 statement: six float arrays (the stored
 * float32 medium) or six double arrays (formed from the FP64 parameter
 * medium by orc_tti_metric); entries xx xy xz yy yz zz. */
typedef struct {
    const float *const *f;
    const double *const *d;
} orc_metric;

static double orc_mget(const orc_metric *M, int k, int64_t t)
{
    return M->d ? M->d[k][t] : (double)M->f[k][t];
}

/* The metric M = a I + b n n^T of the tilted elliptical medium from its FP64
 * parameters (slowness s, Thomsen eps, axis components nx, ny with
 * nz = sqrt(max(0, (1 - nx nx) - ny ny))), cell by cell into six double
 * arrays, in the operation order of the GPU kernels'
 * ell_metric_from_param. */
void orc_tti_metric(const double *S, const double *E, const double *NX, const double *NY, int64_t cells,
                    double *const *out)
{
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < cells; ++c) {
        const double s2 = S[c] * S[c];
        const double a = s2 / (1.0 + 2.0 * E[c]);
        const double b = s2 - a;
        const double nx = NX[c], ny = NY[c];
        const double q = (1.0 - nx * nx) - ny * ny;
        const double nz = sqrt(q > 0.0 ? q : 0.0);
        const double bx = b * nx, by = b * ny, bz = b * nz;
        out[0][c] = a + bx * nx;
        out[1][c] = bx * ny;
        out[2][c] = bx * nz;
        out[3][c] = a + by * ny;
        out[4][c] = by * nz;
        out[5][c] = a + bz * nz;
    }
}

/* index of the global metric component (p,q), arrays ordered xx xy xz yy yz zz */
static int orc_mi(int p, int q)
{
    if (p > q) { int t = p; p = q; q = t; }
    static const int tab[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    return tab[p][q];
}

/* One plane step of the elliptical medium.  M: six float arrays (xx, xy, xz,
 * yy, yz, zz of the metric in the i, j, k axes) in the field layout. */
static void orc_ell_plane_m(double *T, const orc_metric *M, unsigned char *W, int nx, int ny, int nz, double dx,
                            double dy, double dz, int dir, int src)
{
    const orc_grid g = orc_make_grid(nx, ny, nz);
    const orc_dir d = ORC_DIRS[dir];
    const double h[3] = {dx, dy, dz};
    const double hz = h[d.nrm], hx = h[d.xa], hy = h[d.ya];
    const int ax[3] = {d.xa, d.ya, d.nrm};
    const int sgn[3] = {d.xs, d.ys, d.sg};
    const int64_t sn = g.stride[d.nrm];
    const int64_t sx = d.xs * g.stride[d.xa], sy = d.ys * g.stride[d.ya];
    int u = (d.nrm == 0) ? 1 : 0;
    int v = (d.nrm == 2) ? 1 : 2;
    const int nu = g.n[u], nv = g.n[v];
    const int64_t su = g.stride[u], sv = g.stride[v];
#pragma omp parallel for schedule(static)
    for (int b = 1; b <= nv; ++b)
        for (int c = 1; c <= nu; ++c) {
            const int64_t s = (int64_t)src * sn + (int64_t)c * su + (int64_t)b * sv;
            const int64_t t = s + d.sg * sn;
            /* local metric M'_pq = s_p s_q M[ax_p][ax_q], scaled by the spacings */
            orc_aq A;
            A.xx = orc_mget(M, orc_mi(ax[0], ax[0]), t) * hx * hx;
            A.yy = orc_mget(M, orc_mi(ax[1], ax[1]), t) * hy * hy;
            A.zz = orc_mget(M, orc_mi(ax[2], ax[2]), t) * hz * hz;
            A.xy = (double)(sgn[0] * sgn[1]) * orc_mget(M, orc_mi(ax[0], ax[1]), t) * hx * hy;
            A.xz = (double)(sgn[0] * sgn[2]) * orc_mget(M, orc_mi(ax[0], ax[2]), t) * hx * hz;
            A.yz = (double)(sgn[1] * sgn[2]) * orc_mget(M, orc_mi(ax[1], ax[2]), t) * hy * hz;
            double nb[8];
            for (int r = 0; r < 8; ++r) nb[r] = fabs(T[s + ORC_RIM[r][0] * sx + ORC_RIM[r][1] * sy]);
            int win;
            const double nv = orc_ell_point(T[t], fabs(T[s]), nb, &A, &win);
            if (W && memcmp(&nv, &T[t], sizeof nv) != 0)
                W[t] = (win < 0) ? ORC_NOWIN : (unsigned char)(dir * ORC_NCAND + win);
            T[t] = nv;
        }
}

void orc_ell_plane_rec(double *T, const float *const *M, unsigned char *W, int nx, int ny, int nz, double dx,
                       double dy, double dz, int dir, int src)
{
    const orc_metric m = {M, NULL};
    orc_ell_plane_m(T, &m, W, nx, ny, nz, dx, dy, dz, dir, src);
}

/* One plane step with a double metric (the FP64 parameter medium, formed by
 * orc_tti_metric). */
void orc_ell_plane_d(double *T, const double *const *M, int nx, int ny, int nz, double dx, double dy, double dz,
                     int dir, int src)
{
    const orc_metric m = {NULL, M};
    orc_ell_plane_m(T, &m, NULL, nx, ny, nz, dx, dy, dz, dir, src);
}

void orc_ell_plane(double *T, const float *const *M, int nx, int ny, int nz, double dx, double dy, double dz,
                   int dir, int src)
{
    orc_ell_plane_rec(T, M, NULL, nx, ny, nz, dx, dy, dz, dir, src);
}

/* Sweeps of the elliptical medium in the reference's direction order;
 * semantics as orc_solve. */
static int orc_ell_solve_m(double *T, const orc_metric *M, unsigned char *W, int nx, int ny, int nz, double dx,
                           double dy, double dz, int nsweeps, double tol, double *last_delta)
{
    const size_t cells = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    const int n[3] = {nx, ny, nz};
    double *prev = (double *)malloc(cells * sizeof(double));
    if (!prev) return -1;
    int s = 0;
    double delta = 0.0;
    for (s = 0; s < nsweeps;) {
        memcpy(prev, T, cells * sizeof(double));
        for (int dir = 0; dir < 6; ++dir) {
            const orc_dir d = ORC_DIRS[dir];
            const int nn = n[d.nrm];
            if (d.sg > 0)
                for (int p = 1; p < nn; ++p) orc_ell_plane_m(T, M, W, nx, ny, nz, dx, dy, dz, dir, p);
            else
                for (int p = nn; p > 1; --p) orc_ell_plane_m(T, M, W, nx, ny, nz, dx, dy, dz, dir, p);
        }
        ++s;
        delta = 0.0;
        for (size_t c = 0; c < cells; ++c) {
            double e = fabs(T[c] - prev[c]);
            if (e > delta) delta = e;
        }
        if (tol >= 0.0 && delta <= tol) break;
    }
    free(prev);
    if (last_delta) *last_delta = delta;
    return s;
}

int orc_ell_solve_rec(double *T, const float *const *M, unsigned char *W, int nx, int ny, int nz, double dx,
                      double dy, double dz, int nsweeps, double tol, double *last_delta)
{
    const orc_metric m = {M, NULL};
    return orc_ell_solve_m(T, &m, W, nx, ny, nz, dx, dy, dz, nsweeps, tol, last_delta);
}

/* The same with a double metric (the FP64 parameter medium, orc_tti_metric). */
int orc_ell_solve_rec_d(double *T, const double *const *M, unsigned char *W, int nx, int ny, int nz, double dx,
                        double dy, double dz, int nsweeps, double tol, double *last_delta)
{
    const orc_metric m = {NULL, M};
    return orc_ell_solve_m(T, &m, W, nx, ny, nz, dx, dy, dz, nsweeps, tol, last_delta);
}

int orc_ell_solve(double *T, const float *const *M, int nx, int ny, int nz, double dx, double dy, double dz,
                  int nsweeps, double tol, double *last_delta)
{
    return orc_ell_solve_rec(T, M, NULL, nx, ny, nz, dx, dy, dz, nsweeps, tol, last_delta);
}

/* ------------------------------------------------------------------------ */
/* The float32 build of the elliptical solver: the same computation with     */
/* float fields and float arithmetic throughout (spacings rounded to float   */
/* first, float literals, sqrtf), as the GPU's float instantiation.  x86-64  */
/* evaluates float expressions in float (FLT_EVAL_METHOD 0).                 */
/* ------------------------------------------------------------------------ */
typedef struct { float xx, yy, zz, xy, xz, yz; } orc_aqf;

static float orc_bff(const orc_aqf *A, int ui, int uj, int uk, int vi, int vj, int vk)
{
    return (float)(ui * vi) * A->xx + (float)(uj * vj) * A->yy + (float)(uk * vk) * A->zz +
           (float)(ui * vj + uj * vi) * A->xy + (float)(ui * vk + uk * vi) * A->xz +
           (float)(uj * vk + uk * vj) * A->yz;
}

static float ominf(float a, float b) { return (a < b) ? a : b; }

static void orc_ellf_vertex(float *tn, int *win, int id, const orc_aqf *A, float tp, int i, int j)
{
    if (!(*tn > tp)) return;
    const float c = orc_bff(A, -i, -j, 1, -i, -j, 1);
    if (c > 0.0f) {
        const float cand = tp + sqrtf(c);
        if (cand < *tn) { *tn = cand; *win = id; }
    }
}

static void orc_ellf_edge(float *tn, int *win, int id, const orc_aqf *A, float tp, float tq, int pi, int pj, int qi,
                          int qj)
{
    if (!(*tn > ominf(tp, tq))) return;
    const int ei = qi - pi, ej = qj - pj;
    const float a = orc_bff(A, ei, ej, 0, ei, ej, 0);
    const float b = orc_bff(A, ei, ej, 0, -pi, -pj, 1);
    const float c = orc_bff(A, -pi, -pj, 1, -pi, -pj, 1);
    const float d = tq - tp;
    const float den = a - d * d;
    const float disc = a * c - b * b;
    if (den > 0.0f && disc > 0.0f) {
        const float n = sqrtf(disc / den);
        const float lam = (b - d * n) / a;
        if (lam > 0.0f && lam < 1.0f) {
            const float cand = tp + lam * d + n;
            if (cand < *tn) { *tn = cand; *win = id; }
        }
    }
}

static void orc_ellf_tri(float *tn, int *win, int id, const orc_aqf *A, float t0, float ta, float tb, int ai, int aj,
                         int bi, int bj)
{
    if (!(*tn > ominf(t0, ominf(ta, tb)))) return;
    const float p11 = orc_bff(A, ai, aj, 0, ai, aj, 0);
    const float p12 = orc_bff(A, ai, aj, 0, bi, bj, 0);
    const float p22 = orc_bff(A, bi, bj, 0, bi, bj, 0);
    const float q1 = orc_bff(A, ai, aj, 0, 0, 0, 1);
    const float q2 = orc_bff(A, bi, bj, 0, 0, 0, 1);
    const float c = A->zz;
    const float d1 = ta - t0, d2 = tb - t0;
    const float det = p11 * p22 - p12 * p12;
    if (!(det > 0.0f)) return;
    const float u1 = p22 * d1 - p12 * d2, u2 = p11 * d2 - p12 * d1;
    const float w1 = p22 * q1 - p12 * q2, w2 = p11 * q2 - p12 * q1;
    const float s = (d1 * u1 + d2 * u2) / det;
    const float r = c - (q1 * w1 + q2 * w2) / det;
    if (s < 1.0f && r > 0.0f) {
        const float n = sqrtf(r / (1.0f - s));
        const float l1 = (w1 - n * u1) / det, l2 = (w2 - n * u2) / det;
        if (l1 > 0.0f && l2 > 0.0f && l1 + l2 < 1.0f) {
            const float cand = t0 + (l1 * d1 + l2 * d2) + n;
            if (cand < *tn) { *tn = cand; *win = id; }
        }
    }
}

static float orc_ellf_point(float told, float st, const float nb[8], const orc_aqf *A, int *win)
{
    float tn = fabsf(told);
    *win = -1;
    orc_ellf_vertex(&tn, win, 0, A, st, 0, 0);
    float m = st;
    for (int r = 0; r < 8; ++r) m = ominf(m, nb[r]);
    if (tn > m) {
        for (int r = 0; r < 8; ++r) orc_ellf_vertex(&tn, win, 1 + r, A, nb[r], ORC_RIM[r][0], ORC_RIM[r][1]);
        for (int r = 0; r < 8; ++r) orc_ellf_edge(&tn, win, 9 + r, A, st, nb[r], 0, 0, ORC_RIM[r][0], ORC_RIM[r][1]);
        for (int r = 0; r < 8; ++r) {
            const int s = (r + 1) & 7;
            orc_ellf_edge(&tn, win, 17 + r, A, nb[r], nb[s], ORC_RIM[r][0], ORC_RIM[r][1], ORC_RIM[s][0],
                          ORC_RIM[s][1]);
        }
        for (int r = 0; r < 8; ++r) {
            const int s = (r + 1) & 7;
            orc_ellf_tri(&tn, win, 25 + r, A, st, nb[r], nb[s], ORC_RIM[r][0], ORC_RIM[r][1], ORC_RIM[s][0],
                         ORC_RIM[s][1]);
        }
    }
    return ((told > 0.0f) ? 1.0f : -1.0f) * tn;
}

void orc_ellf_plane_rec(float *T, const float *const *M, unsigned char *W, int nx, int ny, int nz, double dx,
                        double dy, double dz, int dir, int src)
{
    const orc_grid g = orc_make_grid(nx, ny, nz);
    const orc_dir d = ORC_DIRS[dir];
    const double h[3] = {dx, dy, dz};
    const float hz = (float)h[d.nrm], hx = (float)h[d.xa], hy = (float)h[d.ya];
    const int ax[3] = {d.xa, d.ya, d.nrm};
    const int sgn[3] = {d.xs, d.ys, d.sg};
    const int64_t sn = g.stride[d.nrm];
    const int64_t sx = d.xs * g.stride[d.xa], sy = d.ys * g.stride[d.ya];
    int u = (d.nrm == 0) ? 1 : 0;
    int v = (d.nrm == 2) ? 1 : 2;
    const int nu = g.n[u], nv = g.n[v];
    const int64_t su = g.stride[u], sv = g.stride[v];
#pragma omp parallel for schedule(static)
    for (int b = 1; b <= nv; ++b)
        for (int c = 1; c <= nu; ++c) {
            const int64_t s = (int64_t)src * sn + (int64_t)c * su + (int64_t)b * sv;
            const int64_t t = s + d.sg * sn;
            orc_aqf A;
            A.xx = M[orc_mi(ax[0], ax[0])][t] * hx * hx;
            A.yy = M[orc_mi(ax[1], ax[1])][t] * hy * hy;
            A.zz = M[orc_mi(ax[2], ax[2])][t] * hz * hz;
            A.xy = (float)(sgn[0] * sgn[1]) * M[orc_mi(ax[0], ax[1])][t] * hx * hy;
            A.xz = (float)(sgn[0] * sgn[2]) * M[orc_mi(ax[0], ax[2])][t] * hx * hz;
            A.yz = (float)(sgn[1] * sgn[2]) * M[orc_mi(ax[1], ax[2])][t] * hy * hz;
            float nb[8];
            for (int r = 0; r < 8; ++r) nb[r] = fabsf(T[s + ORC_RIM[r][0] * sx + ORC_RIM[r][1] * sy]);
            int win;
            const float nvv = orc_ellf_point(T[t], fabsf(T[s]), nb, &A, &win);
            if (W && memcmp(&nvv, &T[t], sizeof nvv) != 0)
                W[t] = (win < 0) ? ORC_NOWIN : (unsigned char)(dir * ORC_NCAND + win);
            T[t] = nvv;
        }
}

/* Sweeps of the float32 build; semantics as orc_ell_solve_rec (the change
 * of a sweep measured in float, reported as double). */
int orc_ellf_solve_rec(float *T, const float *const *M, unsigned char *W, int nx, int ny, int nz, double dx,
                       double dy, double dz, int nsweeps, double tol, double *last_delta)
{
    const size_t cells = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    const int n[3] = {nx, ny, nz};
    float *prev = (float *)malloc(cells * sizeof(float));
    if (!prev) return -1;
    int s = 0;
    double delta = 0.0;
    for (s = 0; s < nsweeps;) {
        memcpy(prev, T, cells * sizeof(float));
        for (int dir = 0; dir < 6; ++dir) {
            const orc_dir d = ORC_DIRS[dir];
            const int nn = n[d.nrm];
            if (d.sg > 0)
                for (int p = 1; p < nn; ++p) orc_ellf_plane_rec(T, M, W, nx, ny, nz, dx, dy, dz, dir, p);
            else
                for (int p = nn; p > 1; --p) orc_ellf_plane_rec(T, M, W, nx, ny, nz, dx, dy, dz, dir, p);
        }
        ++s;
        delta = 0.0;
        for (size_t c = 0; c < cells; ++c) {
            const float df = T[c] - prev[c];
            const double e = fabs((double)df);
            if (e > delta) delta = e;
        }
        if (tol >= 0.0 && delta <= tol) break;
    }
    free(prev);
    if (last_delta) *last_delta = delta;
    return s;
}

/* ------------------------------------------------------------------------ */
/* Adjoint of the elliptical solver                                          */
/* ------------------------------------------------------------------------ */
/*
 * At convergence every reached cell's time equals one candidate of one sweep
 * direction (re-evaluating any direction leaves it unchanged).  That
 * candidate -- the "winner" -- is t(footpoint) + ||X - footpoint||_M with the
 * footpoint on a vertex, edge or triangle of the direction's source plane;
 * by the envelope theorem its derivative with respect to each source time is
 * that source's barycentric weight at the footpoint, and with respect to the
 * local metric entry A_ij it is c_i c_j / (2 n) (c the footpoint-to-target
 * vector in spacing units, n its length; off-diagonal entries count twice).
 *
 * Winner ids: 0 the source point st (vertex), 1..8 rim vertices, 9..16
 * spokes st-rim[r], 17..24 rim edges rim[r]-rim[r+1], 25..32 triangles
 * (st, rim[r], rim[r+1]).  The winner is the first (direction in sweep
 * order, then id) whose value equals |T| bit for bit.
 */
typedef struct {
    int dir, id, np;         /* np source points (0 if none: source or unreached) */
    int64_t src[3];          /* their field indices */
    double w[3];             /* their weights */
    double dM[6];            /* d(time)/d(metric entry xx xy xz yy yz zz), global axes */
} orc_winner;

static const int ORC_RIMX[9] = {0, 1, 1, 0, -1, -1, -1, 0, 1}; /* point 0 = st, 1..8 = rim */
static const int ORC_RIMY[9] = {0, 0, 1, 1, 1, 0, -1, -1, -1};

/* Evaluate candidate `id` without gates; returns its value (or +inf) and
 * fills the footpoint weights over points pt[] (0 = st, 1..8 = rim) and the
 * vector c (spacing units). */
static double orc_ell_cand(const orc_aq *A, const double tv[9], int id, int pt[3], double w[3], int *np,
                           double c[3], double *nlen)
{
    *np = 0;
    if (id <= 8) { /* vertex */
        const int i = ORC_RIMX[id], j = ORC_RIMY[id];
        double q = orc_bf(A, -i, -j, 1, -i, -j, 1);
        if (!(q > 0.0)) return INFINITY;
        *np = 1; pt[0] = id; w[0] = 1.0;
        c[0] = -i; c[1] = -j; c[2] = 1.0;
        *nlen = sqrt(q);
        return tv[id] + *nlen;
    }
    if (id <= 24) { /* edge */
        int P, Q;
        if (id <= 16) { P = 0; Q = id - 8; } else { P = id - 16; Q = (id - 16) % 8 + 1; }
        const int pi = ORC_RIMX[P], pj = ORC_RIMY[P], qi = ORC_RIMX[Q], qj = ORC_RIMY[Q];
        const int ei = qi - pi, ej = qj - pj;
        double a = orc_bf(A, ei, ej, 0, ei, ej, 0);
        double b = orc_bf(A, ei, ej, 0, -pi, -pj, 1);
        double cc = orc_bf(A, -pi, -pj, 1, -pi, -pj, 1);
        double d = tv[Q] - tv[P];
        double den = a - d * d;
        double disc = a * cc - b * b;
        if (!(den > 0.0 && disc > 0.0)) return INFINITY;
        double n = sqrt(disc / den);
        double lam = (b - d * n) / a;
        if (!(lam > 0.0 && lam < 1.0)) return INFINITY;
        *np = 2; pt[0] = P; pt[1] = Q; w[0] = 1.0 - lam; w[1] = lam;
        c[0] = -pi - lam * ei; c[1] = -pj - lam * ej; c[2] = 1.0;
        *nlen = n;
        return tv[P] + lam * d + n;
    }
    { /* triangle st, rim[r], rim[r+1] */
        const int r = id - 25, Pa = r + 1, Pb = (r + 1) % 8 + 1;
        const int ai = ORC_RIMX[Pa], aj = ORC_RIMY[Pa], bi = ORC_RIMX[Pb], bj = ORC_RIMY[Pb];
        double p11 = orc_bf(A, ai, aj, 0, ai, aj, 0);
        double p12 = orc_bf(A, ai, aj, 0, bi, bj, 0);
        double p22 = orc_bf(A, bi, bj, 0, bi, bj, 0);
        double q1 = orc_bf(A, ai, aj, 0, 0, 0, 1);
        double q2 = orc_bf(A, bi, bj, 0, 0, 0, 1);
        double cz = A->zz;
        double d1 = tv[Pa] - tv[0], d2 = tv[Pb] - tv[0];
        double det = p11 * p22 - p12 * p12;
        if (!(det > 0.0)) return INFINITY;
        double u1 = p22 * d1 - p12 * d2, u2 = p11 * d2 - p12 * d1;
        double w1 = p22 * q1 - p12 * q2, w2 = p11 * q2 - p12 * q1;
        double s = (d1 * u1 + d2 * u2) / det;
        double rr = cz - (q1 * w1 + q2 * w2) / det;
        if (!(s < 1.0 && rr > 0.0)) return INFINITY;
        double n = sqrt(rr / (1.0 - s));
        double l1 = (w1 - n * u1) / det, l2 = (w2 - n * u2) / det;
        if (!(l1 > 0.0 && l2 > 0.0 && l1 + l2 < 1.0)) return INFINITY;
        *np = 3; pt[0] = 0; pt[1] = Pa; pt[2] = Pb;
        w[0] = 1.0 - l1 - l2; w[1] = l1; w[2] = l2;
        c[0] = -l1 * ai - l2 * bi; c[1] = -l1 * aj - l2 * bj; c[2] = 1.0;
        *nlen = n;
        return tv[0] + (l1 * d1 + l2 * d2) + n;
    }
}

static void orc_ell_local(const orc_metric *M, int64_t t, const orc_dir *d, const double h[3], orc_aq *A,
                          double *hx, double *hy, double *hz)
{
    const int ax[3] = {d->xa, d->ya, d->nrm};
    const int sgn[3] = {d->xs, d->ys, d->sg};
    *hz = h[d->nrm]; *hx = h[d->xa]; *hy = h[d->ya];
    A->xx = orc_mget(M, orc_mi(ax[0], ax[0]), t) * *hx * *hx;
    A->yy = orc_mget(M, orc_mi(ax[1], ax[1]), t) * *hy * *hy;
    A->zz = orc_mget(M, orc_mi(ax[2], ax[2]), t) * *hz * *hz;
    A->xy = (double)(sgn[0] * sgn[1]) * orc_mget(M, orc_mi(ax[0], ax[1]), t) * *hx * *hy;
    A->xz = (double)(sgn[0] * sgn[2]) * orc_mget(M, orc_mi(ax[0], ax[2]), t) * *hx * *hz;
    A->yz = (double)(sgn[1] * sgn[2]) * orc_mget(M, orc_mi(ax[1], ax[2]), t) * *hy * *hz;
}

/* Winner of interior cell (i,j,k) of a converged field. */
static void orc_ell_winner_at(const double *T, const orc_metric *M, const orc_grid *g, const double h[3], int i,
                              int j, int k, orc_winner *wn)
{
    memset(wn, 0, sizeof *wn);
    wn->dir = -1;
    const int64_t x = i + g->stride[1] * j + g->stride[2] * k;
    const double tx = fabs(T[x]);
    if (!(tx > 0.0) || tx >= ORC_MAXT) return;
    const int c3[3] = {i, j, k};
    double best = INFINITY;
    int bdir = -1, bid = -1;
    /* first pass: the first exact match, else the smallest candidate */
    for (int dir = 0; dir < 6 && !(best == tx); ++dir) {
        const orc_dir d = ORC_DIRS[dir];
        const int sc = c3[d.nrm] - d.sg;
        if (sc < 1 || sc > g->n[d.nrm]) continue;
        const int64_t st = x - d.sg * g->stride[d.nrm];
        const int64_t sx = d.xs * g->stride[d.xa], sy = d.ys * g->stride[d.ya];
        double tv[9];
        for (int p = 0; p < 9; ++p) tv[p] = fabs(T[st + ORC_RIMX[p] * sx + ORC_RIMY[p] * sy]);
        orc_aq A;
        double hx, hy, hz;
        orc_ell_local(M, x, &d, h, &A, &hx, &hy, &hz);
        for (int id = 0; id <= 32; ++id) {
            int pt[3], np;
            double w[3], cv[3], n;
            double v = orc_ell_cand(&A, tv, id, pt, w, &np, cv, &n);
            if (v == tx || v < best) {
                best = v;
                bdir = dir;
                bid = id;
                if (v == tx) break;
            }
        }
    }
    if (bdir < 0) return;
    for (int dir = bdir; dir <= bdir; ++dir) {
        const orc_dir d = ORC_DIRS[dir];
        const int sc = c3[d.nrm] - d.sg; /* source plane coordinate */
        if (sc < 1 || sc > g->n[d.nrm]) continue;
        const int64_t st = x - d.sg * g->stride[d.nrm];
        const int64_t sx = d.xs * g->stride[d.xa], sy = d.ys * g->stride[d.ya];
        int64_t idx[9];
        double tv[9];
        for (int p = 0; p < 9; ++p) {
            idx[p] = st + ORC_RIMX[p] * sx + ORC_RIMY[p] * sy;
            tv[p] = fabs(T[idx[p]]);
        }
        orc_aq A;
        double hx, hy, hz;
        orc_ell_local(M, x, &d, h, &A, &hx, &hy, &hz);
        for (int id = bid; id <= bid; ++id) {
            int pt[3], np;
            double w[3], cv[3], n;
            orc_ell_cand(&A, tv, id, pt, w, &np, cv, &n);
            {
                wn->dir = dir;
                wn->id = id;
                wn->np = np;
                for (int q = 0; q < np; ++q) { wn->src[q] = idx[pt[q]]; wn->w[q] = w[q]; }
                /* d/dA_ij, then to the global entries through A = s_p s_q M h_p h_q */
                const double hh[3] = {hx, hy, hz};
                const int ax[3] = {d.xa, d.ya, d.nrm};
                const int sgn[3] = {d.xs, d.ys, d.sg};
                for (int p = 0; p < 3; ++p)
                    for (int q = p; q < 3; ++q) {
                        double dA = cv[p] * cv[q] / ((p == q ? 2.0 : 1.0) * n);
                        wn->dM[orc_mi(ax[p], ax[q])] += dA * (double)(sgn[p] * sgn[q]) * hh[p] * hh[q];
                    }
                return;
            }
        }
    }
}

/* Weights and metric derivative of the recorded winner (dir, id) of cell x,
 * evaluated with the final field. */
static void orc_ell_weights(const double *T, const orc_metric *M, const orc_grid *g, const double h[3], int64_t x,
                            int dir, int id, orc_winner *wn)
{
    memset(wn, 0, sizeof *wn);
    wn->dir = dir;
    wn->id = id;
    const orc_dir d = ORC_DIRS[dir];
    const int64_t st = x - d.sg * g->stride[d.nrm];
    const int64_t sx = d.xs * g->stride[d.xa], sy = d.ys * g->stride[d.ya];
    int64_t idx[9];
    double tv[9];
    for (int p = 0; p < 9; ++p) {
        idx[p] = st + ORC_RIMX[p] * sx + ORC_RIMY[p] * sy;
        tv[p] = fabs(T[idx[p]]);
    }
    orc_aq A;
    double hx, hy, hz;
    orc_ell_local(M, x, &d, h, &A, &hx, &hy, &hz);
    int pt[3], np;
    double w[3], cv[3], n;
    double v = orc_ell_cand(&A, tv, id, pt, w, &np, cv, &n);
    if (!(v < INFINITY)) return; /* no longer a valid footpoint: no dependency */
    wn->np = np;
    for (int q = 0; q < np; ++q) { wn->src[q] = idx[pt[q]]; wn->w[q] = w[q]; }
    const double hh[3] = {hx, hy, hz};
    const int ax[3] = {d.xa, d.ya, d.nrm};
    const int sgn[3] = {d.xs, d.ys, d.sg};
    for (int p = 0; p < 3; ++p)
        for (int q = p; q < 3; ++q) {
            double dA = cv[p] * cv[q] / ((p == q ? 2.0 : 1.0) * n);
            wn->dM[orc_mi(ax[p], ax[q])] += dA * (double)(sgn[p] * sgn[q]) * hh[p] * hh[q];
        }
}

static const double *orc_sort_T;
static int orc_cmp_desc(const void *a, const void *b)
{
    const double x = fabs(orc_sort_T[*(const int64_t *)a]), y = fabs(orc_sort_T[*(const int64_t *)b]);
    return (x < y) - (x > y);
}

/* Winners of all interior cells: dir/id (-1 if none) and weights, for tests. */
void orc_ell_winners(const double *T, const float *const *Mf, int nx, int ny, int nz, double dx, double dy,
                     double dz, int *dir_out, int *id_out, double *w_out /* 3 per cell */)
{
    const orc_metric mm = {Mf, NULL}, *M = &mm;
    const orc_grid g = orc_make_grid(nx, ny, nz);
    const double h[3] = {dx, dy, dz};
    const size_t cells = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    for (size_t c = 0; c < cells; ++c) { dir_out[c] = -1; id_out[c] = -1; w_out[3 * c] = w_out[3 * c + 1] = w_out[3 * c + 2] = 0.0; }
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                orc_winner wn;
                orc_ell_winner_at(T, M, &g, h, i, j, k, &wn);
                const int64_t x = i + g.stride[1] * j + g.stride[2] * k;
                dir_out[x] = wn.dir;
                id_out[x] = wn.id;
                for (int q = 0; q < 3; ++q) w_out[3 * x + q] = wn.w[q];
            }
}

/* FP64 adjoint: given the converged field T and r = dL/dT (field layout),
 * returns lambda (dL/dT total) and dL/dM (6 arrays, component-major, field
 * layout).  Cells are processed by decreasing time; the return value is the
 * number of winner weights that point to a source point whose time is not
 * smaller (0 for a causal field, for which the order is exact). */
static long orc_ell_adjoint_m(const double *T, const orc_metric *M, const unsigned char *rec, int nx, int ny,
                              int nz, double dx, double dy, double dz, const double *r, double *lambda, double *dLdM)
{
    const orc_grid g = orc_make_grid(nx, ny, nz);
    const double h[3] = {dx, dy, dz};
    const size_t cells = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    orc_winner *W = (orc_winner *)malloc(cells * sizeof(orc_winner));
    int64_t *order = (int64_t *)malloc(cells * sizeof(int64_t));
    if (!W || !order) { free(W); free(order); return -1; }
    memset(W, 0, cells * sizeof(orc_winner));
    size_t nint = 0;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) order[nint++] = i + g.stride[1] * j + g.stride[2] * k;
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < nint; ++q) {
        const int64_t x = order[q];
        const int k = (int)(x / g.stride[2]), j = (int)((x % g.stride[2]) / g.stride[1]), i = (int)(x % g.stride[1]);
        if (rec) {
            if (rec[x] < 6 * ORC_NCAND) orc_ell_weights(T, M, &g, h, x, rec[x] / ORC_NCAND, rec[x] % ORC_NCAND, &W[x]);
        } else {
            orc_ell_winner_at(T, M, &g, h, i, j, k, &W[x]);
        }
    }
    orc_sort_T = T;
    qsort(order, nint, sizeof(int64_t), orc_cmp_desc);
    memcpy(lambda, r, cells * sizeof(double));
    long noncausal = 0;
    for (size_t q = 0; q < nint; ++q) {
        const int64_t x = order[q];
        const orc_winner *wn = &W[x];
        for (int s = 0; s < wn->np; ++s) {
            if (wn->w[s] > 0.0 && !(fabs(T[wn->src[s]]) < fabs(T[x]))) ++noncausal;
            lambda[wn->src[s]] += wn->w[s] * lambda[x];
        }
    }
    for (size_t c = 0; c < 6 * cells; ++c) dLdM[c] = 0.0;
    for (size_t q = 0; q < nint; ++q) {
        const int64_t x = order[q];
        for (int m = 0; m < 6; ++m) dLdM[m * cells + x] = lambda[x] * W[x].dM[m];
    }
    free(W);
    free(order);
    return noncausal;
}

long orc_ell_adjoint_rec(const double *T, const float *const *M, const unsigned char *rec, int nx, int ny, int nz,
                         double dx, double dy, double dz, const double *r, double *lambda, double *dLdM)
{
    const orc_metric m = {M, NULL};
    return orc_ell_adjoint_m(T, &m, rec, nx, ny, nz, dx, dy, dz, r, lambda, dLdM);
}

/* The same with a double metric (the FP64 parameter medium, orc_tti_metric);
 * dLdM is the gradient with respect to its six entries. */
long orc_ell_adjoint_rec_d(const double *T, const double *const *M, const unsigned char *rec, int nx, int ny,
                           int nz, double dx, double dy, double dz, const double *r, double *lambda, double *dLdM)
{
    const orc_metric m = {NULL, M};
    return orc_ell_adjoint_m(T, &m, rec, nx, ny, nz, dx, dy, dz, r, lambda, dLdM);
}

/* Adjoint with winners found from the converged field (first candidate, in
 * direction and id order, equal to the time; else the closest). */
long orc_ell_adjoint(const double *T, const float *const *M, int nx, int ny, int nz, double dx, double dy, double dz,
                     const double *r, double *lambda, double *dLdM)
{
    return orc_ell_adjoint_rec(T, M, NULL, nx, ny, nz, dx, dy, dz, r, lambda, dLdM);
}
