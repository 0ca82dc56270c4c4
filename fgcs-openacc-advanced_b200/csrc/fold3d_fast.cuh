// fold3d_fast.cuh -- the Fold3dPMM point update with its per-direction
// constants folded on the host.
//
// Same results as fold3d_solver.cuh, bit for bit.  Two facts make that
// possible:
//
// 1. Every argument of the reference's 24 local-solver calls that does not
//    depend on the previous-plane values -- the rotated drifts
//    ((ax*dxx + ay*dyy)/dxy and the like, AN_ISO_1_OpenACC.c:243-253,
//    :172-173), F*F - ay*ay, F*F - az*az, the whole fall-back candidate of
//    FoldEdge2Points except the final addition (:99-113), and the 1-D normal
//    candidate except the final addition (:214-228) -- is a constant of the
//    sweep direction and of the side of the target (the drift is negated on
//    the negative side).  The host evaluates those constants with the same
//    expressions and the same IEEE double rounding (no FMA contraction), and
//    the kernel reads them from a table.
//
// 2. Three of the four divisions in each solver body divide by such a
//    constant c.  They are computed as correctly rounded quotients without a
//    division instruction, from r = RN(1/c) (Markstein's method, P. Markstein,
//    "Computation of elementary functions on the IBM RISC System/6000
//    processor", IBM J. Res. Dev. 34(1), 1990): q0 = RN(x*r); one
//    remainder-correction step with the exact FMA remainder x - c*q gives a
//    quotient within one ulp, and a second step then yields RN(x/c).  This
//    holds for normal, finite operands and quotients, which is the case for
//    every such division in the sweep (travel-time differences over grid
//    spacings and bounded slowness terms).
//
// Data-dependent square roots and the two divisions by data-dependent
// values keep CUDA's IEEE operations.  The candidate bodies run as loops over
// table slots instead of 24 inlined copies, which keeps the kernel small.
// Because each solver call only accepts candidates strictly below the
// current time, and every gate that depends on the current time only skips
// calls that could not lower it, the update is min(T_old, candidates), so the
// slot loop may visit the calls in any order; it keeps the reference's order.
//
// 3. One more such gate skips a FoldSurf3Points body (its nested edge still
//    runs) when the current time is at most min(s0, s1, s2) + B.  The body
//    solves the drift medium's eikonal F|p| + a.p = 1 for the plane wave
//    through the three base values and takes the root whose ray, of
//    direction F p/|p| + a, points from the base plane to the target (:152);
//    it accepts the candidate only if that ray leaves the base triangle at a
//    point inside it (:158-163).  The time there, interpolated linearly, is
//    at least the smallest base value, and the ray then crosses the slab of
//    width dzz between base and target, which takes at least dzz / (F + az):
//    one time unit after leaving a point, the front is the sphere
//    |x - a| = F.  B is the larger of that bound and one proved per call
//    site by a search over the body's two gradients (fold3d_tables.cpp),
//    less a relative 1e-3, far above the body's rounding (below 1e-6
//    relative where F^2 >= 1.1 |a|^2, through the square root of a cancelled
//    difference); 0 for stronger drifts.
//
// 4. FoldEdge2Points bodies get a gate of the same kind, B in EdgeK.
//    Its footpoint test (:88,92) does not follow the ray of its own root: it
//    uses the direction w = (F'/F) p/|p| + a2 (F' = sqrt(F^2 - ay^2),
//    a2 = (ax, az), p = (d, c) the plane wave's slowness, which satisfies
//    F'|p| + a2.p = 1), where the ray is F' p/|p| + a2.  So the candidate
//    exceeds the linear time at the test's footpoint (at least min(s0, s1))
//    by dzz (p.w) / w_z, with p.w = 1 - F'|p| (1 - 1/F).  When
//      - ga > 0 and |ax| < sqrt(ga) (then c0 = 1 - d ax > 0 wherever the
//        root exists, and the root is the upper one of F'|p| + a2.p = 1,
//        whose ray points towards the target),
//      - F' > |a2| (so |p| <= 1 / (F' - |a2|)), and
//      - F >= 1 with az >= 0, or F <= 1 with az <= 0 (then w_z > 0 too),
//    p.w >= 1 - F'(1 - 1/F) / (F' - |a2|) for F >= 1 (>= 1 for F <= 1) and
//    w_z <= F'/F + az, which gives one bound; elsewhere it is 0.  B is the
//    larger of that and one proved per call site by an interval search over
//    the body's single gradient d (fold3d_tables.cpp), less the same
//    relative 1e-3 margin.  The fall-back candidate from s1 alone is not
//    gated.
#pragma once
#include <cstdint>
#include <cstring>

namespace fold3d {

// Constants of one FoldEdge2Points call site (AN_ISO_1_OpenACC.c:59-114).
struct EdgeK {
    double ax, ay, az;  // drift arguments as passed
    double hx, hz;      // spacing arguments (dxx, dzz)
    double rhx;         // RN(1/hx)
    double g, rg;       // F*F - ay*ay and RN(1/g)
    double ga, rga;     // g - az*az and RN(1/ga)
    double K;           // fall-back increment g'/c' of :99-113 (when fb_ok)
    double B;           // body skipped when the time is <= min(s0, s1) + B (4. above)
    int early;          // ax > 0: return when s1 > s0 (:71)
    int fb_ok;          // fall-back defined: its q > 0 and c > 0
};

// Constants of one FoldSurf3Points call site (:119-175).
struct SurfK {
    double ax, ay;      // drift arguments (az, F, hz are common)
    double hx, hy;      // dxx, dyy as passed
    double rhx, rhy;
    int e1, e2;         // ax > 0, ay > 0 (early returns of :132)
    int nblock;         // ax*dzz + az*dxx > 0: nested edge skipped when s1 > s2 (:170)
    int pad_;
    double B;           // body skipped when the time is <= min(s0, s1, s2) + B (3. above)
    EdgeK nest;         // the nested FoldEdge2Points call (:172-173)
};

// All constants of one direction on one side of the source surface.
struct SideTable {
    double F, az, hz;
    double g, rg;       // F*F - az*az, RN(1/g)          (:147)
    double K1;          // 1-D candidate increment dzz*dzz/q (:225)
    int d1_ok;          // 1-D candidate defined (:219, :223)
    // the per-call flags below as bit masks, bit k for call k
    unsigned m_e1, m_e2, m_nblock;  // surf[k].e1, .e2, .nblock
    unsigned m_nest_early;          // surf[k].nest.early
    unsigned m_edge_early;          // edge[k].early
    SurfK surf[8];      // the eight FoldSurf3Points calls (:233-240), in order
    EdgeK edge[8];      // the eight FoldEdge2Points calls (:242-253), in order
};

struct DirTable {
    SideTable side[2];  // [0]: target >= 0 (or 0), [1]: target < 0 (drift negated)
};

// Safe operand range of div_by_const: |x| and |c| in [2^-400, 2^401), which
// keeps the quotient, the products and the remainders normal.  The host
// stores r = 0 for a constant outside that range.
constexpr unsigned kDivExpLo = 1023 - 400;
constexpr unsigned kDivExpSpan = 800;

#ifdef __CUDACC__
// The functions below also compile for the host (IEEE double, fma, sqrt and
// division correctly rounded on both sides, no contraction), where a test
// runs them against the CPU statement of the reference.
__host__ __device__ __forceinline__ unsigned hi_word(double x)
{
#ifdef __CUDA_ARCH__
    return (unsigned)__double2hiint(x);
#else
    uint64_t b;
    std::memcpy(&b, &x, sizeof b);
    return (unsigned)(b >> 32);
#endif
}

// Correctly rounded x / c for a constant c given r = RN(1/c) (r == 0: use
// the IEEE division); see above.  Operands outside the safe range, zero
// included, also take the IEEE division.
__host__ __device__ __forceinline__ double div_by_const(double x, double c, double r)
{
    const unsigned ex = (hi_word(x) >> 20) & 0x7ffu;
    if (ex - kDivExpLo > kDivExpSpan || r == 0.0) return x / c;
    double q = x * r;
    double e = fma(-q, c, x);
    q = fma(e, r, q);
    e = fma(-q, c, x);
    return fma(e, r, q);
}

__host__ __device__ __forceinline__ double kmin(double a, double b) { return (a < b) ? a : b; }

__host__ __device__ __forceinline__ void edge_k(double &tn, double s0, double s1, const EdgeK &k, double F)
{
    const double mn = kmin(s1, s0);
    if (tn < mn || (k.early && s1 > s0)) return;
    if (!(tn <= mn + k.B)) {  // 4. above
        const double d = div_by_const(s1 - s0, k.hx, k.rhx);
        double c = (1.0 - d * k.ax);
        double q = k.g * (c * c - d * d * k.ga);
        if (0.0 < q) {
            c = div_by_const(-k.az * c + sqrt(q), k.ga, k.rga);
            q = s0 + k.hz * c;
            if (q < tn && q > mn) {
                const double g = sqrt(div_by_const((d * d + c * c) * F * F, k.g, k.rg));
                const double xe = -k.hz * (d + k.ax * g) / (c + k.az * g);
                if (0.0 < xe && xe < k.hx) tn = q;
            }
        }
    }
    if (tn > s1 && k.fb_ok) tn = kmin(tn, s1 + k.K);
}

__host__ __device__ __forceinline__ void surf_k(double &tn, double s0, double s1, double s2, const SurfK &k,
                                                const SideTable &t)
{
    const double mn = kmin(s0, kmin(s1, s2));
    if (tn < mn || (k.e1 && s1 > s0) || (k.e2 && s2 > s1)) return;
    if (!(tn <= mn + k.B)) {  // 3. above
        const double dx = div_by_const(s1 - s0, k.hx, k.rhx);
        const double dy = div_by_const(s2 - s1, k.hy, k.rhy);
        double dd = dx * dx + dy * dy;
        double al = 1.0 - k.ax * dx - k.ay * dy;
        double q = al * al - dd * t.g;
        if (q > 0.0) {
            al = div_by_const(-t.az * al + t.F * sqrt(q), t.g, t.rg);
            const double g = s0 + t.hz * al;
            if (g < tn && g > mn) {
                q = sqrt(dd + al * al);
                dd = -t.hz / (t.F * al + t.az * q);
                const double xe = dd * (t.F * dx + k.ax * q);
                const double ye = dd * (t.F * dy + k.ay * q);
                if (0.0 <= kmin(xe, ye) && ye * k.hx <= xe * k.hy && xe <= k.hx) tn = g;
            }
        }
    }
    if (tn > kmin(s1, s2) && !(k.nblock && s1 > s2)) edge_k(tn, s1, s2, k.nest, t.F);
}

// New signed value of a target whose stored value is `told`, from the nine
// previous-plane magnitudes (named as in the reference, :195-204).
__host__ __device__ __forceinline__ double point_update_fast(double told, double st, double xt, double yt,
                                                             double xnt, double ynt, double txy, double txm,
                                                             double tym, double txnyn, const DirTable *tab)
{
    double tn = fabs(told);
    const SideTable &t = tab->side[told < 0 ? 1 : 0];
    if (st < tn && t.d1_ok) tn = kmin(tn, st + t.K1);
    if (!(tn < st && tn < kmin(xt, yt) && tn < kmin(txy, txm) && tn < kmin(txnyn, tym))) {
#pragma unroll 1
        for (int k = 0; k < 8; ++k) {
            // (xt,txy) (xt,txm) (xnt,txnyn) (xnt,tym) (ynt,txnyn) (ynt,txm) (yt,txy) (yt,tym)
            const double s1 = (k < 2) ? xt : (k < 4) ? xnt : (k < 6) ? ynt : yt;
            const int m = k & 3;
            const double s2 = (m == 0) ? ((k < 4) ? txy : txnyn)
                            : (m == 1) ? txm
                            : (m == 2) ? ((k < 4) ? txnyn : txy)
                                       : tym;
            surf_k(tn, st, s1, s2, t.surf[k], t);
        }
#pragma unroll 1
        for (int k = 0; k < 8; ++k) {
            // xt, txy, yt, tym, xnt, txnyn, ynt, txm
            const double s1 = (k == 0) ? xt : (k == 1) ? txy : (k == 2) ? yt : (k == 3) ? tym
                            : (k == 4) ? xnt : (k == 5) ? txnyn : (k == 6) ? ynt : txm;
            edge_k(tn, st, s1, t.edge[k], t.F);
        }
    }
    return ((told > 0) ? 1.0 : -1.0) * tn;
}

// ---------------------------------------------------------------------------
// Candidate values for the compacted kernel.  Each function returns the
// smallest candidate its reference call would accept when entered with the
// current time `th` -- or +infinity -- instead of updating a running time.
// Every value returned is below th, so folding them with min gives the same
// result as the reference's sequence of calls (see the header comment).  The
// caller has already applied the call's entry gates.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double edge_cand(double th, double s0, double s1, const EdgeK &k, double F)
{
    double best = th;
    const double d = div_by_const(s1 - s0, k.hx, k.rhx);
    double c = (1.0 - d * k.ax);
    double q = k.g * (c * c - d * d * k.ga);
    if (0.0 < q) {
        c = div_by_const(-k.az * c + sqrt(q), k.ga, k.rga);
        q = s0 + k.hz * c;
        if (q < best && q > kmin(s0, s1)) {
            const double g = sqrt(div_by_const((d * d + c * c) * F * F, k.g, k.rg));
            const double xe = -k.hz * (d + k.ax * g) / (c + k.az * g);
            if (0.0 < xe && xe < k.hx) best = q;
        }
    }
    if (best > s1 && k.fb_ok) best = kmin(best, s1 + k.K);
    return best;
}

__device__ __forceinline__ double surf_cand(double th, double s0, double s1, double s2, const SurfK &k,
                                            const SideTable &t)
{
    double best = th;
    const double dx = div_by_const(s1 - s0, k.hx, k.rhx);
    const double dy = div_by_const(s2 - s1, k.hy, k.rhy);
    double dd = dx * dx + dy * dy;
    double al = 1.0 - k.ax * dx - k.ay * dy;
    double q = al * al - dd * t.g;
    if (q > 0.0) {
        al = div_by_const(-t.az * al + t.F * sqrt(q), t.g, t.rg);
        const double g = s0 + t.hz * al;
        if (g < best && g > kmin(kmin(s0, s1), s2)) {
            q = sqrt(dd + al * al);
            dd = -t.hz / (t.F * al + t.az * q);
            const double xe = dd * (t.F * dx + k.ax * q);
            const double ye = dd * (t.F * dy + k.ay * q);
            if (0.0 <= kmin(xe, ye) && ye * k.hx <= xe * k.hy && xe <= k.hx) best = g;
        }
    }
    return best;
}
#endif  // __CUDACC__

}  // namespace fold3d
