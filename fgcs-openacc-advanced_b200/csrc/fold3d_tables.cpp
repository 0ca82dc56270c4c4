// fold3d_tables.cpp -- host evaluation of the per-direction constants of the
// local solver (see fold3d_fast.cuh).
//
// Every constant is computed with the expression the reference evaluates
// inside its sweep (Stencil-OpenACC/AN_ISO_1_OpenACC.c), with the drift of
// the side the table is for, in IEEE double with no FMA contraction
// (-ffp-contract=off), so the kernel obtains exactly the bits the reference
// computes point by point.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <queue>
#include <vector>

#include "fold3d_fast.cuh"
#include "fold3d_internal.h"

namespace fold3d {

namespace {

// RN(1/c) when c and its reciprocal lie in div_by_const's safe range,
// otherwise 0 (the kernel then divides with the IEEE operation).
double safe_recip(double c)
{
    const double a = std::fabs(c);
    if (!(a >= std::ldexp(1.0, -400) && a < std::ldexp(1.0, 401))) return 0.0;
    return 1.0 / c;
}

// Skip bound of the FoldSurf3Points bodies of one side (fold3d_fast.cuh,
// 3.): dzz / (F + az) less a relative 1e-3, or 0 (no skipping beyond the
// reference's own gates) unless F^2 >= 1.1 |a|^2.
double surf_skip_bound(double F, double ax, double ay, double az, double dzz)
{
    const double a2 = ax * ax + ay * ay + az * az;
    if (!(F > 0.0 && dzz > 0.0 && F * F >= 1.1 * a2)) return 0.0;
    const double B = dzz / (F + az) * (1.0 - 1e-3);
    return (std::isfinite(B) && B > 0.0) ? B : 0.0;
}

// Skip bound of a FoldEdge2Points body with arguments (F, ax, ay, az, dxx,
// dzz) (fold3d_fast.cuh, 4.): dzz P / W less a relative 1e-3, with
// P = 1 - F'(1 - 1/F) / (F' - |a2|) (1 for F <= 1) and W = F'/F + az, where
// F' = sqrt(F^2 - ay^2) and a2 = (ax, az); 0 unless the conditions of 4. hold
// with some room: F^2 >= 1.1 |a|^2, |ax| < sqrt(ga) and F' > |a2| by 5%.
double edge_skip_bound(double F, double ax, double ay, double az, double dzz)
{
    const double Fp2 = F * F - ay * ay, ga = Fp2 - az * az;
    if (!(F > 0.0 && dzz > 0.0 && F * F >= 1.1 * (ax * ax + ay * ay + az * az) && ga > 0.0)) return 0.0;
    const double Fp = std::sqrt(Fp2), a2 = std::sqrt(ax * ax + az * az);
    if (!(std::fabs(ax) < 0.95 * std::sqrt(ga) && a2 < 0.95 * Fp)) return 0.0;
    if (!((F >= 1.0 && az >= 0.0) || (F <= 1.0 && az <= 0.0))) return 0.0;
    const double P = (F >= 1.0) ? 1.0 - Fp * (1.0 - 1.0 / F) / (Fp - a2) : 1.0;
    const double W = Fp / F + az;
    if (!(P > 0.0 && W > 0.0)) return 0.0;
    const double B = dzz * P / W * (1.0 - 1e-3);
    return (std::isfinite(B) && B > 0.0) ? B : 0.0;
}

// ---------------------------------------------------------------------------
// A proved lower bound on the accepted increment of one FoldEdge2Points call
// site, by interval branch and bound.  With d = (s1 - s0)/dxx the body
// computes c0 = 1 - d ax, Q = g (c0^2 - d^2 ga), c = (-az c0 + sqrt Q)/ga
// and accepts q = s0 + dzz c when Q > 0, q > min(s0, s1) and the footpoint
// xe = -dzz (d + ax G)/(c + az G), G = sqrt((d^2 + c^2) F^2 / g), lies in
// (0, dxx) (:71-95).  Its increment over min(s0, s1),
// D(d) = dzz c + max(0, -d dxx), depends on d alone, and d ranges over the
// bounded interval where Q > 0 when |ax| < sqrt(ga).  The search encloses D
// and the acceptance tests on sub-intervals of d in interval arithmetic
// rounded outwards, drops sub-intervals where no d can be accepted (Q <= 0,
// D <= 0, num * den >= 0 or dzz |num| >= dxx |den| for xe = -dzz num/den,
// the last also near the pole den = 0), splits the one with the smallest
// enclosure of D, and returns the smallest lower end left.  The constants are
// the table's own doubles; the kernel's rounding is covered by the caller's
// relative margin.
// ---------------------------------------------------------------------------
struct Iv {
    double lo, hi;
};
inline double rdn(double x) { return std::nextafter(x, -HUGE_VAL); }
inline double rup(double x) { return std::nextafter(x, HUGE_VAL); }
inline Iv ivp(double x) { return {x, x}; }
inline Iv iadd(Iv a, Iv b) { return {rdn(a.lo + b.lo), rup(a.hi + b.hi)}; }
inline Iv isub(Iv a, Iv b) { return {rdn(a.lo - b.hi), rup(a.hi - b.lo)}; }
inline Iv imul(Iv a, Iv b)
{
    const double p0 = a.lo * b.lo, p1 = a.lo * b.hi, p2 = a.hi * b.lo, p3 = a.hi * b.hi;
    return {rdn(std::min(std::min(p0, p1), std::min(p2, p3))), rup(std::max(std::max(p0, p1), std::max(p2, p3)))};
}
inline Iv isqr(Iv a)
{
    if (a.lo >= 0.0) return {rdn(a.lo * a.lo), rup(a.hi * a.hi)};
    if (a.hi <= 0.0) return {rdn(a.hi * a.hi), rup(a.lo * a.lo)};
    return {0.0, rup(std::max(a.lo * a.lo, a.hi * a.hi))};
}
inline Iv idivp(Iv a, double b) { return {rdn(a.lo / b), rup(a.hi / b)}; }  // b > 0
inline Iv isqrt(Iv a) { return {a.lo > 0.0 ? rdn(std::sqrt(a.lo)) : 0.0, a.hi > 0.0 ? rup(std::sqrt(a.hi)) : 0.0}; }
inline Iv iabs(Iv a)
{
    if (a.lo >= 0.0) return a;
    if (a.hi <= 0.0) return {-a.hi, -a.lo};
    return {0.0, std::max(-a.lo, a.hi)};
}

// Encloses D over the d in `d` when some of them may be accepted; false when
// none can be.
bool edge_increment(const EdgeK &k, double F, Iv d, Iv &D)
{
    const Iv c0 = isub(ivp(1.0), imul(d, ivp(k.ax)));
    const Iv Q = imul(ivp(k.g), isub(isqr(c0), imul(isqr(d), ivp(k.ga))));
    if (!(Q.hi > 0.0)) return false;
    const Iv c = idivp(iadd(imul(ivp(-k.az), c0), isqrt(Q)), k.ga);
    const Iv m = imul(d, ivp(-k.hx));
    D = iadd(imul(ivp(k.hz), c), Iv{std::max(0.0, m.lo), std::max(0.0, m.hi)});
    if (!(D.hi > 0.0)) return false;
    const Iv G = isqrt(idivp(imul(imul(iadd(isqr(d), isqr(c)), ivp(F)), ivp(F)), k.g));
    const Iv num = iadd(d, imul(ivp(k.ax), G)), den = iadd(c, imul(ivp(k.az), G));
    if (!(imul(num, den).lo < 0.0)) return false;  // xe > 0 needs num * den < 0
    return imul(ivp(k.hz), iabs(num)).lo < imul(ivp(k.hx), iabs(den)).hi;  // |xe| < dxx
}

// The increment the body accepts at one d, or +inf (double arithmetic; only
// used to stop the search once its bound is within 1% of it).
double edge_point(const EdgeK &k, double F, double d)
{
    const double c0 = 1.0 - d * k.ax, Q = k.g * (c0 * c0 - d * d * k.ga);
    if (!(Q > 0.0)) return HUGE_VAL;
    const double c = (-k.az * c0 + std::sqrt(Q)) / k.ga, D = k.hz * c - std::min(0.0, d * k.hx);
    if (!(D > 0.0)) return HUGE_VAL;
    const double G = std::sqrt((d * d + c * c) * F * F / k.g), xe = -k.hz * (d + k.ax * G) / (c + k.az * G);
    return (0.0 < xe && xe < k.hx) ? D : HUGE_VAL;
}

// The proved lower bound (0 when the search does not apply).
double edge_bb_search(const EdgeK &k, double F)
{
    if (!(k.g > 0.0 && k.ga > 0.0 && k.hx > 0.0 && k.hz > 0.0 && F > 0.0)) return 0.0;
    const double sga = std::sqrt(k.ga);
    if (!(std::fabs(k.ax) < 0.99 * sga)) return 0.0;
    // Q > 0 between the roots 1/(ax - sqrt ga) < 0 < 1/(ax + sqrt ga), widened
    double lo = 1.0 / (k.ax - sga) * (1.0 + 1e-9), hi = 1.0 / (k.ax + sga) * (1.0 + 1e-9);
    if (k.early) hi = 0.0;  // ax > 0: the body returns when s1 > s0, i.e. d > 0 (:71)
    if (!(lo < hi) || !std::isfinite(lo) || !std::isfinite(hi)) return 0.0;
    using Item = std::pair<double, Iv>;
    auto cmp = [](const Item &a, const Item &b) { return a.first > b.first; };
    std::priority_queue<Item, std::vector<Item>, decltype(cmp)> heap(cmp);
    Iv D;
    if (edge_increment(k, F, Iv{lo, hi}, D)) heap.push({D.lo, Iv{lo, hi}});
    const double min_width = (hi - lo) * 1e-12;
    double frozen = HUGE_VAL;  // sub-intervals too narrow to split
    double seen = HUGE_VAL;    // smallest increment accepted at a sampled point
    for (int it = 0; it < 2000 && !heap.empty(); ++it) {
        const Item top = heap.top();
        if (top.first >= 0.99 * seen) break;  // within 1%: the bound is tight enough
        heap.pop();
        const Iv x = top.second;
        const double mid = 0.5 * (x.lo + x.hi);
        seen = std::min(seen, edge_point(k, F, mid));
        if (!(x.hi - x.lo > min_width) || !(mid > x.lo && mid < x.hi)) {
            frozen = std::min(frozen, top.first);
            continue;
        }
        const Iv halves[2] = {{x.lo, mid}, {mid, x.hi}};
        for (const Iv &h : halves)
            if (edge_increment(k, F, h, D)) heap.push({D.lo, h});
    }
    double b = frozen;
    if (!heap.empty()) b = std::min(b, heap.top().first);
    if (b == HUGE_VAL) return 0.0;  // nothing can be accepted; 0 keeps the plain gates
    return std::max(b, 0.0);
}

// The same search for a FoldSurf3Points call site (drift arguments ax, ay;
// the side's F, az, dzz; spacings dxx, dyy), over the two gradients
// dx = (s1 - s0)/dxx, dy = (s2 - s1)/dyy.  The body (:131-165) computes
// al = 1 - ax dx - ay dy, q = al^2 - (dx^2 + dy^2) g with g = F^2 - az^2,
// al' = (-az al + F sqrt q)/g and accepts s0 + dzz al' when q > 0, it lies
// above min(s0, s1, s2) and its footpoint xe = -dzz nx/den,
// ye = -dzz ny/den (nx = F dx + ax r, ny = F dy + ay r, den = F al' + az r,
// r = sqrt(dx^2 + dy^2 + al'^2)) satisfies 0 <= min(xe, ye),
// ye dxx <= xe dyy and xe <= dxx.  Its increment over min(s0, s1, s2) is
// D = dzz al' - min(0, dx dxx, dx dxx + dy dyy).  The gradients range over
// the disc where q > 0, of radius 1/(sqrt g - |(ax, ay)|), and the early
// returns (:132) keep dx <= 0 when ax > 0 and dy <= 0 when ay > 0.
struct Box {
    Iv x, y;
};

bool surf_increment(double F, double az, double hz, double g, double ax, double ay, double hx, double hy, const Box &b,
                    Iv &D)
{
    const Iv dd = iadd(isqr(b.x), isqr(b.y));
    const Iv al = isub(isub(ivp(1.0), imul(ivp(ax), b.x)), imul(ivp(ay), b.y));
    const Iv q = isub(isqr(al), imul(dd, ivp(g)));
    if (!(q.hi > 0.0)) return false;
    const Iv al2 = idivp(iadd(imul(ivp(-az), al), imul(ivp(F), isqrt(q))), g);
    const Iv ux = imul(b.x, ivp(hx)), uxy = iadd(ux, imul(b.y, ivp(hy)));
    const Iv mn = {std::min(0.0, std::min(ux.lo, uxy.lo)), std::min(0.0, std::min(ux.hi, uxy.hi))};
    D = isub(imul(ivp(hz), al2), mn);
    if (!(D.hi > 0.0)) return false;
    const Iv r = isqrt(iadd(dd, isqr(al2)));
    const Iv den = iadd(imul(ivp(F), al2), imul(ivp(az), r));
    const Iv nx = iadd(imul(ivp(F), b.x), imul(ivp(ax), r)), ny = iadd(imul(ivp(F), b.y), imul(ivp(ay), r));
    if (imul(nx, den).lo > 0.0 || imul(ny, den).lo > 0.0) return false;  // xe >= 0 and ye >= 0 need <= 0
    const Iv ad = iabs(den);
    if (imul(ivp(hz), iabs(nx)).lo > imul(ivp(hx), ad).hi) return false;  // |xe| <= dxx
    if (imul(ivp(hz), iabs(ny)).lo > imul(ivp(hy), ad).hi) return false;  // |ye| <= dyy (implied by the two tests)
    // ye dxx <= xe dyy:  -dzz (ny dxx - nx dyy) / den <= 0, i.e. den (ny dxx - nx dyy) >= 0
    if (imul(den, isub(imul(ny, ivp(hx)), imul(nx, ivp(hy)))).hi < 0.0) return false;
    return true;
}

// The increment the body accepts at one (dx, dy), or +inf (double
// arithmetic; only used to stop the search).
double surf_point(double F, double az, double hz, double g, double ax, double ay, double hx, double hy, double dx,
                  double dy)
{
    const double dd = dx * dx + dy * dy, al = 1.0 - ax * dx - ay * dy, q = al * al - dd * g;
    if (!(q > 0.0)) return HUGE_VAL;
    const double al2 = (-az * al + F * std::sqrt(q)) / g;
    const double D = hz * al2 - std::min(0.0, std::min(dx * hx, dx * hx + dy * hy));
    if (!(D > 0.0)) return HUGE_VAL;
    const double r = std::sqrt(dd + al2 * al2), m = -hz / (F * al2 + az * r);
    const double xe = m * (F * dx + ax * r), ye = m * (F * dy + ay * r);
    return (0.0 <= std::min(xe, ye) && ye * hx <= xe * hy && xe <= hx) ? D : HUGE_VAL;
}

double surf_bb_search(double F, double az, double hz, double ax, double ay, double hx, double hy)
{
    const double g = F * F - az * az;
    if (!(g > 0.0 && hx > 0.0 && hy > 0.0 && hz > 0.0 && F > 0.0)) return 0.0;
    const double ain = std::sqrt(ax * ax + ay * ay), sg = std::sqrt(g);
    if (!(ain < 0.99 * sg)) return 0.0;
    const double R = 1.0 / (sg - ain) * (1.0 + 1e-9);
    Box root{{-R, ax > 0.0 ? 0.0 : R}, {-R, ay > 0.0 ? 0.0 : R}};
    using Item = std::pair<double, Box>;
    auto cmp = [](const Item &a, const Item &b) { return a.first > b.first; };
    std::priority_queue<Item, std::vector<Item>, decltype(cmp)> heap(cmp);
    Iv D;
    if (surf_increment(F, az, hz, g, ax, ay, hx, hy, root, D)) heap.push({D.lo, root});
    const double min_width = R * 1e-12;
    double frozen = HUGE_VAL;
    double seen = HUGE_VAL;
    for (int it = 0; it < 6000 && !heap.empty(); ++it) {
        const Item top = heap.top();
        if (top.first >= 0.99 * seen) break;
        heap.pop();
        const Box b = top.second;
        seen = std::min(seen, surf_point(F, az, hz, g, ax, ay, hx, hy, 0.5 * (b.x.lo + b.x.hi), 0.5 * (b.y.lo + b.y.hi)));
        const bool along_x = (b.x.hi - b.x.lo) >= (b.y.hi - b.y.lo);
        const Iv w = along_x ? b.x : b.y;
        const double mid = 0.5 * (w.lo + w.hi);
        if (!(w.hi - w.lo > min_width) || !(mid > w.lo && mid < w.hi)) {
            frozen = std::min(frozen, top.first);
            continue;
        }
        Box h0 = b, h1 = b;
        if (along_x) {
            h0.x.hi = mid;
            h1.x.lo = mid;
        } else {
            h0.y.hi = mid;
            h1.y.lo = mid;
        }
        for (const Box &h : {h0, h1})
            if (surf_increment(F, az, hz, g, ax, ay, hx, hy, h, D)) heap.push({D.lo, h});
    }
    double bound = frozen;
    if (!heap.empty()) bound = std::min(bound, heap.top().first);
    if (bound == HUGE_VAL) return 0.0;
    return std::max(bound, 0.0);
}

// The searches run inside the C entry points: an allocation failure there
// gives the bound 0, which skips nothing and is always valid.
double edge_bb_bound(const EdgeK &k, double F)
{
    try {
        return edge_bb_search(k, F);
    } catch (...) {
        return 0.0;
    }
}

double surf_bb_bound(double F, double az, double hz, double ax, double ay, double hx, double hy)
{
    try {
        return surf_bb_search(F, az, hz, ax, ay, hx, hy);
    } catch (...) {
        return 0.0;
    }
}

// FoldEdge2Points call with arguments (F, ax, ay, az, dxx=hx, dzz=hz),
// AN_ISO_1_OpenACC.c:59-114.
EdgeK edge_consts(double F, double ax, double ay, double az, double hx, double hz, bool search)
{
    EdgeK k;
    std::memset(&k, 0, sizeof k);
    k.ax = ax;
    k.ay = ay;
    k.az = az;
    k.hx = hx;
    k.hz = hz;
    k.rhx = safe_recip(hx);
    k.g = F * F - ay * ay;     // :77
    k.rg = safe_recip(k.g);
    k.ga = k.g - az * az;      // :80, :83
    k.rga = safe_recip(k.ga);
    k.early = (ax > 0.0);      // :71
    // the larger of two proved lower bounds, less the relative margin
    k.B = edge_skip_bound(F, ax, ay, az, hz);
    if (search && F * F >= 1.1 * (ax * ax + ay * ay + az * az)) {
        const double bb = edge_bb_bound(k, F) * (1.0 - 1e-3);
        if (std::isfinite(bb) && bb > k.B) k.B = bb;
    }
    // fall-back candidate from xt alone, :99-113, up to the final addition
    double c = (-hx * ax + hz * az);
    const double g = hx * hx + hz * hz;
    double q = (F * F - ax * ax - ay * ay - az * az) * g + c * c;
    k.fb_ok = 0;
    k.K = 0.0;
    if (q > 0.0) {
        c = c + std::sqrt(q);
        if (c > 0.0) {
            k.fb_ok = 1;
            k.K = g / c;
        }
    }
    return k;
}

// FoldSurf3Points call with drift arguments (ax, ay) and spacings
// (dxx=hx, dyy=hy, dxz=hxz); F, az, dzz are the direction's.  :119-175.
SurfK surf_consts(double F, double ax, double ay, double az, double hx, double hy, double hz, double hxz,
                  bool search)
{
    SurfK k;
    std::memset(&k, 0, sizeof k);
    k.ax = ax;
    k.ay = ay;
    k.hx = hx;
    k.hy = hy;
    k.rhx = safe_recip(hx);
    k.rhy = safe_recip(hy);
    k.e1 = (ax > 0.0);
    k.e2 = (ay > 0.0);
    k.nblock = (ax * hz + az * hx > 0.0);  // :170
    k.nest = edge_consts(F, ay, (ax * hz + az * hx) / hxz, (-ax * hx + az * hz) / hxz, hy, hxz, search);  // :172-173
    // body-skip bound (fold3d_fast.cuh, 3.): the larger of the physical bound
    // and the searched one, less the relative margin
    k.B = surf_skip_bound(F, ax, ay, az, hz);
    if (search && F * F >= 1.1 * (ax * ax + ay * ay + az * az)) {
        const double bb = surf_bb_bound(F, az, hz, ax, ay, hx, hy) * (1.0 - 1e-3);
        if (std::isfinite(bb) && bb > k.B) k.B = bb;
    }
    return k;
}

void side_table(const LocalFrameH &L, bool negative, bool search, SideTable &t)
{
    std::memset(&t, 0, sizeof t);
    const double F = L.F, hz = L.hz, hx = L.hx, hy = L.hy;
    const double hxy = L.hxy, hxz = L.hxz, hyz = L.hyz;
    double ax = L.ax, ay = L.ay, az = L.az;
    if (negative) {  // :207-212
        ax *= -1;
        ay *= -1;
        az *= -1;
    }
    t.F = F;
    t.az = az;
    t.hz = hz;
    t.g = F * F - az * az;  // :147
    t.rg = safe_recip(t.g);
    // 1-D normal candidate, :214-228, up to the final addition
    double q = (F * F - (ax * ax + ay * ay)) * hz * hz;
    t.d1_ok = 0;
    t.K1 = 0.0;
    if (q > 0.0) {
        q = az * hz + std::sqrt(q);
        if (q > 0.0) {
            t.d1_ok = 1;
            t.K1 = hz * hz / q;
        }
    }
    // the eight FoldSurf3Points calls, :233-240
    t.surf[0] = surf_consts(F, ax, ay, az, hx, hy, hz, hxz, search);
    t.surf[1] = surf_consts(F, ax, -ay, az, hx, hy, hz, hxz, search);
    t.surf[2] = surf_consts(F, -ax, -ay, az, hx, hy, hz, hxz, search);
    t.surf[3] = surf_consts(F, -ax, ay, az, hx, hy, hz, hxz, search);
    t.surf[4] = surf_consts(F, -ay, -ax, az, hy, hx, hz, hyz, search);
    t.surf[5] = surf_consts(F, -ay, ax, az, hy, hx, hz, hyz, search);
    t.surf[6] = surf_consts(F, ay, ax, az, hy, hx, hz, hyz, search);
    t.surf[7] = surf_consts(F, ay, -ax, az, hy, hx, hz, hyz, search);
    // the eight FoldEdge2Points calls, :242-253
    t.edge[0] = edge_consts(F, ax, ay, az, hx, hz, search);
    t.edge[1] = edge_consts(F, (ax * hx + ay * hy) / hxy, (-ax * hy + ay * hx) / hxy, az, hxy, hz, search);
    t.edge[2] = edge_consts(F, ay, ax, az, hy, hz, search);
    t.edge[3] = edge_consts(F, -(ax * hx - ay * hy) / hxy, (ax * hy + ay * hx) / hxy, az, hxy, hz, search);
    t.edge[4] = edge_consts(F, -ax, ay, az, hx, hz, search);
    t.edge[5] = edge_consts(F, -(ax * hx + ay * hy) / hxy, (-ax * hy + ay * hx) / hxy, az, hxy, hz, search);
    t.edge[6] = edge_consts(F, -ay, ax, az, hy, hz, search);
    t.edge[7] = edge_consts(F, (ax * hx - ay * hy) / hxy, (ax * hy + ay * hx) / hxy, az, hxy, hz, search);
    t.m_e1 = t.m_e2 = t.m_nblock = t.m_nest_early = t.m_edge_early = 0;
    for (int k = 0; k < 8; ++k) {
        t.m_e1 |= (unsigned)(t.surf[k].e1 != 0) << k;
        t.m_e2 |= (unsigned)(t.surf[k].e2 != 0) << k;
        t.m_nblock |= (unsigned)(t.surf[k].nblock != 0) << k;
        t.m_nest_early |= (unsigned)(t.surf[k].nest.early != 0) << k;
        t.m_edge_early |= (unsigned)(t.edge[k].early != 0) << k;
    }
}

}  // namespace

void build_dir_table(const LocalFrameH &L, DirTable &out, bool search)
{
    if (!search) {  // closed-form bounds only: nothing allocated
        side_table(L, false, false, out.side[0]);
        side_table(L, true, false, out.side[1]);
        return;
    }
    // The skip bounds take a search per call site; a solve asks for the same
    // six frames every sweep, so each thread keeps its last twelve tables.
    struct Entry {
        LocalFrameH key;
        DirTable tab;
        bool used;
    };
    constexpr int kEntries = 12;
    thread_local std::unique_ptr<Entry[]> memo;
    thread_local int next = 0;
    if (!memo) memo.reset(new (std::nothrow) Entry[kEntries]());  // stays empty if that fails
    if (memo)
        for (int i = 0; i < kEntries; ++i)
            if (memo[i].used && std::memcmp(&memo[i].key, &L, sizeof L) == 0) {
                out = memo[i].tab;
                return;
            }
    side_table(L, false, true, out.side[0]);
    side_table(L, true, true, out.side[1]);
    if (!memo) return;
    Entry &e = memo[next];
    next = (next + 1) % kEntries;
    e.key = L;
    e.tab = out;
    e.used = true;
}

}  // namespace fold3d
