// fold3d_tables.cpp -- host evaluation of the per-direction constants of the
// local solver (see fold3d_fast.cuh).
//
// Every constant is computed with the expression the reference evaluates
// inside its sweep (Stencil-OpenACC/AN_ISO_1_OpenACC.c), with the drift of
// the side the table is for, in IEEE double with no FMA contraction
// (-ffp-contract=off), so the kernel obtains exactly the bits the reference
// computes point by point.
#include <cmath>
#include <cstring>

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

// FoldEdge2Points call with arguments (F, ax, ay, az, dxx=hx, dzz=hz),
// AN_ISO_1_OpenACC.c:59-114.
EdgeK edge_consts(double F, double ax, double ay, double az, double hx, double hz)
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
    k.B = edge_skip_bound(F, ax, ay, az, hz);
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
SurfK surf_consts(double F, double ax, double ay, double az, double hx, double hy, double hz, double hxz)
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
    k.nest = edge_consts(F, ay, (ax * hz + az * hx) / hxz, (-ax * hx + az * hz) / hxz, hy, hxz);  // :172-173
    return k;
}

void side_table(const LocalFrameH &L, bool negative, SideTable &t)
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
    t.Bs = surf_skip_bound(F, ax, ay, az, hz);
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
    t.surf[0] = surf_consts(F, ax, ay, az, hx, hy, hz, hxz);
    t.surf[1] = surf_consts(F, ax, -ay, az, hx, hy, hz, hxz);
    t.surf[2] = surf_consts(F, -ax, -ay, az, hx, hy, hz, hxz);
    t.surf[3] = surf_consts(F, -ax, ay, az, hx, hy, hz, hxz);
    t.surf[4] = surf_consts(F, -ay, -ax, az, hy, hx, hz, hyz);
    t.surf[5] = surf_consts(F, -ay, ax, az, hy, hx, hz, hyz);
    t.surf[6] = surf_consts(F, ay, ax, az, hy, hx, hz, hyz);
    t.surf[7] = surf_consts(F, ay, -ax, az, hy, hx, hz, hyz);
    // the eight FoldEdge2Points calls, :242-253
    t.edge[0] = edge_consts(F, ax, ay, az, hx, hz);
    t.edge[1] = edge_consts(F, (ax * hx + ay * hy) / hxy, (-ax * hy + ay * hx) / hxy, az, hxy, hz);
    t.edge[2] = edge_consts(F, ay, ax, az, hy, hz);
    t.edge[3] = edge_consts(F, -(ax * hx - ay * hy) / hxy, (ax * hy + ay * hx) / hxy, az, hxy, hz);
    t.edge[4] = edge_consts(F, -ax, ay, az, hx, hz);
    t.edge[5] = edge_consts(F, -(ax * hx + ay * hy) / hxy, (-ax * hy + ay * hx) / hxy, az, hxy, hz);
    t.edge[6] = edge_consts(F, -ay, ax, az, hy, hz);
    t.edge[7] = edge_consts(F, (ax * hx - ay * hy) / hxy, (ax * hy + ay * hx) / hxy, az, hxy, hz);
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

void build_dir_table(const LocalFrameH &L, DirTable &out)
{
    side_table(L, false, out.side[0]);
    side_table(L, true, out.side[1]);
}

}  // namespace fold3d
