// fold3d_solver.cuh -- the Fold3dPMM local upwind solver, device side.
//
// Every floating-point expression keeps the operand order of the reference
// (Stencil-OpenACC/AN_ISO_1_OpenACC.c:59-175, :195-326), and the translation
// units that include this header are compiled with --fmad=false, so that each
// add and multiply rounds on its own exactly as the reference's host build
// (-ffp-contract=off) does.  CUDA's double '/' and sqrt are IEEE correctly
// rounded.  Together this makes the GPU result bit-identical to the
// reference's.
//
// Structure of the update (used by the skipping and reordering logic in the
// kernels): every candidate a solver can accept is strictly greater than the
// minimum of the previous-plane values it is built from, and every early
// return only fires when no candidate could beat the current time.  The
// result of a point update is therefore min(T_old, M(neighbours)), where
// M depends on the nine previous-plane values and on the side (sign) of the
// target only.
#pragma once
#include <cstdint>

namespace fold3d {

// The reference's fmin macro (AN_ISO_1_OpenACC.c:32-34): a plain ternary.
__device__ __forceinline__ double tmin(double a, double b) { return (a < b) ? a : b; }

// Local-frame constants of one sweep direction: speed, drift in the
// (local x, local y, normal) frame, spacings and diagonals.
struct LocalFrame {
    double F, ax, ay, az;
    double hz, hx, hy;       // normal, local x, local y spacing  (dzz, dxx, dyy)
    double hxy, hxz, hyz;    // diagonals                          (dxy, dxz, dyz)
};

// FoldEdge2Points, AN_ISO_1_OpenACC.c:59-114 (OPTTEST off).
__device__ __forceinline__ void edge2(double &tn, double s0, double s1, double F, double ax,
                                      double ay, double az, double hx, double hz)
{
    if (tn < tmin(s1, s0) || (ax > 0.0 && s1 > s0)) return;
    double g = F * F - ay * ay;
    double d = (s1 - s0) / hx;
    double c = (1.0 - d * ax);
    double q = g * (c * c - d * d * (g - az * az));
    if (0.0 < q) {
        c = (-az * c + sqrt(q)) / (g - az * az);
        q = s0 + hz * c;
        if (q < tn && q > tmin(s0, s1)) {
            g = sqrt((d * d + c * c) * F * F / g);
            double xe = -hz * (d + ax * g) / (c + az * g);
            if (0.0 < xe && xe < hx) tn = q;
        }
    }
    if (tn > s1) {
        c = (-hx * ax + hz * az);
        g = hx * hx + hz * hz;
        q = (F * F - ax * ax - ay * ay - az * az) * g + c * c;
        if (q > 0.0) {
            c = c + sqrt(q);
            if (c > 0.0) tn = tmin(tn, s1 + g / c);
        }
    }
}

// FoldSurf3Points, AN_ISO_1_OpenACC.c:119-175 (UNROLLED on, OPTTEST off).
__device__ __forceinline__ void surf3(double &tn, double s0, double s1, double s2, double F,
                                      double ax, double ay, double az, double hx, double hy,
                                      double hz, double hxz)
{
    if (tn < tmin(s0, tmin(s1, s2)) || (ax > 0.0 && s1 > s0) || (ay > 0.0 && s2 > s1)) return;
    double dx = (s1 - s0) / hx;
    double dy = (s2 - s1) / hy;
    double dd = dx * dx + dy * dy;
    double g = F * F - az * az;
    double al = 1.0 - ax * dx - ay * dy;
    double q = al * al - dd * g;
    if (q > 0.0) {
        al = (-az * al + F * sqrt(q)) / g;
        g = s0 + hz * al;
        if (g < tn && g > tmin(tmin(s0, s1), s2)) {
            q = sqrt(dd + al * al);
            dd = -hz / (F * al + az * q);
            double xe = dd * (F * dx + ax * q);
            double ye = dd * (F * dy + ay * q);
            if (0.0 <= tmin(xe, ye) && ye * hx <= xe * hy && xe <= hx) tn = g;
        }
    }
    if (tn > tmin(s1, s2) && (!(ax * hz + az * hx > 0.0 && s1 > s2)))
        edge2(tn, s1, s2, F, ay, (ax * hz + az * hx) / hxz, (-ax * hx + az * hz) / hxz, hy, hxz);
}

// The nine previous-plane magnitudes around a target point, named as in the
// reference (:195-204): xt/yt local +x/+y, xnt/ynt -x/-y, txy = +x+y,
// txm = +x-y, tym = -x+y, txnyn = -x-y.
struct Stencil9 {
    double st, xt, yt, xnt, ynt, txy, txm, tym, txnyn;
};

// Point update (:206-326): returns the new signed value of a target whose
// stored value is `told`.
__device__ __forceinline__ double point_update(double told, const Stencil9 &s, const LocalFrame &L)
{
    double tnew = fabs(told);
    double ax = L.ax, ay = L.ay, az = L.az;
    const double F = L.F, hz = L.hz, hx = L.hx, hy = L.hy;
    if (told < 0) {  // negative side: reversed drift (:207-212)
        ax = -ax;
        ay = -ay;
        az = -az;
    }
    if (s.st < tnew) {  // 1-D normal candidate (:214-228)
        double q = (F * F - (ax * ax + ay * ay)) * hz * hz;
        if (q > 0.0) {
            q = az * hz + sqrt(q);
            if (q > 0.0) tnew = tmin(tnew, s.st + hz * hz / q);
        }
    }
    if (!(tnew < s.st && tnew < tmin(s.xt, s.yt) && tnew < tmin(s.txy, s.txm) &&
          tnew < tmin(s.txnyn, s.tym))) {
        const double hxy = L.hxy, hxz = L.hxz, hyz = L.hyz;
        surf3(tnew, s.st, s.xt, s.txy, F, ax, ay, az, hx, hy, hz, hxz);
        surf3(tnew, s.st, s.xt, s.txm, F, ax, -ay, az, hx, hy, hz, hxz);
        surf3(tnew, s.st, s.xnt, s.txnyn, F, -ax, -ay, az, hx, hy, hz, hxz);
        surf3(tnew, s.st, s.xnt, s.tym, F, -ax, ay, az, hx, hy, hz, hxz);
        surf3(tnew, s.st, s.ynt, s.txnyn, F, -ay, -ax, az, hy, hx, hz, hyz);
        surf3(tnew, s.st, s.ynt, s.txm, F, -ay, ax, az, hy, hx, hz, hyz);
        surf3(tnew, s.st, s.yt, s.txy, F, ay, ax, az, hy, hx, hz, hyz);
        surf3(tnew, s.st, s.yt, s.tym, F, ay, -ax, az, hy, hx, hz, hyz);

        edge2(tnew, s.st, s.xt, F, ax, ay, az, hx, hz);
        edge2(tnew, s.st, s.txy, F, (ax * hx + ay * hy) / hxy, (-ax * hy + ay * hx) / hxy, az, hxy, hz);
        edge2(tnew, s.st, s.yt, F, ay, ax, az, hy, hz);
        edge2(tnew, s.st, s.tym, F, -(ax * hx - ay * hy) / hxy, (ax * hy + ay * hx) / hxy, az, hxy, hz);
        edge2(tnew, s.st, s.xnt, F, -ax, ay, az, hx, hz);
        edge2(tnew, s.st, s.txnyn, F, -(ax * hx + ay * hy) / hxy, (-ax * hy + ay * hx) / hxy, az, hxy, hz);
        edge2(tnew, s.st, s.ynt, F, -ay, ax, az, hy, hz);
        edge2(tnew, s.st, s.txm, F, (ax * hx - ay * hy) / hxy, (ax * hy + ay * hx) / hxy, az, hxy, hz);
    }
    return ((told > 0) ? 1.0 : -1.0) * tnew;  // sign(T) maps 0 to -1 (:36-38, :326)
}

}  // namespace fold3d
