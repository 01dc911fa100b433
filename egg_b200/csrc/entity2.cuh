// Closed-form 2D boundary entities of constrained DOFs (host + device, fp64),
// with the reference's geometry (src/geometry.hpp):
//   LineSeg   (sx, sy, ex, ey)  projection clamped to the segment   :288-316
//   LineRail  (sx, sy, ex, ey)  open-ended: identity beyond its ends :322-360
//   Circle    (cx, cy, r)       radial projection                   :398-430
//   Ellipse   (cx, cy, rx, ry)  radial-scaling projection           :432-472
//   CircleArc (cx, cy, r, t0, t1, closed)  trimmed arc: angle foot,
//             period re-representation, trim clamp       :129-140,195-229,562-579
// and the tangent-reduced Newton step of a curve DOF (tangent dimension 1):
// M = b^T H b, r = b^T g, y = solve1x1(M, r), delta = b y
// (src/patch.hpp:355-413 newton_step_from_basis / newton_delta,
// src/solve.hpp:83-90 solve1x1).  A rail whose foot lies outside [0, 1]
// releases its node: the full 2x2 step, as a free DOF.
#pragma once

#include "egg_b200.h"
#include "metric.cuh"

namespace egg_b200
{

constexpr double kGeomTiny = 1e-30;   // denominator floor (src/core.hpp:46)
constexpr double kGeomZnorm = 1e-15;  // zero-vector guard (src/core.hpp:47)

// Unclamped foot parameter of (px, py) on the line through the record's
// segment (sx, sy) -> (ex, ey).
EGG_HD double seg_foot(const double* e, double px, double py)
{
    const double abx = e[2] - e[0], aby = e[3] - e[1];
    const double ab_sq = abx * abx + aby * aby;
    return ((px - e[0]) * abx + (py - e[1]) * aby) / fmax(ab_sq, kGeomTiny);
}

// ---- trimmed circular arc, record (cx, cy, r, t0, t1, closed) ---------------
constexpr double kArcPeriod = 6.283185307179586;  // 2 pi, the angle's period

// Wrap x into [a, b) (a closed arc); unchanged when b <= a.
EGG_HD double arc_wrap(double x, double a, double b)
{
    const double L = b - a;
    if (L <= 0.0) { return x; }
    double t = fmod(x - a, L);
    if (t < 0.0) { t += L; }
    return a + t;
}

EGG_HD bool arc_contains(const double* e, double q) { return e[5] != 0.0 || (q >= e[3] && q <= e[4]); }

EGG_HD double arc_clamp(const double* e, double q)
{
    if (e[5] != 0.0) { return arc_wrap(q, e[3], e[4]); }
    return q < e[3] ? e[3] : (q > e[4] ? e[4] : q);
}

// Raw foot angle of (px, py): one branch representative.
EGG_HD double arc_invert(const double* e, double px, double py) { return atan2(py - e[1], px - e[0]); }

EGG_HD void arc_eval(const double* e, double q, double& x, double& y)
{
    x = e[0] + e[2] * cos(q);
    y = e[1] + e[2] * sin(q);
}

// Raw tangent column r (-sin q, cos q).
EGG_HD void arc_frame(const double* e, double q, double& jx, double& jy)
{
    jx = -e[2] * sin(q);
    jy = e[2] * cos(q);
}

// Unit vector (1/n) v, or e_0 below the zero-vector guard.
EGG_HD void unit_or_e0(double vx, double vy, double& ux, double& uy)
{
    const double n = sqrt(vx * vx + vy * vy);
    if (n < kGeomZnorm) {
        ux = 1.0;
        uy = 0.0;
        return;
    }
    const double inv = 1.0 / n;
    ux = inv * vx;
    uy = inv * vy;
}

// Cold foot: the representative nearest the trim interval (open arcs), then
// clamped onto it.
EGG_HD double arc_cold_foot(const double* e, double px, double py)
{
    double q = arc_invert(e, px, py);
    if (e[5] == 0.0) {
        const double mid = 0.5 * (e[3] + e[4]);
        q = mid + remainder(q - mid, kArcPeriod);
    }
    if (!arc_contains(e, q)) { q = arc_clamp(e, q); }
    return q;
}

// Warm step of an arc DOF (sweeps after the first of a run call): the Newton
// step on the tangent at the raw foot q*, reduced to an angle step
// dq = (J.J)^-1 J.delta and damped by omega; trials are q* + alpha dq,
// clamped onto the trim and evaluated.
EGG_HD void arc_warm_step(const double* e, const double H[4], const double g[2], double px, double py, double omega,
                          double& qstar, double& dq)
{
    qstar = arc_invert(e, px, py);
    double jx, jy, bx, by;
    arc_frame(e, qstar, jx, jy);
    unit_or_e0(jx, jy, bx, by);
    const double hb0 = H[0] * bx + H[1] * by;
    const double hb1 = H[2] * bx + H[3] * by;
    const double M = bx * hb0 + by * hb1;
    const double r = bx * g[0] + by * g[1];
    double y = 0.0;
    const double rn = fabs(r);
    if (!(rn < kGeomZnorm)) {
        y = -r / M;
        if (!isfinite(y)) { y = -0.1 * r / rn; }
    }
    const double dx = bx * y, dy = by * y;
    const double jtj = jx * jx + jy * jy;
    const double jtd = jx * dx + jy * dy;
    dq = (fabs(jtj) > kGeomTiny) ? jtd / jtj : 0.0;
    dq *= omega;
}

// Projection of (px, py) onto the entity.
EGG_HD void entity_project(int tag, const double* e, double px, double py, double& qx, double& qy)
{
    if (tag == EGG_B200_TAG_CIRCLEARC) {
        arc_eval(e, arc_cold_foot(e, px, py), qx, qy);
        return;
    }
    if (tag == EGG_B200_TAG_LINESEG || tag == EGG_B200_TAG_LINERAIL) {
        double t = seg_foot(e, px, py);
        if (tag == EGG_B200_TAG_LINERAIL) {
            if (t < 0.0 || t > 1.0) {  // beyond an end: released
                qx = px;
                qy = py;
                return;
            }
            qx = e[0] + t * (e[2] - e[0]);
            qy = e[1] + t * (e[3] - e[1]);
            return;
        }
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        qx = e[0] + t * (e[2] - e[0]);
        qy = e[1] + t * (e[3] - e[1]);
        return;
    }
    const double dx = px - e[0], dy = py - e[1];
    if (tag == EGG_B200_TAG_CIRCLE) {
        const double dist = sqrt(dx * dx + dy * dy);
        if (dist < kGeomZnorm) {  // any point of the circle
            qx = e[0] + e[2];
            qy = e[1];
            return;
        }
        qx = e[0] + e[2] * dx / dist;
        qy = e[1] + e[2] * dy / dist;
        return;
    }
    // ellipse
    const double sx = dx / e[2], sy = dy / e[3];
    const double dist = sqrt(sx * sx + sy * sy);
    double ux, uy;
    if (dist < kGeomZnorm) {
        ux = uy = 1.0 / 1.4142135623730951;  // (1, 1) / sqrt(2), as the double quotient
    } else {
        ux = sx / dist;
        uy = sy / dist;
    }
    qx = e[0] + ux * e[2];
    qy = e[1] + uy * e[3];
}

// Unit tangent of the entity at (px, py).
EGG_HD void entity_tangent(int tag, const double* e, double px, double py, double& tx, double& ty)
{
    if (tag == EGG_B200_TAG_CIRCLEARC) {  // at the cold foot
        double jx, jy;
        arc_frame(e, arc_cold_foot(e, px, py), jx, jy);
        unit_or_e0(jx, jy, tx, ty);
        return;
    }
    if (tag == EGG_B200_TAG_LINESEG || tag == EGG_B200_TAG_LINERAIL) {
        const double abx = e[2] - e[0], aby = e[3] - e[1];
        const double norm = sqrt(abx * abx + aby * aby);
        if (norm < kGeomZnorm) {
            tx = 1.0;
            ty = 0.0;
            return;
        }
        tx = abx / norm;
        ty = aby / norm;
        return;
    }
    const double dx = px - e[0], dy = py - e[1];
    if (tag == EGG_B200_TAG_CIRCLE) {
        const double rn = sqrt(dx * dx + dy * dy);
        double nx = 1.0, ny = 0.0;
        if (!(rn < kGeomZnorm)) {
            nx = dx / rn;
            ny = dy / rn;
        }
        tx = -ny;
        ty = nx;
        return;
    }
    // ellipse: parametric angle of the radially scaled point
    const double ang = atan2(dy / e[3], dx / e[2]);
    const double ax = -e[2] * sin(ang), ay = e[3] * cos(ang);
    const double norm = sqrt(ax * ax + ay * ay);
    if (norm < kGeomZnorm) {
        tx = 1.0;
        ty = 0.0;
        return;
    }
    tx = ax / norm;
    ty = ay / norm;
}

// Newton step of a constrained DOF at pos from its patch gradient g and
// Hessian H (row-major 2x2).
EGG_HD void entity_newton_step(int tag, const double* e, const double H[4], const double g[2], double px,
                               double py, double out[2])
{
    if (tag == EGG_B200_TAG_LINERAIL) {
        const double t = seg_foot(e, px, py);
        if (t < 0.0 || t > 1.0) {  // released: the full-space step
            solve2<double>(H, g, out);
            return;
        }
    }
    double bx, by;
    entity_tangent(tag, e, px, py, bx, by);
    const double hb0 = H[0] * bx + H[1] * by;
    const double hb1 = H[2] * bx + H[3] * by;
    const double M = bx * hb0 + by * hb1;
    const double r = bx * g[0] + by * g[1];
    double y = 0.0;
    const double rn = fabs(r);
    if (!(rn < kGeomZnorm)) {
        y = -r / M;
        if (!isfinite(y)) { y = -0.1 * r / rn; }
    }
    out[0] = bx * y;
    out[1] = by * y;
}

// Tags this core relaxes in dimension dim.
EGG_HD bool entity_supported(int dim, int tag)
{
    if (dim == 3) { return tag == EGG_B200_TAG_PLANE || tag == EGG_B200_TAG_LINERAIL3; }
    return dim == 2 && (tag == EGG_B200_TAG_LINESEG || tag == EGG_B200_TAG_CIRCLE ||
                        tag == EGG_B200_TAG_ELLIPSE || tag == EGG_B200_TAG_LINERAIL ||
                        tag == EGG_B200_TAG_CIRCLEARC);
}

}  // namespace egg_b200
