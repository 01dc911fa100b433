// Closed-form 2D boundary entities of constrained DOFs (host + device, fp64),
// with the reference's geometry (src/geometry.hpp):
//   LineSeg   (sx, sy, ex, ey)  projection clamped to the segment   :288-316
//   LineRail  (sx, sy, ex, ey)  open-ended: identity beyond its ends :322-360
//   Circle    (cx, cy, r)       radial projection                   :398-430
//   Ellipse   (cx, cy, rx, ry)  radial-scaling projection           :432-472
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

// Projection of (px, py) onto the entity.
EGG_HD void entity_project(int tag, const double* e, double px, double py, double& qx, double& qy)
{
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

// Tags this core relaxes (2D closed-form curves).
EGG_HD bool entity_supported(int dim, int tag)
{
    return dim == 2 && (tag == EGG_B200_TAG_LINESEG || tag == EGG_B200_TAG_CIRCLE ||
                        tag == EGG_B200_TAG_ELLIPSE || tag == EGG_B200_TAG_LINERAIL);
}

}  // namespace egg_b200
