// Closed-form 2D boundary entities of constrained DOFs (host + device, fp64),
// with the reference's geometry (src/geometry.hpp):
//   LineSeg   (sx, sy, ex, ey)  projection clamped to the segment   :288-316
//   LineRail  (sx, sy, ex, ey)  open-ended: identity beyond its ends :322-360
//   Circle    (cx, cy, r)       radial projection                   :398-430
//   Ellipse   (cx, cy, rx, ry)  radial-scaling projection           :432-472
//   trimmed curves (CircleArc, EllipseArc, QuadBezier, CubicBezier): foot,
//             period re-representation, trim clamp   :129-140,195-229,498-672
// and the tangent-reduced Newton step of a curve DOF (tangent dimension 1):
// M = b^T H b, r = b^T g, y = solve1x1(M, r), delta = b y
// (src/patch.hpp:355-413 newton_step_from_basis / newton_delta,
// src/solve.hpp:83-90 solve1x1).  A rail whose foot lies outside [0, 1]
// releases its node: the full 2x2 step, as a free DOF.
#pragma once

#include "egg_b200.h"
#include "metric.cuh"

// Out-of-line on the device: the iterative curve routines (grid + Newton
// feet, B-spline evaluation, composite search) are called from many sites and
// only for constrained DOFs, so inlining them would only grow the kernels.
#ifdef __CUDACC__
#define EGG_OUTLINE __host__ __device__ __noinline__
#else
#define EGG_OUTLINE inline
#endif

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

// ---- trimmed parametric curves -------------------------------------------
//   CircleArc    (cx, cy, r, t0, t1, closed)           foot: polar angle
//   EllipseArc   (cx, cy, a, b, phi, t0, t1, closed)    foot: grid + Newton on [0, 2 pi]
//   QuadBezier   (p0, p1, p2, t0, t1)                   foot: grid + Newton on [0, 1]
//   CubicBezier  (p0, p1, p2, p3, t0, t1)               foot: grid + Newton on [0, 1]
// (src/geometry.hpp:498-672, records :1929-2095).  The arcs' angle is
// periodic: the cold foot takes the representative nearest the trim.
constexpr double kArcPeriod = 6.283185307179586;  // 2 pi, the angle's period

EGG_HD bool is_tcurve(int tag)
{
    return tag == EGG_B200_TAG_CIRCLEARC || tag == EGG_B200_TAG_ELLIPSEARC || tag == EGG_B200_TAG_QUADBEZIER ||
           tag == EGG_B200_TAG_CUBICBEZIER;
}

// Trim (t0, t1, closed) of a curve record.
EGG_HD void tc_trim(int tag, const double* e, double& t0, double& t1, bool& closed)
{
    switch (tag) {
    case EGG_B200_TAG_CIRCLEARC: t0 = e[3], t1 = e[4], closed = e[5] != 0.0; return;
    case EGG_B200_TAG_ELLIPSEARC: t0 = e[5], t1 = e[6], closed = e[7] != 0.0; return;
    case EGG_B200_TAG_QUADBEZIER: t0 = e[6], t1 = e[7], closed = false; return;
    default: t0 = e[8], t1 = e[9], closed = false; return;
    }
}

// Wrap x into [a, b) (a closed curve); unchanged when b <= a.
EGG_HD double arc_wrap(double x, double a, double b)
{
    const double L = b - a;
    if (L <= 0.0) { return x; }
    double t = fmod(x - a, L);
    if (t < 0.0) { t += L; }
    return a + t;
}

EGG_HD bool tc_contains(int tag, const double* e, double q)
{
    double t0, t1;
    bool closed;
    tc_trim(tag, e, t0, t1, closed);
    return closed || (q >= t0 && q <= t1);
}

EGG_HD double tc_clamp(int tag, const double* e, double q)
{
    double t0, t1;
    bool closed;
    tc_trim(tag, e, t0, t1, closed);
    if (closed) { return arc_wrap(q, t0, t1); }
    return q < t0 ? t0 : (q > t1 ? t1 : q);
}

// Position (nd = 0), first (nd = 1) or second (nd = 2) derivative at t.
EGG_OUTLINE void tc_eval(int tag, const double* e, double t, int nd, double& x, double& y)
{
    if (tag == EGG_B200_TAG_CIRCLEARC) {
        const double c = cos(t), s = sin(t);
        if (nd == 0) {
            x = e[0] + e[2] * c;
            y = e[1] + e[2] * s;
        } else if (nd == 1) {
            x = -e[2] * s;
            y = e[2] * c;
        } else {
            x = -e[2] * c;
            y = -e[2] * s;
        }
        return;
    }
    if (tag == EGG_B200_TAG_ELLIPSEARC) {
        const double cp = cos(e[4]), sp = sin(e[4]);
        double u, v;
        if (nd == 0) {
            u = e[2] * cos(t);
            v = e[3] * sin(t);
            x = (e[0] + cp * u) - sp * v;
            y = (e[1] + sp * u) + cp * v;
            return;
        }
        if (nd == 1) {
            u = -e[2] * sin(t);
            v = e[3] * cos(t);
        } else {
            u = -e[2] * cos(t);
            v = -e[3] * sin(t);
        }
        x = cp * u - sp * v;
        y = sp * u + cp * v;
        return;
    }
    const double w = 1.0 - t;
    if (tag == EGG_B200_TAG_QUADBEZIER) {
        if (nd == 0) {
            const double b0 = w * w, b1 = 2.0 * w * t, b2 = t * t;
            x = (b0 * e[0] + b1 * e[2]) + b2 * e[4];
            y = (b0 * e[1] + b1 * e[3]) + b2 * e[5];
        } else if (nd == 1) {
            const double c0 = 2.0 * w, c1 = 2.0 * t;
            x = c0 * (e[2] - e[0]) + c1 * (e[4] - e[2]);
            y = c0 * (e[3] - e[1]) + c1 * (e[5] - e[3]);
        } else {
            x = 2.0 * ((e[4] - 2.0 * e[2]) + e[0]);
            y = 2.0 * ((e[5] - 2.0 * e[3]) + e[1]);
        }
        return;
    }
    // cubic
    if (nd == 0) {
        const double b0 = w * w * w, b1 = 3.0 * w * w * t, b2 = 3.0 * w * t * t, b3 = t * t * t;
        x = ((b0 * e[0] + b1 * e[2]) + b2 * e[4]) + b3 * e[6];
        y = ((b0 * e[1] + b1 * e[3]) + b2 * e[5]) + b3 * e[7];
    } else if (nd == 1) {
        const double c0 = 3.0 * w * w, c1 = 6.0 * w * t, c2 = 3.0 * t * t;
        x = (c0 * (e[2] - e[0]) + c1 * (e[4] - e[2])) + c2 * (e[6] - e[4]);
        y = (c0 * (e[3] - e[1]) + c1 * (e[5] - e[3])) + c2 * (e[7] - e[5]);
    } else {
        const double c0 = 6.0 * w, c1 = 6.0 * t;
        x = c0 * ((e[4] - 2.0 * e[2]) + e[0]) + c1 * ((e[6] - 2.0 * e[4]) + e[2]);
        y = c0 * ((e[5] - 2.0 * e[3]) + e[1]) + c1 * ((e[7] - 2.0 * e[5]) + e[3]);
    }
}

// Nearest-foot parameter on [lo, hi]: the best of 17 grid samples, then 8
// Newton steps on (C(t) - q).C'(t) (src/geometry.hpp:518-560 project_param).
EGG_OUTLINE double tc_grid_newton(int tag, const double* e, double qx, double qy, double lo, double hi)
{
    double best_t = lo, best_d = INFINITY;
    for (int i = 0; i <= 16; ++i) {
        const double tc = lo + ((hi - lo) * double(i)) / 16.0;
        double x, y;
        tc_eval(tag, e, tc, 0, x, y);
        const double dx = x - qx, dy = y - qy;
        const double dd = dx * dx + dy * dy;
        if (dd < best_d) {
            best_d = dd;
            best_t = tc;
        }
    }
    double t = best_t;
    for (int it = 0; it < 8; ++it) {
        double x, y, d1x, d1y, d2x, d2y;
        tc_eval(tag, e, t, 0, x, y);
        tc_eval(tag, e, t, 1, d1x, d1y);
        tc_eval(tag, e, t, 2, d2x, d2y);
        const double dx = x - qx, dy = y - qy;
        const double f = dx * d1x + dy * d1y;
        const double fp = (d1x * d1x + d1y * d1y) + (dx * d2x + dy * d2y);
        if (fabs(fp) < kGeomTiny) { break; }
        t -= f / fp;
    }
    return t;
}

// Raw foot parameter of (px, py): one representative for the arcs.
EGG_HD double tc_invert(int tag, const double* e, double px, double py)
{
    switch (tag) {
    case EGG_B200_TAG_CIRCLEARC: return atan2(py - e[1], px - e[0]);
    case EGG_B200_TAG_ELLIPSEARC: return tc_grid_newton(tag, e, px, py, 0.0, kArcPeriod);
    default: return tc_grid_newton(tag, e, px, py, 0.0, 1.0);
    }
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

// Cold foot: for the arcs the representative nearest the trim interval (open
// trims), then clamped onto the trim.
EGG_HD double tc_cold_foot(int tag, const double* e, double px, double py)
{
    double q = tc_invert(tag, e, px, py);
    double t0, t1;
    bool closed;
    tc_trim(tag, e, t0, t1, closed);
    if ((tag == EGG_B200_TAG_CIRCLEARC || tag == EGG_B200_TAG_ELLIPSEARC) && !closed) {
        const double mid = 0.5 * (t0 + t1);
        q = mid + remainder(q - mid, kArcPeriod);
    }
    if (!tc_contains(tag, e, q)) { q = tc_clamp(tag, e, q); }
    return q;
}

// Warm step of a curve DOF (sweeps after the first of a run call): the Newton
// step on the tangent at the raw foot q*, reduced to a parameter step
// dq = (J.J)^-1 J.delta and damped by omega; trials are q* + alpha dq,
// clamped onto the trim and evaluated.
EGG_HD void tc_warm_step(int tag, const double* e, const double H[4], const double g[2], double px, double py,
                         double omega, double& qstar, double& dq)
{
    qstar = tc_invert(tag, e, px, py);
    double jx, jy, bx, by;
    tc_eval(tag, e, qstar, 1, jx, jy);
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

// ---- B-spline / NURBS curve (tag 10) ----------------------------------------
// Record (degree, n_ctrl, t0, t1, closed, has_w, knots_at, ctrl_at, w_at): the
// last three are offsets into the session's entity arena (knots: n_ctrl +
// degree + 1 reals, control points: 2 n_ctrl, weights: n_ctrl when has_w).
// Basis functions and derivatives by the triangular recurrences of Piegl and
// Tiller, "The NURBS Book", algorithms A2.1 (span) and A2.3 (derivatives);
// the rational form by the quotient rule (src/geometry.hpp:720-965).
constexpr int kBSplineMaxDegree = 7;  // the reference's default curve degree cap
constexpr int kBSplineCap = kBSplineMaxDegree + 1;

struct BSplineCurve {
    int p, n;  // degree, control points
    const double* knots;
    const double* ctrl;
    const double* w;  // NULL: polynomial
    double t0, t1;
    bool closed;
};

EGG_HD BSplineCurve bspline_view(const double* e, const double* arena)
{
    BSplineCurve c;
    c.p = int(e[0]);
    c.n = int(e[1]);
    c.t0 = e[2];
    c.t1 = e[3];
    c.closed = e[4] != 0.0;
    c.knots = arena + int64_t(e[6]);
    c.ctrl = arena + int64_t(e[7]);
    c.w = e[5] != 0.0 ? arena + int64_t(e[8]) : nullptr;
    return c;
}

// Knot span of u: the last knot interval [k_i, k_i+1) that holds it, clamped
// to [degree, n_ctrl - 1].
EGG_HD int bspline_span(const BSplineCurve& c, double u)
{
    const int last = c.n - 1;
    if (u >= c.knots[last + 1]) { return last; }
    if (u <= c.knots[c.p]) { return c.p; }
    int lo = c.p, hi = last + 1;
    int mid = (lo + hi) / 2;
    while (u < c.knots[mid] || u >= c.knots[mid + 1]) {
        if (u < c.knots[mid]) {
            hi = mid;
        } else {
            lo = mid;
        }
        mid = (lo + hi) / 2;
    }
    return mid;
}

// der[k][j]: k-th derivative (k <= nd <= 2) of the j-th nonzero basis
// function at u in span.
EGG_HD void bspline_basis(const BSplineCurve& c, int span, double u, int nd, double der[3][kBSplineCap])
{
    const int p = c.p;
    double tab[kBSplineCap][kBSplineCap];  // lower: knot differences, upper: basis values
    double lft[kBSplineCap], rgt[kBSplineCap];
    tab[0][0] = 1.0;
    for (int j = 1; j <= p; ++j) {
        lft[j] = u - c.knots[span + 1 - j];
        rgt[j] = c.knots[span + j] - u;
        double carry = 0.0;
        for (int r = 0; r < j; ++r) {
            tab[j][r] = rgt[r + 1] + lft[j - r];
            const double q = tab[r][j - 1] / tab[j][r];
            tab[r][j] = carry + rgt[r + 1] * q;
            carry = lft[j - r] * q;
        }
        tab[j][j] = carry;
    }
    for (int j = 0; j <= p; ++j) { der[0][j] = tab[j][p]; }
    double co[2][kBSplineCap];
    for (int r = 0; r <= p; ++r) {
        int cur = 0, nxt = 1;
        co[0][0] = 1.0;
        for (int k = 1; k <= nd; ++k) {
            double acc = 0.0;
            const int rk = r - k, pk = p - k;
            if (r >= k) {
                co[nxt][0] = co[cur][0] / tab[pk + 1][rk];
                acc = co[nxt][0] * tab[rk][pk];
            }
            const int jlo = rk >= -1 ? 1 : -rk;
            const int jhi = r - 1 <= pk ? k - 1 : p - r;
            for (int j = jlo; j <= jhi; ++j) {
                co[nxt][j] = (co[cur][j] - co[cur][j - 1]) / tab[pk + 1][rk + j];
                acc += co[nxt][j] * tab[rk + j][pk];
            }
            if (r <= pk) {
                co[nxt][k] = -co[cur][k - 1] / tab[pk + 1][r];
                acc += co[nxt][k] * tab[r][pk];
            }
            der[k][r] = acc;
            const int t = cur;
            cur = nxt;
            nxt = t;
        }
    }
    double f = double(p);  // scale row k by p! / (p - k)!
    for (int k = 1; k <= nd; ++k) {
        for (int j = 0; j <= p; ++j) { der[k][j] *= f; }
        f *= double(p - k);
    }
}

// Curve point (order 0) or its first / second derivative at u.
EGG_OUTLINE void bspline_point(const BSplineCurve& c, double u, int order, double& x, double& y)
{
    const int span = bspline_span(c, u);
    double der[3][kBSplineCap];
    bspline_basis(c, span, u, order, der);
    if (c.w == nullptr) {
        double ax = 0.0, ay = 0.0;
        for (int j = 0; j <= c.p; ++j) {
            const int i = span - c.p + j;
            ax = ax + der[order][j] * c.ctrl[2 * i];
            ay = ay + der[order][j] * c.ctrl[2 * i + 1];
        }
        x = ax;
        y = ay;
        return;
    }
    // rational: A^(k) = sum N^(k) w P, w^(k) = sum N^(k) w; C = A / w,
    // C' = (A' - w' C) / w, C'' = (A'' - 2 w' C' - w'' C) / w
    double Ax[3] = {0.0, 0.0, 0.0}, Ay[3] = {0.0, 0.0, 0.0}, W[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k <= order; ++k) {
        for (int j = 0; j <= c.p; ++j) {
            const int i = span - c.p + j;
            const double nw = der[k][j] * c.w[i];
            Ax[k] = Ax[k] + nw * c.ctrl[2 * i];
            Ay[k] = Ay[k] + nw * c.ctrl[2 * i + 1];
            W[k] += nw;
        }
    }
    const double iw = 1.0 / W[0];
    double Cx[3], Cy[3];
    Cx[0] = iw * Ax[0];
    Cy[0] = iw * Ay[0];
    if (order >= 1) {
        Cx[1] = iw * (Ax[1] - W[1] * Cx[0]);
        Cy[1] = iw * (Ay[1] - W[1] * Cy[0]);
    }
    if (order >= 2) {
        Cx[2] = iw * ((Ax[2] - 2.0 * W[1] * Cx[1]) - W[2] * Cx[0]);
        Cy[2] = iw * ((Ay[2] - 2.0 * W[1] * Cy[1]) - W[2] * Cy[0]);
    }
    x = Cx[order];
    y = Cy[order];
}

// Seeded nearest-foot parameter on the live domain [knots[p], knots[n]]:
// from the clamped seed when it is finite, else the best of 17 grid samples;
// then 8 Newton steps (src/geometry.hpp:518-560 project_param_seeded).
EGG_OUTLINE double bspline_foot(const BSplineCurve& c, double qx, double qy, double seed)
{
    const double lo = c.knots[c.p], hi = c.knots[c.n];
    double t;
    if (isfinite(seed)) {
        t = seed < lo ? lo : (seed > hi ? hi : seed);
    } else {
        double best_t = lo, best_d = INFINITY;
        for (int i = 0; i <= 16; ++i) {
            const double tc = lo + ((hi - lo) * double(i)) / 16.0;
            double x, y;
            bspline_point(c, tc, 0, x, y);
            const double dx = x - qx, dy = y - qy;
            const double dd = dx * dx + dy * dy;
            if (dd < best_d) {
                best_d = dd;
                best_t = tc;
            }
        }
        t = best_t;
    }
    for (int it = 0; it < 8; ++it) {
        double x, y, d1x, d1y, d2x, d2y;
        bspline_point(c, t, 0, x, y);
        bspline_point(c, t, 1, d1x, d1y);
        bspline_point(c, t, 2, d2x, d2y);
        const double dx = x - qx, dy = y - qy;
        const double f = dx * d1x + dy * d1y;
        const double fp = (d1x * d1x + d1y * d1y) + (dx * d2x + dy * d2y);
        if (fabs(fp) < kGeomTiny) { break; }
        t -= f / fp;
    }
    return t;
}

EGG_HD double bspline_clamp(const BSplineCurve& c, double q)
{
    if (c.closed) { return arc_wrap(q, c.t0, c.t1); }
    return q < c.t0 ? c.t0 : (q > c.t1 ? c.t1 : q);
}

EGG_HD bool bspline_inside(const BSplineCurve& c, double q) { return c.closed || (q >= c.t0 && q <= c.t1); }

// Seeded projection (cold path, one trial): foot from the seed, stored back
// unclamped, clamped onto the trim and evaluated.
EGG_HD void bspline_project_seeded(const BSplineCurve& c, double px, double py, double& seed, double& qx, double& qy)
{
    double q = bspline_foot(c, px, py, seed);
    seed = q;
    if (!bspline_inside(c, q)) { q = bspline_clamp(c, q); }
    bspline_point(c, q, 0, qx, qy);
}

// Cold Newton step: the tangent at the seeded foot of pos (seed updated).
EGG_HD void bspline_cold_step(const BSplineCurve& c, const double H[4], const double g[2], double px, double py,
                              double& seed, double out[2])
{
    double q = bspline_foot(c, px, py, seed);
    seed = q;
    if (!bspline_inside(c, q)) { q = bspline_clamp(c, q); }
    double jx, jy, bx, by;
    bspline_point(c, q, 1, jx, jy);
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
    out[0] = bx * y;
    out[1] = by * y;
}

// Warm step: seeded foot q* of pos (stored as the seed), the step on the raw
// tangent there, dq = (J.J)^-1 J.delta damped by omega.
EGG_HD void bspline_warm_step(const BSplineCurve& c, const double H[4], const double g[2], double px, double py,
                              double omega, double& seed, double& qstar, double& dq)
{
    qstar = bspline_foot(c, px, py, seed);
    seed = qstar;
    double jx, jy, bx, by;
    bspline_point(c, qstar, 1, jx, jy);
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
    if (is_tcurve(tag)) {
        tc_eval(tag, e, tc_cold_foot(tag, e, px, py), 0, qx, qy);
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
    if (is_tcurve(tag)) {  // at the cold foot
        double jx, jy;
        tc_eval(tag, e, tc_cold_foot(tag, e, px, py), 1, jx, jy);
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

// ---- composite path (tag 11) -------------------------------------------------
// Record (n_segs, rec_off, .., slice_at): segment records of kCompositeRec
// reals each, [tag, params...] with the positional params of that tag, at
// arena[slice_at + rec_off ...].  A point projects onto every segment and
// keeps the nearest (strictly closer wins; the first on a tie); the tangent is
// that segment's (src/geometry.hpp:955-981, 2587-2617).
constexpr int kCompositeRec = 13;

EGG_HD bool composite_segment_ok(int tag)
{
    return tag == EGG_B200_TAG_LINESEG || tag == EGG_B200_TAG_CIRCLE || tag == EGG_B200_TAG_ELLIPSE ||
           tag == EGG_B200_TAG_LINERAIL || tag == EGG_B200_TAG_BSPLINE || is_tcurve(tag);
}

// A B-spline segment of a composite path: blob [degree, n_ctrl, knot_off,
// ctrl_off, t0, t1, w_off, has_w], offsets into the path's arena slice, an
// open trim (src/geometry.hpp:1524-1550).
EGG_HD BSplineCurve composite_bspline(const double* b, const double* slice)
{
    BSplineCurve c;
    c.p = int(b[0]);
    c.n = int(b[1]);
    c.knots = slice + int64_t(b[2]);
    c.ctrl = slice + int64_t(b[3]);
    c.t0 = b[4];
    c.t1 = b[5];
    c.closed = false;
    c.w = b[7] != 0.0 ? slice + int64_t(b[6]) : nullptr;
    return c;
}

// Nearest segment of a composite path (src/geometry.hpp:2587-2617): every
// segment projects cold (a B-spline from its grid, unseeded) and the closest
// foot wins, with its segment's unit tangent.  `slice` is the path's arena
// slice (B-spline data offsets are relative to it), `recs` its records.
EGG_OUTLINE void composite_frame(const double* slice, const double* recs, int n_segs, double px, double py,
                                 double& qx, double& qy, double& tx, double& ty)
{
    qx = px;
    qy = py;
    tx = 1.0;
    ty = 0.0;
    double best = INFINITY;
    for (int k = 0; k < n_segs; ++k) {
        const double* rec = recs + k * kCompositeRec;
        const int tag = int(rec[0]);
        if (!composite_segment_ok(tag)) { continue; }
        double fx, fy;
        if (tag == EGG_B200_TAG_BSPLINE) {
            const BSplineCurve c = composite_bspline(rec + 1, slice);
            double q = bspline_foot(c, px, py, INFINITY);
            if (!bspline_inside(c, q)) { q = bspline_clamp(c, q); }
            bspline_point(c, q, 0, fx, fy);
            const double dx = fx - px, dy = fy - py;
            const double dd = dx * dx + dy * dy;
            if (dd < best) {
                best = dd;
                qx = fx;
                qy = fy;
                double jx, jy;
                bspline_point(c, q, 1, jx, jy);
                unit_or_e0(jx, jy, tx, ty);
            }
            continue;
        }
        entity_project(tag, rec + 1, px, py, fx, fy);
        const double dx = fx - px, dy = fy - py;
        const double dd = dx * dx + dy * dy;
        if (dd < best) {
            best = dd;
            qx = fx;
            qy = fy;
            entity_tangent(tag, rec + 1, px, py, tx, ty);
        }
    }
}

EGG_HD void composite_newton_step(const double* slice, const double* recs, int n_segs, const double H[4],
                                  const double g[2], double px, double py, double out[2])
{
    double qx, qy, bx, by;
    composite_frame(slice, recs, n_segs, px, py, qx, qy, bx, by);
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
    if (dim == 3) {
        return tag == EGG_B200_TAG_PLANE || tag == EGG_B200_TAG_SPHERE || tag == EGG_B200_TAG_CYLINDER ||
               tag == EGG_B200_TAG_LINE3 || tag == EGG_B200_TAG_LINERAIL3 || tag == EGG_B200_TAG_BSPLINESURF;
    }
    return dim == 2 && (tag == EGG_B200_TAG_LINESEG || tag == EGG_B200_TAG_CIRCLE ||
                        tag == EGG_B200_TAG_ELLIPSE || tag == EGG_B200_TAG_LINERAIL || is_tcurve(tag) ||
                        tag == EGG_B200_TAG_BSPLINE || tag == EGG_B200_TAG_COMPOSITE);
}

}  // namespace egg_b200
