// 3D boundary entities of constrained DOFs (host + device, fp64), with the
// reference's geometry (src/geometry.hpp):
//   Plane, Sphere, Cylinder (untrimmed surfaces) and Line3 (a trimmed line):
//              foot, evaluation and raw frame           :1001-1092, :2271-2420
//   LineRail3  (s(3), e(3))  open-ended segment: identity beyond its ends
//                                                           :363-396
// and the Newton step reduced onto an orthonormal tangent basis B (3 x K):
// M = B^T H B, r = B^T g, y = solve(M, r), delta = B y (src/patch.hpp:355-388,
// K = 1: solve1x1, K = 2: solveNxN<2>).  A parametric DOF after the first
// sweep of a run call searches in its parameters instead
// (src/sweep.hpp:1718-1832): dq = (J^T J)^-1 J^T delta, trials eval(q* + alpha dq).
#pragma once

#include "entity2.cuh"
#include "metric3.cuh"

namespace egg_b200
{

EGG_HD double dot3v(const double* a, const double* b)
{
    double acc = 0.0;
    acc += a[0] * b[0];
    acc += a[1] * b[1];
    acc += a[2] * b[2];
    return acc;
}

// a / |a| as (1/|a|) a, or e_0 below the zero-vector guard.
EGG_HD void normalize3(const double* a, double* out)
{
    const double n = sqrt(dot3v(a, a));
    if (n < kGeomZnorm) {
        out[0] = 1.0;
        out[1] = 0.0;
        out[2] = 0.0;
        return;
    }
    const double inv = 1.0 / n;
    for (int i = 0; i < 3; ++i) { out[i] = inv * a[i]; }
}

EGG_HD void cross3v(const double* a, const double* b, double* out)
{
    out[0] = a[1] * b[2] - a[2] * b[1];
    out[1] = a[2] * b[0] - a[0] * b[2];
    out[2] = a[0] * b[1] - a[1] * b[0];
}

// ---- 3D parametric entities (untrimmed surfaces, trimmed line) -------------
//   Plane     (o(3), ax(3), ay(3))        q = in-plane coordinates
//   Sphere    (c(3), r, ax(3), ay(3))     q = (azimuth, latitude), az = ax x ay
//   Cylinder  (o(3), ax(3), ay(3), r)     q = (angle about az, height), az = ax x ay
//   Line3     (p0(3), p1(3), t0, t1)      q = foot parameter, trimmed to [t0, t1]
// (src/geometry.hpp:1001-1092, records :2271-2420).
EGG_HD bool is_surf3(int tag)
{
    return tag == EGG_B200_TAG_PLANE || tag == EGG_B200_TAG_SPHERE || tag == EGG_B200_TAG_CYLINDER;
}

EGG_HD bool is_param3(int tag) { return is_surf3(tag) || tag == EGG_B200_TAG_LINE3; }

EGG_HD void p3_invert(int tag, const double* e, const double* p, double q[2])
{
    if (tag == EGG_B200_TAG_PLANE) {
        const double d[3] = {p[0] - e[0], p[1] - e[1], p[2] - e[2]};
        q[0] = dot3v(d, e + 3);
        q[1] = dot3v(d, e + 6);
        return;
    }
    if (tag == EGG_B200_TAG_SPHERE) {
        const double d[3] = {p[0] - e[0], p[1] - e[1], p[2] - e[2]};
        double m[3], az[3];
        normalize3(d, m);
        cross3v(e + 4, e + 7, az);
        const double w = dot3v(m, az);
        q[0] = atan2(dot3v(m, e + 7), dot3v(m, e + 4));
        q[1] = asin(w < -1.0 ? -1.0 : (w > 1.0 ? 1.0 : w));
        return;
    }
    if (tag == EGG_B200_TAG_CYLINDER) {
        const double d[3] = {p[0] - e[0], p[1] - e[1], p[2] - e[2]};
        double az[3];
        cross3v(e + 3, e + 6, az);
        q[0] = atan2(dot3v(d, e + 6), dot3v(d, e + 3));
        q[1] = dot3v(d, az);
        return;
    }
    // line
    const double ab[3] = {e[3] - e[0], e[4] - e[1], e[5] - e[2]};
    const double d[3] = {p[0] - e[0], p[1] - e[1], p[2] - e[2]};
    q[0] = dot3v(d, ab) / fmax(dot3v(ab, ab), kGeomTiny);
    q[1] = 0.0;
}

EGG_HD void p3_eval(int tag, const double* e, const double q[2], double* out)
{
    if (tag == EGG_B200_TAG_PLANE) {
        for (int i = 0; i < 3; ++i) { out[i] = (e[i] + q[0] * e[3 + i]) + q[1] * e[6 + i]; }
        return;
    }
    if (tag == EGG_B200_TAG_SPHERE) {
        const double cu = cos(q[0]), su = sin(q[0]), cv = cos(q[1]), sv = sin(q[1]);
        double az[3];
        cross3v(e + 4, e + 7, az);
        const double a = cv * cu, b = cv * su;
        for (int i = 0; i < 3; ++i) { out[i] = e[i] + e[3] * ((a * e[4 + i] + b * e[7 + i]) + sv * az[i]); }
        return;
    }
    if (tag == EGG_B200_TAG_CYLINDER) {
        const double cu = cos(q[0]), su = sin(q[0]);
        double az[3];
        cross3v(e + 3, e + 6, az);
        for (int i = 0; i < 3; ++i) { out[i] = (e[i] + e[9] * (cu * e[3 + i] + su * e[6 + i])) + q[1] * az[i]; }
        return;
    }
    for (int i = 0; i < 3; ++i) { out[i] = e[i] + q[0] * (e[3 + i] - e[i]); }
}

// Raw tangent columns J[0..K-1] at q.
EGG_HD void p3_frame(int tag, const double* e, const double q[2], double J[2][3])
{
    if (tag == EGG_B200_TAG_PLANE) {
        for (int i = 0; i < 3; ++i) {
            J[0][i] = e[3 + i];
            J[1][i] = e[6 + i];
        }
        return;
    }
    if (tag == EGG_B200_TAG_SPHERE) {
        const double cu = cos(q[0]), su = sin(q[0]), cv = cos(q[1]), sv = sin(q[1]);
        double az[3];
        cross3v(e + 4, e + 7, az);
        const double a0 = cv * -su, b0 = cv * cu, a1 = -sv * cu, b1 = sv * su;
        for (int i = 0; i < 3; ++i) {
            J[0][i] = e[3] * (a0 * e[4 + i] + b0 * e[7 + i]);
            J[1][i] = e[3] * ((a1 * e[4 + i] - b1 * e[7 + i]) + cv * az[i]);
        }
        return;
    }
    if (tag == EGG_B200_TAG_CYLINDER) {
        const double cu = cos(q[0]), su = sin(q[0]);
        double az[3];
        cross3v(e + 3, e + 6, az);
        for (int i = 0; i < 3; ++i) {
            J[0][i] = e[9] * (-su * e[3 + i] + cu * e[6 + i]);
            J[1][i] = az[i];
        }
        return;
    }
    for (int i = 0; i < 3; ++i) {
        J[0][i] = e[3 + i] - e[i];
        J[1][i] = 0.0;
    }
}

// Trim clamp (surfaces here are untrimmed; the line is trimmed to [t0, t1]).
EGG_HD void p3_clamp(int tag, const double* e, double q[2])
{
    if (tag == EGG_B200_TAG_LINE3) { q[0] = q[0] < e[6] ? e[6] : (q[0] > e[7] ? e[7] : q[0]); }
}

// Gram-Schmidt of K raw columns.
EGG_HD void p3_basis(int tag, const double J[2][3], double B[2][3])
{
    normalize3(J[0], B[0]);
    if (!is_surf3(tag)) { return; }
    double t[3];
    const double c = dot3v(J[1], B[0]);
    for (int i = 0; i < 3; ++i) { t[i] = J[1][i] - c * B[0][i]; }
    normalize3(t, B[1]);
}

EGG_HD double rail3_foot(const double* e, const double* p)
{
    const double ax = e[3] - e[0], ay = e[4] - e[1], az = e[5] - e[2];
    const double ab_sq = ax * ax + ay * ay + az * az;
    return ((p[0] - e[0]) * ax + (p[1] - e[1]) * ay + (p[2] - e[2]) * az) / fmax(ab_sq, kGeomTiny);
}

// Newton step reduced onto K orthonormal columns B (H: full 3x3 row-major).
template <int K> EGG_HD void step_from_basis3(const double g[3], const double H[9], const double B[][3], double d[3])
{
    double M[K * K], r[K];
    for (int a = 0; a < K; ++a) {
        double Hb[3];
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int j = 0; j < 3; ++j) { s += H[i * 3 + j] * B[a][j]; }
            Hb[i] = s;
        }
        for (int b = 0; b < K; ++b) {
            double s = 0.0;
            for (int i = 0; i < 3; ++i) { s += B[b][i] * Hb[i]; }
            M[a * K + b] = s;
        }
        double s = 0.0;
        for (int i = 0; i < 3; ++i) { s += B[a][i] * g[i]; }
        r[a] = s;
    }
    double y[K];
    if constexpr (K == 1) {
        y[0] = 0.0;
        const double rn = fabs(r[0]);
        if (!(rn < kGeomZnorm)) {
            y[0] = -r[0] / M[0];
            if (!isfinite(y[0])) { y[0] = -0.1 * r[0] / rn; }
        }
    } else {
        solve2<double>(M, r, y);
    }
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int a = 0; a < K; ++a) { s += B[a][i] * y[a]; }
        d[i] = s;
    }
}

EGG_HD void entity3_project(int tag, const double* e, const double* p, double* out)
{
    if (is_param3(tag)) {  // cold foot (clamped onto the trim), evaluated
        double q[2];
        p3_invert(tag, e, p, q);
        p3_clamp(tag, e, q);
        p3_eval(tag, e, q, out);
        return;
    }
    // rail
    const double t = rail3_foot(e, p);
    if (t < 0.0 || t > 1.0) {
        for (int i = 0; i < 3; ++i) { out[i] = p[i]; }
        return;
    }
    for (int i = 0; i < 3; ++i) { out[i] = e[i] + t * (e[3 + i] - e[i]); }
}

// Cold Newton step of a constrained 3D DOF (h: packed symmetric xx, xy, xz,
// yy, yz, zz): reduced onto the orthonormal frame at the cold foot.
EGG_HD void entity3_newton_step(int tag, const double* e, const double h[6], const double g[3], const double* pos,
                                double d[3])
{
    const double H[9] = {h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]};
    if (is_param3(tag)) {
        double q[2], J[2][3], B[2][3];
        p3_invert(tag, e, pos, q);
        p3_clamp(tag, e, q);
        p3_frame(tag, e, q, J);
        p3_basis(tag, J, B);
        if (is_surf3(tag)) {
            step_from_basis3<2>(g, H, B, d);
        } else {
            step_from_basis3<1>(g, H, B, d);
        }
        return;
    }
    const double t = rail3_foot(e, pos);
    if (t < 0.0 || t > 1.0) {  // released: the full-space step
        solve3<double>(h, g, d);
        return;
    }
    const double ax = e[3] - e[0], ay = e[4] - e[1], az = e[5] - e[2];
    const double norm = sqrt(ax * ax + ay * ay + az * az);
    double B[1][3] = {{1.0, 0.0, 0.0}};
    if (!(norm < kGeomZnorm)) {
        B[0][0] = ax / norm;
        B[0][1] = ay / norm;
        B[0][2] = az / norm;
    }
    step_from_basis3<1>(g, H, B, d);
}

// Warm step of a 3D parametric DOF (sweeps after the first of a run call):
// raw foot q*, the step on the orthonormalized raw frame J, reduced to
// dq = (J^T J)^-1 J^T delta and damped by omega; trials eval(clamp(q* + alpha dq)).
EGG_HD void param3_warm_step(int tag, const double* e, const double h[6], const double g[3], const double* pos,
                             double omega, double qstar[2], double dq[2])
{
    p3_invert(tag, e, pos, qstar);
    const double H[9] = {h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]};
    double J[2][3], B[2][3], d[3];
    p3_frame(tag, e, qstar, J);
    p3_basis(tag, J, B);
    dq[0] = dq[1] = 0.0;
    if (!is_surf3(tag)) {
        step_from_basis3<1>(g, H, B, d);
        const double m = dot3v(J[0], J[0]);
        dq[0] = (fabs(m) > kGeomTiny) ? dot3v(J[0], d) / m : 0.0;
        dq[0] *= omega;
        return;
    }
    step_from_basis3<2>(g, H, B, d);
    double M[4], b[2];
    for (int a = 0; a < 2; ++a) {
        for (int c = 0; c < 2; ++c) { M[a * 2 + c] = dot3v(J[a], J[c]); }
        b[a] = dot3v(J[a], d);
    }
    const double det = M[0] * M[3] - M[1] * M[2];
    if (!(fabs(det) < kGeomTiny)) {
        const double inv = 1.0 / det;
        dq[0] = inv * (M[3] * b[0] - M[1] * b[1]);
        dq[1] = inv * (-M[2] * b[0] + M[0] * b[1]);
    }
    dq[0] *= omega;
    dq[1] *= omega;
}

}  // namespace egg_b200
