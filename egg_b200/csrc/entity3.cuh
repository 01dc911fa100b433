// 3D boundary entities of constrained DOFs (host + device, fp64), with the
// reference's geometry (src/geometry.hpp):
//   Plane      (o(3), ax(3), ay(3))  untrimmed plane; foot = in-plane
//              coordinates, frame = (ax, ay)               :1001-1015, :2271-2303
//   LineRail3  (s(3), e(3))  open-ended segment: identity beyond its ends
//                                                           :363-396
// and the Newton step reduced onto an orthonormal tangent basis B (3 x K):
// M = B^T H B, r = B^T g, y = solve(M, r), delta = B y (src/patch.hpp:355-388,
// K = 1: solve1x1, K = 2: solveNxN<2>).  A plane DOF after the first sweep of
// a run call searches in its in-plane coordinates instead
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

// Gram-Schmidt of the plane's frame (ax, ay).
EGG_HD void plane_basis(const double* e, double B[2][3])
{
    normalize3(e + 3, B[0]);
    double t[3];
    const double c = dot3v(e + 6, B[0]);
    for (int i = 0; i < 3; ++i) { t[i] = e[6 + i] - c * B[0][i]; }
    normalize3(t, B[1]);
}

EGG_HD void plane_invert(const double* e, const double* p, double q[2])
{
    const double d[3] = {p[0] - e[0], p[1] - e[1], p[2] - e[2]};
    q[0] = dot3v(d, e + 3);
    q[1] = dot3v(d, e + 6);
}

EGG_HD void plane_eval(const double* e, const double q[2], double* out)
{
    for (int i = 0; i < 3; ++i) { out[i] = (e[i] + q[0] * e[3 + i]) + q[1] * e[6 + i]; }
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
    if (tag == EGG_B200_TAG_PLANE) {
        double q[2];
        plane_invert(e, p, q);
        plane_eval(e, q, out);
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
// yy, yz, zz).
EGG_HD void entity3_newton_step(int tag, const double* e, const double h[6], const double g[3], const double* pos,
                                double d[3])
{
    const double H[9] = {h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]};
    if (tag == EGG_B200_TAG_PLANE) {
        double B[2][3];
        plane_basis(e, B);
        step_from_basis3<2>(g, H, B, d);
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

// Warm in-plane step of a plane DOF: foot q*, step dq (damped by omega).
EGG_HD void plane_warm_step(const double* e, const double h[6], const double g[3], const double* pos, double omega,
                            double qstar[2], double dq[2])
{
    plane_invert(e, pos, qstar);
    const double H[9] = {h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]};
    double B[2][3], d[3];
    plane_basis(e, B);
    step_from_basis3<2>(g, H, B, d);
    const double* J[2] = {e + 3, e + 6};
    double M[4], b[2];
    for (int a = 0; a < 2; ++a) {
        for (int c = 0; c < 2; ++c) { M[a * 2 + c] = dot3v(J[a], J[c]); }
        b[a] = dot3v(J[a], d);
    }
    const double det = M[0] * M[3] - M[1] * M[2];
    if (fabs(det) < kGeomTiny) {
        dq[0] = dq[1] = 0.0;
    } else {
        const double inv = 1.0 / det;
        dq[0] = inv * (M[3] * b[0] - M[1] * b[1]);
        dq[1] = inv * (-M[2] * b[0] + M[0] * b[1]);
    }
    dq[0] *= omega;
    dq[1] *= omega;
}

}  // namespace egg_b200
