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

// ---- B-spline / NURBS surfaces (tag 14) -------------------------------------
// Record: (pu, pv, nu, nv, ku_at, kv_at, ctrl_at, w_at, has_w, trim_at), the
// *_at fields arena offsets of the knot vectors (nu + pu + 1, nv + pv + 1),
// the control net (3 nu nv, u-major) and the weights (nu nv); trim_at < 0
// for an untrimmed surface, else the offset of (n_loop_entries, loops_at,
// verts_at): the UV trim polygon's loop offsets [0, n0, n0 + n1, ..., total]
// and its vertices (u, v) (src/geometry.hpp:1095-1420, decode :1616-1650,
// trim :144-191).  Evaluation by the tensor product of the curve bases
// (The NURBS Book A2.3 in each direction, the rational form by the
// quotient rule); the foot by Newton on ((S - p) . S_u, (S - p) . S_v) = 0:
// Gauss-Newton from a seed (the DOF's last foot), else from the 4 best of a
// 9 x 9 parameter grid polished by damped Newton (Levenberg-Marquardt with
// residual backtracking), the nearest foot winning.  These functions are
// inlined into one out-of-line entry, bsurf_dof: out-of-line device copies
// of them calling one another returned wrong partials on sm_100a, and
// inlining them into every stored-patch kernel instantiation costs more
// compile time than the entry's call does at run time.
constexpr double kSurfTiny = 1e-30;    // det / denominator floor
constexpr double kSurfNewton = 1e-9;   // |dq| break of the foot iterations

struct BSplineSurf {
    BSplineCurve u, v;  // degree, count and knots per direction
    int nu, nv;
    const double* ctrl;
    const double* w;       // NULL: polynomial
    const double* loops;   // NULL: untrimmed
    const double* verts;
    int n_loop;
};

// Host check of a tag-14 record against its arena: integral degrees in
// 1..kBSplineMaxDegree with more controls than the degree, and every
// addressed span (knots, net, weights, trim header, loops, vertices) inside
// the arena, the loop offsets non-decreasing from 0.
inline bool bsurf_record_ok(const double* e, const double* arena, int64_t len)
{
    auto integral = [](double x) { return std::isfinite(x) && double(int64_t(x)) == x; };
    auto span_ok = [&](double at, double n) { return integral(at) && at >= 0.0 && n >= 0.0 && at + n <= double(len); };
    for (int k = 0; k < 9; ++k) {
        if (k != 8 && !integral(e[k])) { return false; }
    }
    const double pu = e[0], pv = e[1], nu = e[2], nv = e[3];
    if (pu < 1 || pu > kBSplineMaxDegree || pv < 1 || pv > kBSplineMaxDegree || nu < pu + 1 || nv < pv + 1 ||
        nu * nv > 1e9) {
        return false;
    }
    if (!arena || !span_ok(e[4], nu + pu + 1) || !span_ok(e[5], nv + pv + 1) || !span_ok(e[6], 3 * nu * nv) ||
        (e[8] != 0.0 && !span_ok(e[7], nu * nv))) {
        return false;
    }
    if (!(e[9] >= 0.0)) { return true; }
    if (!span_ok(e[9], 3)) { return false; }
    const double* h = arena + int64_t(e[9]);
    const double nl = h[0];
    if (!integral(nl) || nl < 2 || !span_ok(h[1], nl)) { return false; }
    const double* loops = arena + int64_t(h[1]);
    if (loops[0] != 0.0) { return false; }
    for (int64_t l = 0; l + 1 < int64_t(nl); ++l) {
        if (!integral(loops[l + 1]) || loops[l + 1] < loops[l]) { return false; }
    }
    return span_ok(h[2], 2.0 * loops[int64_t(nl) - 1]);
}

EGG_HD BSplineSurf bsurf_view(const double* e, const double* arena)
{
    BSplineSurf s;
    s.u.p = int(e[0]);
    s.v.p = int(e[1]);
    s.nu = s.u.n = int(e[2]);
    s.nv = s.v.n = int(e[3]);
    s.u.knots = arena + int64_t(e[4]);
    s.v.knots = arena + int64_t(e[5]);
    s.u.ctrl = s.v.ctrl = nullptr;
    s.u.w = s.v.w = nullptr;
    s.u.t0 = s.v.t0 = 0.0;
    s.u.t1 = s.v.t1 = 1.0;
    s.u.closed = s.v.closed = false;
    s.ctrl = arena + int64_t(e[6]);
    s.w = e[8] != 0.0 ? arena + int64_t(e[7]) : nullptr;
    s.loops = s.verts = nullptr;
    s.n_loop = 0;
    if (e[9] >= 0.0) {
        const double* h = arena + int64_t(e[9]);
        s.n_loop = int(h[0]);
        s.loops = arena + int64_t(h[1]);
        s.verts = arena + int64_t(h[2]);
    }
    return s;
}

// Surface partials S00, S10, S01, S20, S02, S11 (rows 0..5) up to order nd.
EGG_HD void bsurf_ders(const BSplineSurf& s, const double q[2], int nd, double S[6][3])
{
    const int su = bspline_span(s.u, q[0]), sv = bspline_span(s.v, q[1]);
    double du[3][kBSplineCap], dv[3][kBSplineCap];
    bspline_basis(s.u, su, q[0], nd, du);
    bspline_basis(s.v, sv, q[1], nd, dv);
    double A[6][3] = {}, wsum[6] = {};
    for (int i = 0; i <= s.u.p; ++i) {
        const int iu = su - s.u.p + i;
        for (int j = 0; j <= s.v.p; ++j) {
            const int iv = sv - s.v.p + j;
            const int64_t c = int64_t(iu) * s.nv + iv;
            const double wt = s.w ? s.w[c] : 1.0;
            const double Pw[3] = {wt * s.ctrl[3 * c], wt * s.ctrl[3 * c + 1], wt * s.ctrl[3 * c + 2]};
            double n[6];
            n[0] = du[0][i] * dv[0][j];
            if (nd >= 1) {
                n[1] = du[1][i] * dv[0][j];
                n[2] = du[0][i] * dv[1][j];
            }
            if (nd >= 2) {
                n[5] = du[1][i] * dv[1][j];
                n[3] = du[2][i] * dv[0][j];
                n[4] = du[0][i] * dv[2][j];
            }
            const int rows = nd == 0 ? 1 : (nd == 1 ? 3 : 6);
            for (int r = 0; r < rows; ++r) {
                for (int k = 0; k < 3; ++k) { A[r][k] = A[r][k] + n[r] * Pw[k]; }
                wsum[r] += n[r] * wt;
            }
        }
    }
    if (!s.w) {
        for (int r = 0; r < 6; ++r) {
            for (int k = 0; k < 3; ++k) { S[r][k] = A[r][k]; }
        }
        return;
    }
    const double iw = 1.0 / wsum[0];
    for (int k = 0; k < 3; ++k) { S[0][k] = iw * A[0][k]; }
    if (nd >= 1) {
        for (int k = 0; k < 3; ++k) {
            S[1][k] = iw * (A[1][k] - wsum[1] * S[0][k]);
            S[2][k] = iw * (A[2][k] - wsum[2] * S[0][k]);
        }
    }
    if (nd >= 2) {
        for (int k = 0; k < 3; ++k) {
            S[5][k] = iw * (A[5][k] - wsum[1] * S[2][k] - wsum[2] * S[1][k] - wsum[5] * S[0][k]);
            S[3][k] = iw * (A[3][k] - 2.0 * wsum[1] * S[1][k] - wsum[3] * S[0][k]);
            S[4][k] = iw * (A[4][k] - 2.0 * wsum[2] * S[2][k] - wsum[4] * S[0][k]);
        }
    }
}

EGG_HD void bsurf_eval(const BSplineSurf& s, const double q[2], double out[3])
{
    double S[6][3];
    bsurf_ders(s, q, 0, S);
    for (int k = 0; k < 3; ++k) { out[k] = S[0][k]; }
}

EGG_HD void bsurf_domain(const BSplineSurf& s, double& u0, double& u1, double& v0, double& v1)
{
    u0 = s.u.knots[s.u.p];
    u1 = s.u.knots[s.nu];
    v0 = s.v.knots[s.v.p];
    v1 = s.v.knots[s.nv];
}

EGG_HD double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Even-odd test of (u, v) against the trim loops; untrimmed contains all.
EGG_HD bool bsurf_contains(const BSplineSurf& s, const double q[2])
{
    if (s.n_loop < 2) { return true; }
    bool inside = false;
    for (int l = 0; l + 1 < s.n_loop; ++l) {
        const int lo = int(s.loops[l]), hi = int(s.loops[l + 1]);
        for (int i = lo, j = hi - 1; i < hi; j = i++) {
            const double au = s.verts[2 * i], av = s.verts[2 * i + 1], bu = s.verts[2 * j], bv = s.verts[2 * j + 1];
            if ((av > q[1]) != (bv > q[1]) && q[0] < ((bu - au) * (q[1] - av) / (bv - av)) + au) { inside = !inside; }
        }
    }
    return inside;
}

// Nearest point of the trim loops' polylines (closed loops); untrimmed: q.
EGG_HD void bsurf_trim_clamp(const BSplineSurf& s, double q[2])
{
    double bu = q[0], bv = q[1], best = INFINITY;
    for (int l = 0; l + 1 < s.n_loop; ++l) {
        const int lo = int(s.loops[l]), hi = int(s.loops[l + 1]);
        for (int i = lo, j = hi - 1; i < hi; j = i++) {
            const double au = s.verts[2 * j], av = s.verts[2 * j + 1];
            const double eu = s.verts[2 * i] - au, ev = s.verts[2 * i + 1] - av;
            const double ab = eu * eu + ev * ev;
            double t = ab > kSurfTiny ? ((q[0] - au) * eu + (q[1] - av) * ev) / ab : 0.0;
            t = clampd(t, 0.0, 1.0);
            const double pu = au + t * eu, pv = av + t * ev;
            const double du = pu - q[0], dv = pv - q[1];
            const double dd = du * du + dv * dv;
            if (dd < best) {
                best = dd;
                bu = pu;
                bv = pv;
            }
        }
    }
    q[0] = bu;
    q[1] = bv;
}

// Newton on the foot conditions from q, iterates clamped to the domain,
// stopping when the clamped iterate moves less than kSurfNewton or the
// Jacobian is singular.  EXACT adds the curvature terms (d . S_uv...).  J
// receives the raw frame (S_u, S_v) of the last iterate evaluated.
EGG_HD void bsurf_newton(const BSplineSurf& s, const double* p, double q[2], bool exact, double J[2][3])
{
    double u0, u1, v0, v1;
    bsurf_domain(s, u0, u1, v0, v1);
    #pragma unroll 1
    for (int it = 0; it < 12; ++it) {
        double S[6][3];
        bsurf_ders(s, q, exact ? 2 : 1, S);
        for (int k = 0; k < 3; ++k) {
            J[0][k] = S[1][k];
            J[1][k] = S[2][k];
        }
        const double d[3] = {S[0][0] - p[0], S[0][1] - p[1], S[0][2] - p[2]};
        const double f1 = dot3v(d, S[1]), f2 = dot3v(d, S[2]);
        double j11 = dot3v(S[1], S[1]), j12 = dot3v(S[1], S[2]), j22 = dot3v(S[2], S[2]);
        if (exact) {
            j11 += dot3v(d, S[3]);
            j12 += dot3v(d, S[5]);
            j22 += dot3v(d, S[4]);
        }
        const double det = j11 * j22 - j12 * j12;
        if (fabs(det) < kSurfTiny) { break; }
        const double qu = clampd(q[0] - (j22 * f1 - j12 * f2) / det, u0, u1);
        const double qv = clampd(q[1] - (-j12 * f1 + j11 * f2) / det, v0, v1);
        const bool done = fabs(qu - q[0]) + fabs(qv - q[1]) < kSurfNewton;
        q[0] = qu;
        q[1] = qv;
        if (done) { break; }
    }
}

// Damped Newton from one seed (cold multi-start only): the damping bridges
// Gauss-Newton and gradient descent, and a step is kept only if it lowers
// |S - p|^2 (up to 6 damping increases per iteration).
EGG_HD void bsurf_newton_lm(const BSplineSurf& s, const double* p, double q[2], double J[2][3])
{
    double u0, u1, v0, v1;
    bsurf_domain(s, u0, u1, v0, v1);
    q[0] = clampd(q[0], u0, u1);
    q[1] = clampd(q[1], v0, v1);
    double S[6][3];
    bsurf_ders(s, q, 2, S);
    double d[3] = {S[0][0] - p[0], S[0][1] - p[1], S[0][2] - p[2]};
    double r = dot3v(d, d);
    double lambda = 1e-3 * (dot3v(S[1], S[1]) + dot3v(S[2], S[2]) + kSurfTiny);
    #pragma unroll 1
    for (int it = 0; it < 16; ++it) {
        const double f1 = dot3v(d, S[1]), f2 = dot3v(d, S[2]);
        const double j11 = dot3v(S[1], S[1]) + dot3v(d, S[3]);
        const double j12 = dot3v(S[1], S[2]) + dot3v(d, S[5]);
        const double j22 = dot3v(S[2], S[2]) + dot3v(d, S[4]);
        double du = 0.0, dv = 0.0;
        bool accepted = false;
        #pragma unroll 1
        for (int bt = 0; bt < 6; ++bt) {
            const double a11 = j11 + lambda, a22 = j22 + lambda;
            const double det = a11 * a22 - j12 * j12;
            if (fabs(det) < kSurfTiny) {
                lambda *= 4.0;
                continue;
            }
            du = -((a22 * f1 - j12 * f2) / det);
            dv = -((-j12 * f1 + a11 * f2) / det);
            const double qn[2] = {clampd(q[0] + du, u0, u1), clampd(q[1] + dv, v0, v1)};
            double e[3];
            bsurf_eval(s, qn, e);
            const double dn[3] = {e[0] - p[0], e[1] - p[1], e[2] - p[2]};
            const double rn = dot3v(dn, dn);
            if (rn < r) {
                q[0] = qn[0];
                q[1] = qn[1];
                r = rn;
                bsurf_ders(s, q, 2, S);
                for (int k = 0; k < 3; ++k) { d[k] = S[0][k] - p[k]; }
                lambda = fmax(lambda * 0.3, kSurfTiny);
                accepted = true;
                break;
            }
            lambda *= 4.0;
        }
        if (!accepted || fabs(du) + fabs(dv) < kSurfNewton) { break; }
    }
    for (int k = 0; k < 3; ++k) {
        J[0][k] = S[1][k];
        J[1][k] = S[2][k];
    }
}

// Foot parameter of p (src/geometry.hpp:1342-1420 invert_seeded): from the
// seed when there is one (Gauss-Newton), else the multi-start search; J is
// the raw frame the chosen iteration saw last.
EGG_HD void bsurf_invert(const BSplineSurf& s, const double* p, const double seed[2], bool has_seed, double q[2],
                              double J[2][3])
{
    double u0, u1, v0, v1;
    bsurf_domain(s, u0, u1, v0, v1);
    if (has_seed) {
        q[0] = clampd(seed[0], u0, u1);
        q[1] = clampd(seed[1], v0, v1);
        bsurf_newton(s, p, q, false, J);
        return;
    }
    constexpr int kGrid = 8, kStarts = 4;
    double bestd[kStarts], bestq[kStarts][2];
    for (int k = 0; k < kStarts; ++k) {
        bestd[k] = INFINITY;
        bestq[k][0] = u0;
        bestq[k][1] = v0;
    }
    #pragma unroll 1
    for (int i = 0; i <= kGrid; ++i) {
        #pragma unroll 1
        for (int j = 0; j <= kGrid; ++j) {
            const double t[2] = {u0 + ((u1 - u0) * i) / kGrid, v0 + ((v1 - v0) * j) / kGrid};
            double e[3];
            bsurf_eval(s, t, e);
            const double dx[3] = {e[0] - p[0], e[1] - p[1], e[2] - p[2]};
            const double dd = dot3v(dx, dx);
            if (dd < bestd[kStarts - 1]) {
                int k = kStarts - 1;
                for (; k > 0 && dd < bestd[k - 1]; --k) {
                    bestd[k] = bestd[k - 1];
                    bestq[k][0] = bestq[k - 1][0];
                    bestq[k][1] = bestq[k - 1][1];
                }
                bestd[k] = dd;
                bestq[k][0] = t[0];
                bestq[k][1] = t[1];
            }
        }
    }
    q[0] = u0;
    q[1] = v0;
    double best = INFINITY;
    #pragma unroll 1
    for (int k = 0; k < kStarts; ++k) {
        if (bestd[k] == INFINITY) { continue; }
        double f[2] = {bestq[k][0], bestq[k][1]}, Jk[2][3];
        bsurf_newton_lm(s, p, f, Jk);
        double e[3];
        bsurf_eval(s, f, e);
        const double dx[3] = {e[0] - p[0], e[1] - p[1], e[2] - p[2]};
        const double dd = dot3v(dx, dx);
        if (dd < best) {
            best = dd;
            q[0] = f[0];
            q[1] = f[1];
            for (int a = 0; a < 2; ++a) {
                for (int c = 0; c < 3; ++c) { J[a][c] = Jk[a][c]; }
            }
        }
    }
}

// Seeded projection / tangent basis of a constrained DOF (the seed becomes
// the unclamped foot; a foot outside the trim is clamped onto it): the
// world-space path of the first sweep of a run call and of cold trials
// (src/geometry.hpp:230-260).
EGG_HD void bsurf_foot_seeded(const BSplineSurf& s, const double* p, double seed[2], double q[2])
{
    const bool has = isfinite(seed[0]);
    double J[2][3];
    bsurf_invert(s, p, seed, has, q, J);
    seed[0] = q[0];
    seed[1] = q[1];
    if (!bsurf_contains(s, q)) { bsurf_trim_clamp(s, q); }
}

EGG_HD void bsurf_project_seeded(const BSplineSurf& s, const double* p, double seed[2], double out[3])
{
    double q[2];
    bsurf_foot_seeded(s, p, seed, q);
    bsurf_eval(s, q, out);
}

EGG_HD void bsurf_basis_at(const BSplineSurf& s, const double q[2], double B[2][3])
{
    double S[6][3];
    bsurf_ders(s, q, 1, S);
    const double J[2][3] = {{S[1][0], S[1][1], S[1][2]}, {S[2][0], S[2][1], S[2][2]}};
    p3_basis(EGG_B200_TAG_PLANE, J, B);
}

// Warm step of a B-spline-surface DOF (src/sweep.hpp:1785-1832): foot q* and
// raw frame J from Gauss-Newton off the seed (the seed becomes q*), the
// Newton step on the orthonormalised J, reduced to dq = (J^T J)^-1 J^T delta
// and damped by omega.
EGG_HD void bsurf_warm_step(const BSplineSurf& s, const double h[6], const double g[3], const double* pos,
                            double omega, double seed[2], double qstar[2], double dq[2])
{
    double J[2][3], B[2][3], d[3];
    bsurf_invert(s, pos, seed, true, qstar, J);
    seed[0] = qstar[0];
    seed[1] = qstar[1];
    const double H[9] = {h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]};
    p3_basis(EGG_B200_TAG_PLANE, J, B);
    step_from_basis3<2>(g, H, B, d);
    double M[4], b[2];
    for (int a = 0; a < 2; ++a) {
        for (int c = 0; c < 2; ++c) { M[a * 2 + c] = dot3v(J[a], J[c]); }
        b[a] = dot3v(J[a], d);
    }
    dq[0] = dq[1] = 0.0;
    const double det = M[0] * M[3] - M[1] * M[2];
    if (!(fabs(det) < kGeomTiny)) {
        const double inv = 1.0 / det;
        dq[0] = inv * (M[3] * b[0] - M[1] * b[1]);
        dq[1] = inv * (-M[2] * b[0] + M[0] * b[1]);
    }
    dq[0] *= omega;
    dq[1] *= omega;
}

// Cold step of a B-spline-surface DOF (the first sweep of a run call): the
// seeded foot's orthonormal frame (the seed becomes the foot), the Newton
// step on it.
EGG_HD void bsurf_cold_step(const BSplineSurf& s, const double h[6], const double g[3], const double* pos,
                            double seed[2], double d[3])
{
    double q[2], B[2][3];
    bsurf_foot_seeded(s, pos, seed, q);
    bsurf_basis_at(s, q, B);
    const double H[9] = {h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]};
    step_from_basis3<2>(g, H, B, d);
}

// Cold projection without a seed and its basis (src/geometry.hpp:204-222).
EGG_HD void bsurf_project_frame(const BSplineSurf& s, const double* p, double foot[3], double B[2][3])
{
    double seed[2] = {NAN, NAN}, q[2];
    bsurf_foot_seeded(s, p, seed, q);
    bsurf_eval(s, q, foot);
    bsurf_basis_at(s, q, B);
}

// The one out-of-line entry into the B-spline-surface code for the kernels
// (record er, arena): kBsurfCold -- the cold step d on the seeded foot's
// frame (io = d); kBsurfWarm -- the warm parametric step (qs, dq), seed :=
// q*; kBsurfColdTrial -- io (a raw trial) projected from the seed, which it
// advances; kBsurfWarmTrial -- io = eval(trim clamp(qs + alpha dq));
// kBsurfFrame -- io (a point) replaced by its cold foot, B the basis there.
enum BsurfOp : int { kBsurfCold = 0, kBsurfWarm, kBsurfColdTrial, kBsurfWarmTrial, kBsurfFrame };

EGG_OUTLINE void bsurf_dof(int op, const double* er, const double* arena, const double* h, const double* g,
                           const double* pos, double omega, double alpha, double* seed, double* qs, double* dq,
                           double* io, double* B)
{
    const BSplineSurf s = bsurf_view(er, arena);
    if (op == kBsurfCold) {
        bsurf_cold_step(s, h, g, pos, seed, io);
    } else if (op == kBsurfWarm) {
        bsurf_warm_step(s, h, g, pos, omega, seed, qs, dq);
    } else if (op == kBsurfColdTrial) {
        const double raw[3] = {io[0], io[1], io[2]};
        bsurf_project_seeded(s, raw, seed, io);
    } else if (op == kBsurfWarmTrial) {
        double qt[2] = {qs[0] + alpha * dq[0], qs[1] + alpha * dq[1]};
        bsurf_trim_clamp(s, qt);
        bsurf_eval(s, qt, io);
    } else {
        const double p[3] = {io[0], io[1], io[2]};
        double Bl[2][3];
        bsurf_project_frame(s, p, io, Bl);
        for (int a = 0; a < 2; ++a) {
            for (int k = 0; k < 3; ++k) { B[a * 3 + k] = Bl[a][k]; }
        }
    }
}

}  // namespace egg_b200
