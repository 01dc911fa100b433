// Soft energy terms of a moving DOF, added to the shape objective.
//
//   directional samples (src/directional.hpp:38-279), D = 2 or 3:
//     parallel (nodes i, j)   E = w (u.n)^2,        u the eps-unit of X[j] - X[i]
//     line     (nodes a, c, b) E = w |qa + qb|^2,   q the eps-units away from c
//     stem     (nodes n, c)    E = w (q.a)^2,       q the eps-unit of X[n] - X[c]
//   block-interface C2 curvature windows (src/curvature.hpp:29-183), 2D:
//     four nodes p0..p3        E = w (turn(p0,p1,p2) - turn(p1,p2,p3))^2
//
// Each term gives the DOF a closed-form gradient, a Gauss-Newton Hessian
// block plus a diagonal stabiliser for the coupling to its frozen partners,
// and an energy; the line search adds the term's energy with the DOF moved to
// the trial.  The det barrier is untouched.  eps-unit: x / sqrt(|x|^2 + eps^2).
#pragma once

#include <cmath>
#include <cstdint>

namespace egg_b200
{

constexpr int kSoftParallel = 0;
constexpr int kSoftLine = 1;
constexpr int kSoftStem = 2;
constexpr int kSoftCurv = 64;  // internal: a curvature window

// One term of a DOF (or of the whole-sample table, slot unused): node ids are
// packed-store slots, -1 pads.
struct SoftTerm {
    int32_t node[4];
    int32_t slot;  // the DOF's place in the tuple
    int32_t kind;  // kSoft*
    double ref[3];  // frozen reference vector (directional kinds)
    double w;
};

__host__ __device__ inline int soft_arity(int kind)
{
    if (kind == kSoftLine) { return 3; }
    if (kind == kSoftParallel || kind == kSoftStem) { return 2; }
    if (kind == kSoftCurv) { return 4; }
    return 0;  // reserved kinds contribute nothing
}

// c = (u.ref) / s, s = sqrt(|u|^2 + eps^2); dr = dc/du = ref/s - c u / s^2.
template <int D>
__device__ inline double soft_dot_residual(const double* u, const double* ref, double eps, double* dr)
{
    double s2 = eps * eps, c = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        s2 += u[k] * u[k];
        c += u[k] * ref[k];
    }
    const double s = sqrt(s2);
    c /= s;
    const double is = 1.0 / s, is2 = 1.0 / s2;
#pragma unroll
    for (int k = 0; k < D; ++k) { dr[k] = ref[k] * is - c * u[k] * is2; }
    return c;
}

// q = v / s and its symmetric Jacobian J = (I - v v^T / s^2) / s.
template <int D> __device__ inline void soft_unit(const double* v, double eps, double* q, double* J)
{
    double s2 = eps * eps;
#pragma unroll
    for (int k = 0; k < D; ++k) { s2 += v[k] * v[k]; }
    const double s = sqrt(s2);
    const double is = 1.0 / s, is3 = is / s2;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        q[i] = v[i] * is;
#pragma unroll
        for (int j = 0; j < D; ++j) { J[i * D + j] = (i == j ? is : 0.0) - v[i] * v[j] * is3; }
    }
}

// Signed turn at b along a -> b -> c.
__device__ inline double soft_turn(const double* a, const double* b, const double* c)
{
    const double e1x = b[0] - a[0], e1y = b[1] - a[1];
    const double e2x = c[0] - b[0], e2y = c[1] - b[1];
    return atan2(e1x * e2y - e1y * e2x, e1x * e2x + e1y * e2y);
}

// r = turn(p0,p1,p2) - turn(p1,p2,p3) and dr/dp for the four slots; the
// gradient of an edge's angle is perp(e) / |e|^2 (zero for a null edge).
__device__ inline double soft_curv_residual(const double (*p)[3], double (*dr)[2])
{
    double e[3][2], g[3][2];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        e[k][0] = p[k + 1][0] - p[k][0];
        e[k][1] = p[k + 1][1] - p[k][1];
        const double l = e[k][0] * e[k][0] + e[k][1] * e[k][1];
        const double il = l > 0.0 ? 1.0 / l : 0.0;
        g[k][0] = -e[k][1] * il;
        g[k][1] = e[k][0] * il;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        dr[0][c] = g[0][c];
        dr[1][c] = -g[0][c] - 2.0 * g[1][c];
        dr[2][c] = 2.0 * g[1][c] + g[2][c];
        dr[3][c] = -g[2][c];
    }
    return atan2(e[0][0] * e[1][1] - e[0][1] * e[1][0], e[0][0] * e[1][0] + e[0][1] * e[1][1]) -
           atan2(e[1][0] * e[2][1] - e[1][1] * e[2][0], e[1][0] * e[2][0] + e[1][1] * e[2][1]);
}

// Energy of one term at positions p (slot order).
template <int D> __device__ inline double soft_energy(const SoftTerm& t, const double (*p)[3], double eps)
{
    if (t.kind == kSoftParallel || t.kind == kSoftStem) {
        const int head = t.kind == kSoftParallel ? 1 : 0;
        double u[D], dr[D];
#pragma unroll
        for (int k = 0; k < D; ++k) { u[k] = p[head][k] - p[1 - head][k]; }
        const double c = soft_dot_residual<D>(u, t.ref, eps, dr);
        return t.w * c * c;
    }
    if (t.kind == kSoftLine) {
        double v1[D], v2[D], q1[D], q2[D], J[D * D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            v1[k] = p[0][k] - p[1][k];
            v2[k] = p[2][k] - p[1][k];
        }
        soft_unit<D>(v1, eps, q1, J);
        soft_unit<D>(v2, eps, q2, J);
        double e = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) { e += (q1[k] + q2[k]) * (q1[k] + q2[k]); }
        return t.w * e;
    }
    if constexpr (D == 2) {
        if (t.kind == kSoftCurv) {
            const double r = soft_turn(p[0], p[1], p[2]) - soft_turn(p[1], p[2], p[3]);
            return t.w * (r * r);
        }
    }
    return 0.0;
}

template <int D> __device__ inline void soft_load(const SoftTerm& t, const double* X, double (*p)[3])
{
    const int n = soft_arity(t.kind);
    for (int m = 0; m < n; ++m) {
#pragma unroll
        for (int k = 0; k < D; ++k) { p[m][k] = X[int64_t(t.node[m]) * D + k]; }
    }
}

// Adds the term's gradient, Hessian block and energy for the DOF at t.slot.
template <int D>
__device__ inline void soft_accumulate(const SoftTerm& t, const double* X, double eps, double* g, double* H,
                                       double& e0)
{
    double p[4][3];
    soft_load<D>(t, X, p);
    const int s = t.slot;
    if (t.kind == kSoftParallel || t.kind == kSoftStem) {
        const int head = t.kind == kSoftParallel ? 1 : 0;
        double u[D], dr[D];
#pragma unroll
        for (int k = 0; k < D; ++k) { u[k] = p[head][k] - p[1 - head][k]; }
        const double c = soft_dot_residual<D>(u, t.ref, eps, dr);
        e0 += t.w * c * c;
        const double gc = 2.0 * t.w * c * (s == head ? 1.0 : -1.0), hc = 2.0 * t.w;
        double dd = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            g[k] += gc * dr[k];
            dd += dr[k] * dr[k];
        }
#pragma unroll
        for (int i = 0; i < D; ++i) {
#pragma unroll
            for (int j = 0; j < D; ++j) { H[i * D + j] += hc * dr[i] * dr[j]; }
            H[i * D + i] += hc * dd;  // the partner's residual gradient is -dr
        }
        return;
    }
    if (t.kind == kSoftLine) {
        double v1[D], v2[D], q1[D], q2[D], J1[D * D], J2[D * D], r[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            v1[k] = p[0][k] - p[1][k];
            v2[k] = p[2][k] - p[1][k];
        }
        soft_unit<D>(v1, eps, q1, J1);
        soft_unit<D>(v2, eps, q2, J2);
        double e = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            r[k] = q1[k] + q2[k];
            e += r[k] * r[k];
        }
        e0 += t.w * e;
        // dr/dp_slot: J1 (slot 0), J2 (slot 2), -(J1 + J2) (slot 1, the centre)
        double Js[D * D], f1 = 0.0, f2 = 0.0, fc = 0.0;
#pragma unroll
        for (int k = 0; k < D * D; ++k) {
            Js[k] = s == 0 ? J1[k] : (s == 2 ? J2[k] : -(J1[k] + J2[k]));
            f1 += J1[k] * J1[k];
            f2 += J2[k] * J2[k];
            fc += (J1[k] + J2[k]) * (J1[k] + J2[k]);
        }
        const double gc = 2.0 * t.w;
#pragma unroll
        for (int i = 0; i < D; ++i) {
            double gi = 0.0;
#pragma unroll
            for (int j = 0; j < D; ++j) { gi += Js[i * D + j] * r[j]; }
            g[i] += gc * gi;
#pragma unroll
            for (int j = 0; j < D; ++j) {
                double h = 0.0;
#pragma unroll
                for (int m = 0; m < D; ++m) { h += Js[i * D + m] * Js[j * D + m]; }
                H[i * D + j] += gc * h;
            }
        }
        // coupling stabiliser from the Frobenius norms of the slot Jacobians
        f1 = sqrt(f1);
        f2 = sqrt(f2);
        fc = sqrt(fc);
        const double fs = s == 0 ? f1 : (s == 2 ? f2 : fc);
        const double stab = gc * fs * (f1 + f2 + fc - fs);
#pragma unroll
        for (int i = 0; i < D; ++i) { H[i * D + i] += stab; }
        return;
    }
    if constexpr (D == 2) {
        if (t.kind == kSoftCurv) {
            double dr[4][2];
            const double r = soft_curv_residual(p, dr);
            const double gc = 2.0 * t.w * r, hc = 2.0 * t.w;
            g[0] += gc * dr[s][0];
            g[1] += gc * dr[s][1];
            H[0] += hc * dr[s][0] * dr[s][0];
            H[1] += hc * dr[s][0] * dr[s][1];
            H[2] += hc * dr[s][1] * dr[s][0];
            H[3] += hc * dr[s][1] * dr[s][1];
            // block-Jacobi stabiliser |dr_s| sum_{m != s} |dr_m| on the diagonal
            double off = 0.0;
            for (int m = 0; m < 4; ++m) {
                if (m != s) { off += sqrt(dr[m][0] * dr[m][0] + dr[m][1] * dr[m][1]); }
            }
            const double stab = hc * sqrt(dr[s][0] * dr[s][0] + dr[s][1] * dr[s][1]) * off;
            H[0] += stab;
            H[3] += stab;
            e0 += t.w * r * r;
        }
    }
}

// The term's energy with the DOF (slot t.slot) moved to `trial`.
template <int D>
__device__ inline double soft_trial(const SoftTerm& t, const double* X, double eps, const double* trial)
{
    double p[4][3];
    soft_load<D>(t, X, p);
#pragma unroll
    for (int k = 0; k < D; ++k) { p[t.slot][k] = trial[k]; }
    return soft_energy<D>(t, p, eps);
}

// Per-DOF soft tables of a stored-patch level: terms [off[d], off[d+1]) of
// stored DOF d (curvature windows first, then directional samples, each in
// the wire's slot order); off == nullptr when the level has none.
struct SoftTable {
    const int32_t* off;
    const SoftTerm* terms;
    double eps;
};

template <int D>
__device__ inline void soft_dof_accumulate(const SoftTable& st, int64_t d, bool with_curv, const double* X,
                                           double* g, double* H, double& e0)
{
    if (st.off == nullptr) { return; }
    for (int32_t k = st.off[d]; k < st.off[d + 1]; ++k) {
        const SoftTerm t = st.terms[k];
        if (t.kind == kSoftCurv && !with_curv) { continue; }
        soft_accumulate<D>(t, X, st.eps, g, H, e0);
    }
}

template <int D>
__device__ inline double soft_dof_trial(const SoftTable& st, int64_t d, bool with_curv, const double* X,
                                        const double* trial)
{
    double e = 0.0;
    if (st.off == nullptr) { return e; }
    for (int32_t k = st.off[d]; k < st.off[d + 1]; ++k) {
        const SoftTerm t = st.terms[k];
        if (t.kind == kSoftCurv && !with_curv) { continue; }
        e += soft_trial<D>(t, X, st.eps, trial);
    }
    return e;
}

}  // namespace egg_b200
