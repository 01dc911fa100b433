// Per-sample TMOP metrics: value, gradient w.r.t. vec(T) and Hessian, for the
// three objectives of the egg smoother (2D).  Host + device.
//
// vec(T) = [a, b, c, d] = [T00, T01, T10, T11], D = det T = ad - bc,
// s = |T|^2, cof = dD/dvec(T) = [d, -c, -b, a], P = d(cof)/d(vec T).
//
//   shape       mu = s / (2D) - 1                       (src/metric.hpp:38-102)
//   shape_size  mu = (s / (2D))^2 - 1 + (D - 1)^2       (src/metric.hpp:150-197)
//   untangle    mu = s / (2 Dh) - 1,
//               Dh = (D + sqrt(D^2 + 4 delta^2)) / 2    (src/metric.hpp:133-142)
//
// All three are written as  mu = s * f(D) [+ size term]  so one closed form
// covers value, gradient and Hessian:
//   grad = 2 f T + s f' cof
//   Hess = 2 f I + 2 f' (T cof^T + cof T^T) + s f'' cof cof^T + s f' P
// with f = 1/(2D) for shape, f = 1/(2 Dh) for untangle (f' = -Dh'/(2Dh^2),
// f'' = -Dh''/(2Dh^2) + Dh'^2/Dh^3, Dh' = Dh/r, Dh'' = 2 delta^2 / r^3,
// r = sqrt(D^2 + 4 delta^2)).  The reference evaluates the untangle
// derivatives by forward-mode dual numbers; this closed form is the same
// function, so results agree to rounding.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define EGG_HD __host__ __device__ __forceinline__
#else
#define EGG_HD inline
#endif

namespace egg_b200
{

#ifndef __CUDACC__
// host builds (the tests' native checks): the C++ names of the CUDA math calls
using std::isfinite;
#endif

enum ObjectiveKind : int { kShape = 0, kUntangle = 1, kShapeSize = 2 };

// Line-search slack / zero-gradient guard of the working precision
// (src/core.hpp:37-51).
template <class R> struct Tol;
template <> struct Tol<double> {
    static constexpr double energy = 1e-12;
    static constexpr double znorm = 1e-15;
};
template <> struct Tol<float> {
    static constexpr float energy = 1e-6f;
    static constexpr float znorm = 1e-7f;
};

template <class R> EGG_HD R det2(const R t[4]) { return t[0] * t[3] - t[1] * t[2]; }

// f(D) and its first two derivatives for the shape-type objectives.
template <class R> struct ScaleFn {
    R f, fp, fpp;
};

template <class R> EGG_HD ScaleFn<R> shape_scale(R D)
{
    const R inv = R(1) / D;
    ScaleFn<R> r;
    r.f = R(0.5) * inv;
    r.fp = -R(0.5) * inv * inv;
    r.fpp = inv * inv * inv;
    return r;
}

// Untangle surrogate denominator, in the reference's literal form
// Dh = (D + sqrt(D^2 + 4 delta^2)) / 2 (fp64 parity path).
template <class R> EGG_HD R untangle_dh(R D, R delta)
{
    const R r = sqrt(D * D + R(4) * delta * delta);
    return R(0.5) * (D + r);
}

template <class R> EGG_HD ScaleFn<R> untangle_scale(R D, R delta)
{
    const R r = sqrt(D * D + R(4) * delta * delta);
    const R Dh = R(0.5) * (D + r);
    const R dh1 = Dh / r;                                  // dDh/dD
    const R dh2 = R(2) * delta * delta / (r * r * r);       // d2Dh/dD2
    const R inv = R(1) / Dh;
    ScaleFn<R> s;
    s.f = R(0.5) * inv;
    s.fp = -R(0.5) * dh1 * inv * inv;
    s.fpp = -R(0.5) * dh2 * inv * inv + dh1 * dh1 * inv * inv * inv;
    return s;
}

// Metric value only.
template <class R> EGG_HD R mu_value(int kind, const R t[4], R delta)
{
    const R D = det2(t);
    const R s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + t[3] * t[3];
    if (kind == kShape) { return s / (R(2) * D) - R(1); }
    if (kind == kUntangle) { return s / (R(2) * untangle_dh(D, delta)) - R(1); }
    const R m = s / (R(2) * D);
    const R dm1 = D - R(1);
    return m * m - R(1) + dm1 * dm1;
}

// Value, gradient (4) and full symmetric Hessian (4x4 row-major).
template <class R> EGG_HD void mu_eval(int kind, const R t[4], R delta, R& mu, R g[4], R H[16])
{
    const R D = det2(t);
    const R s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + t[3] * t[3];
    const R cof[4] = {t[3], -t[2], -t[1], t[0]};
    // P[i][j] = d cof_i / d t_j: nonzero (0,3)=1, (1,2)=-1, (2,1)=-1, (3,0)=1.
    auto Pm = [](int i, int j) -> R {
        const int k = i * 4 + j;
        return (k == 3 || k == 12) ? R(1) : ((k == 6 || k == 9) ? R(-1) : R(0));
    };
    ScaleFn<R> sf;
    if (kind == kUntangle) {
        sf = untangle_scale(D, delta);
    } else {
        sf = shape_scale(D);
    }
    const R m = s * sf.f;  // s/(2D) (or s/(2Dh))
    R g2[4];
    for (int i = 0; i < 4; ++i) { g2[i] = R(2) * sf.f * t[i] + s * sf.fp * cof[i]; }
    // Terms with an exact-zero factor (off-diagonal 2f, Pm = 0) are left out
    // once the loops are unrolled, instead of being multiplied by 0.
    R H2[16];
    for (int i = 0; i < 4; ++i) {
        for (int j = 0; j < 4; ++j) {
            const R p = Pm(i, j);
            R h = R(2) * sf.fp * (t[i] * cof[j] + cof[i] * t[j]);
            if (i == j) { h = R(2) * sf.f + h; }
            h = h + s * sf.fpp * cof[i] * cof[j];
            if (p != R(0)) { h = h + s * sf.fp * p; }
            H2[i * 4 + j] = h;
        }
    }
    if (kind != kShapeSize) {
        mu = m - R(1);
        for (int i = 0; i < 4; ++i) { g[i] = g2[i]; }
        for (int i = 0; i < 16; ++i) { H[i] = H2[i]; }
        return;
    }
    // shape_size: mu = m^2 - 1 + (D-1)^2, m = s/(2D)
    const R dm1 = D - R(1);
    mu = m * m - R(1) + dm1 * dm1;
    for (int i = 0; i < 4; ++i) { g[i] = R(2) * m * g2[i] + R(2) * dm1 * cof[i]; }
    for (int i = 0; i < 4; ++i) {
        for (int j = 0; j < 4; ++j) {
            const R p = Pm(i, j);
            R h = R(2) * g2[i] * g2[j] + R(2) * m * H2[i * 4 + j] + R(2) * cof[i] * cof[j];
            if (p != R(0)) { h = h + R(2) * dm1 * p; }
            H[i * 4 + j] = h;
        }
    }
}

// Change of the metric mu(T + dT) - mu(T), formed without subtracting two
// metric values, for line searches in working precision: the accept test
// e' <= e0 + tol is a test on the sum of these changes, which fp32 resolves
// even where mu itself is ~1 and a step changes it by 1e-12 (the size term
// of shape_size at small cells).  With s = |T|^2 and D = det T:
//   ds = 2 T:dT + |dT|^2,   dD = cof(T):dT + det(dT)   (exact, no cancellation)
//   shape        d(s/2D) = (ds D - s dD) / (2 D D')
//   shape_size   d(m^2) + d((D-1)^2) = dm (2m + dm) + dD (D' + D - 2)
//   untangle     D -> Dh = (D + r)/2, r = sqrt(D^2 + 4 delta^2), with Dh and
//                dDh in forms free of cancellation for either sign of D.
// Returns the change; dnew = det(T + dT).
// a / b inside the difference forms: fp32 on the device uses the fast
// division (about 2 ulp), ample for an accept test on a sum of changes.
template <class R> EGG_HD R ls_div(R a, R b) { return a / b; }
#if defined(__CUDACC__)
template <> __host__ __device__ __forceinline__ float ls_div<float>(float a, float b)
{
#if defined(__CUDA_ARCH__)
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
#endif

template <class R> EGG_HD R untangle_dh_stable(R D, R r, R delta)
{
    return D >= R(0) ? R(0.5) * (D + r) : ls_div(R(2) * delta * delta, r - D);
}

template <class R> EGG_HD R untangle_ddh(R D, R Dn, R r, R rn, R dD, R delta)
{
    const R q = ls_div(Dn + D, rn + r);
    return (Dn + D >= R(0)) ? R(0.5) * dD * (R(1) + q) : ls_div(R(2) * delta * delta * dD * (R(1) - q), (rn - Dn) * (r - D));
}

// The change from s, D and their exact increments ds, dD.
template <class R> EGG_HD R dmu2_from(int kind, R s, R D, R ds, R dD, R delta, R& dnew)
{
    const R Dn = D + dD;
    dnew = Dn;
    if (kind == kUntangle) {
        const R d2 = R(4) * delta * delta;
        const R r = sqrt(D * D + d2), rn = sqrt(Dn * Dn + d2);
        const R Dh = untangle_dh_stable(D, r, delta), Dhn = untangle_dh_stable(Dn, rn, delta);
        const R dDh = untangle_ddh(D, Dn, r, rn, dD, delta);
        return ls_div(ds * Dh - s * dDh, R(2) * Dh * Dhn);
    }
    const R dm = ls_div(ds * D - s * dD, R(2) * D * Dn);
    if (kind == kShape) { return dm; }
    const R m = ls_div(s, R(2) * D);
    return dm * (R(2) * m + dm) + dD * (Dn + D - R(2));
}

template <class R> EGG_HD R dmu2(int kind, const R t[4], const R dt[4], R delta, R& dnew)
{
    const R s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + t[3] * t[3];
    const R D = t[0] * t[3] - t[1] * t[2];
    const R ds = R(2) * (t[0] * dt[0] + t[1] * dt[1] + t[2] * dt[2] + t[3] * dt[3]) +
                 (dt[0] * dt[0] + dt[1] * dt[1] + dt[2] * dt[2] + dt[3] * dt[3]);
    const R dD = (t[0] * dt[3] + dt[0] * t[3] - t[1] * dt[2] - dt[1] * t[2]) + (dt[0] * dt[3] - dt[1] * dt[2]);
    return dmu2_from(kind, s, D, ds, dD, delta, dnew);
}

// dmu2 for a move of column COL of T = [t0 t1; t2 t3] by (ex, ey), the other
// column fixed: the zero entries of dT are left out of the sums (IEEE
// arithmetic keeps x * 0 and x + 0, so passing zeros would cost instructions),
// and det(dT) = 0.
template <class R, int COL> EGG_HD R dmu2_col(int kind, const R t[4], R ex, R ey, R delta, R& dnew)
{
    const R s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + t[3] * t[3];
    const R D = t[0] * t[3] - t[1] * t[2];
    R ds, dD;
    if constexpr (COL == 0) {
        ds = R(2) * (t[0] * ex + t[2] * ey) + (ex * ex + ey * ey);
        dD = ex * t[3] - t[1] * ey;
    } else {
        ds = R(2) * (t[1] * ex + t[3] * ey) + (ex * ex + ey * ey);
        dD = t[0] * ey - ex * t[2];
    }
    return dmu2_from(kind, s, D, ds, dD, delta, dnew);
}

// Barrier accept policy: shape-type objectives never cross det A <= 0; the
// untangle surrogate accepts any finite energy decrease (src/metric.hpp:855,981).
EGG_HD bool accept_mindet(int kind, double md) { return kind == kUntangle ? true : (md > 0.0); }

// Newton step -H^{-1} g for a 2x2 system with the reference fallbacks
// (src/solve.hpp:32-46): |g| < znorm -> 0; non-finite -> -0.1 g/|g|.
template <class R> EGG_HD void solve2(const R H[4], const R g[2], R x[2])
{
    const R gn = sqrt(g[0] * g[0] + g[1] * g[1]);
    if (gn < Tol<R>::znorm) {
        x[0] = R(0);
        x[1] = R(0);
        return;
    }
    const R det = H[0] * H[3] - H[1] * H[2];
    const R inv = R(1) / det;
    x[0] = -inv * (H[3] * g[0] - H[1] * g[1]);
    x[1] = -inv * (-H[2] * g[0] + H[0] * g[1]);
    if (!(isfinite(x[0]) && isfinite(x[1]))) {
        const R c = R(-0.1) / gn;
        x[0] = c * g[0];
        x[1] = c * g[1];
    }
}

}  // namespace egg_b200
