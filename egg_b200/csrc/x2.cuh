// Two-lane fp32 arithmetic for the packed 2D sweep (sm_100a).
//
// Blackwell issues FADD2 / FMUL2 / FFMA2: one instruction performs the same
// fp32 operation on both halves of a register pair, correctly rounded per
// lane.  The 2D mixed sweep evaluates two corner samples per instruction
// stream this way.  Host builds (the tests' native checks) get per-lane
// equivalents with the same rounding (fmaf for the fused form).
//
// Also here: the per-sample role contributions of a pair of 2D samples
// (value-free: gradient and Hessian contracted per role, as the cell pass
// needs them) and the metric change of a pair of trial samples, both for the
// three objectives.  The formulas are those of metric.cuh:
//   grad = 2 f T + s f' cof,
//   Hess = 2 f I + 2 f' (T cof^T + cof T^T) + s f'' cof cof^T + s f' P,
// written out entry by entry for vec(T) = [t0 t1 t2 t3] = [a b c d],
// cof = [t3, -t2, -t1, t0].
#pragma once

#include "metric.cuh"

#include <cmath>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#define X2_HD __host__ __device__ __forceinline__
#else
struct float2 {
    float x, y;
};
inline float2 make_float2(float a, float b) { return float2 {a, b}; }
#define X2_HD inline
#endif

namespace egg_b200
{

X2_HD float2 p2(float a) { return make_float2(a, a); }

X2_HD float2 add2(float2 a, float2 b)
{
#if defined(__CUDA_ARCH__)
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}

X2_HD float2 mul2(float2 a, float2 b)
{
#if defined(__CUDA_ARCH__)
    return __fmul2_rn(a, b);
#else
    return make_float2(a.x * b.x, a.y * b.y);
#endif
}

// a * b + c, one rounding per lane
X2_HD float2 fma2(float2 a, float2 b, float2 c)
{
#if defined(__CUDA_ARCH__)
    return __ffma2_rn(a, b, c);
#else
    return make_float2(std::fmaf(a.x, b.x, c.x), std::fmaf(a.y, b.y, c.y));
#endif
}

// a - b: b * (-1) + a is exact before its one rounding, so this equals the
// correctly rounded difference.
X2_HD float2 sub2(float2 a, float2 b) { return fma2(b, p2(-1.0f), a); }

X2_HD float2 neg2(float2 a) { return mul2(a, p2(-1.0f)); }

// Per-lane quotient with the same division as the scalar fp32 line search.
X2_HD float2 ldiv2(float2 a, float2 b) { return make_float2(ls_div(a.x, b.x), ls_div(a.y, b.y)); }

// The scale factors of mu = s f(D): 2f, 2f', s f'', s f'.
struct Scale2 {
    float2 twof, A, B, sfp;
};

template <int KIND> X2_HD Scale2 scale2(float2 s, float2 D, float delta)
{
    Scale2 o;
    if constexpr (KIND == kUntangle) {
        const ScaleFn<float> fx = untangle_scale(D.x, delta), fy = untangle_scale(D.y, delta);
        o.twof = make_float2(2.0f * fx.f, 2.0f * fy.f);
        o.A = make_float2(2.0f * fx.fp, 2.0f * fy.fp);
        o.B = mul2(s, make_float2(fx.fpp, fy.fpp));
        o.sfp = mul2(s, make_float2(fx.fp, fy.fp));
    } else {
        // f = 1/(2D): 2f = 1/D, 2f' = -1/D^2, s f'' = s/D^3, s f' = -s/(2D^2)
        const float2 inv = make_float2(1.0f / D.x, 1.0f / D.y);
        const float2 inv2 = mul2(inv, inv);
        const float2 si2 = mul2(s, inv2);
        o.twof = inv;
        o.A = neg2(inv2);
        o.B = mul2(si2, inv);
        o.sfp = mul2(si2, p2(-0.5f));
    }
    return o;
}

// Role contributions of two samples (one per lane), each [gx, gy, hxx, hxy,
// hyy] for the node the sample moves in that role:
//   r1: axis-0 neighbour  (s0 g0, s0 g2, H00, H02, H22)
//   r2: axis-1 neighbour  (s1 g1, s1 g3, H11, H13, H33)
//   r0: corner            (-(r1 + r2) gradient,
//                          H00 + H11 + 2 ss H01, H02 + H13 + ss (H03 + H12), H22 + H33 + 2 ss H23)
// (role_Jb / accumulate_sample of src/patch.hpp:204-320 with W_inv = I).
// s0, s1 are the per-lane sample signs, ss = s0 s1.  Also returns det T and
// the squared column norms (for the cell's shape test).
struct Roles2 {
    float2 r0[5], r1[5], r2[5];
    float2 D, n0, n1;
};

template <int KIND>
X2_HD void roles2(float2 t0, float2 t1, float2 t2, float2 t3, float2 s0, float2 s1, float delta, Roles2& o)
{
    const float2 q0 = mul2(t0, t0), q1 = mul2(t1, t1), q2 = mul2(t2, t2), q3 = mul2(t3, t3);
    const float2 q03 = add2(q0, q3), q12 = add2(q1, q2);
    const float2 s = add2(q03, q12);
    const float2 u = mul2(t0, t3), v = mul2(t1, t2);
    const float2 D = sub2(u, v);
    o.D = D;
    o.n0 = add2(q0, q2);
    o.n1 = add2(q1, q3);
    const Scale2 k = scale2<KIND>(s, D, delta);
    const float2 nsfp = neg2(k.sfp);
    // grad of s f(D)
    float2 g0 = fma2(k.twof, t0, mul2(k.sfp, t3));
    float2 g1 = fma2(k.twof, t1, mul2(nsfp, t2));
    float2 g2 = fma2(k.twof, t2, mul2(nsfp, t1));
    float2 g3 = fma2(k.twof, t3, mul2(k.sfp, t0));
    // Hessian of s f(D): the ten distinct entries
    const float2 A2 = add2(k.A, k.A), nA = neg2(k.A), nB = neg2(k.B);
    const float2 p01 = mul2(t0, t1), p02 = mul2(t0, t2), p13 = mul2(t1, t3), p23 = mul2(t2, t3);
    const float2 d1302 = sub2(p13, p02), d2301 = sub2(p23, p01);
    float2 h00 = fma2(A2, u, fma2(k.B, q3, k.twof));
    float2 h33 = fma2(A2, u, fma2(k.B, q0, k.twof));
    float2 h11 = fma2(neg2(A2), v, fma2(k.B, q2, k.twof));
    float2 h22 = fma2(neg2(A2), v, fma2(k.B, q1, k.twof));
    float2 h01 = fma2(k.A, d1302, mul2(nB, p23));
    float2 h02 = fma2(k.A, d2301, mul2(nB, p13));
    float2 h13 = fma2(nA, d2301, mul2(nB, p02));
    float2 h23 = fma2(nA, d1302, mul2(nB, p01));
    float2 h03 = fma2(k.A, q03, fma2(k.B, u, k.sfp));
    float2 h12 = fma2(nA, q12, fma2(k.B, v, nsfp));
    if constexpr (KIND == kShapeSize) {
        // mu = m^2 - 1 + (D - 1)^2, m = s f:  grad = 2m g + 2(D-1) cof,
        // Hess = 2 g g^T + 2m H + 2 cof cof^T + 2(D-1) P
        const float2 m2 = mul2(s, k.twof);  // 2m
        const float2 dm2 = add2(add2(D, D), p2(-2.0f));  // 2(D-1)
        const float2 two = p2(2.0f);
        auto H = [&](float2 h, float2 gi, float2 gj, float2 cc) { return fma2(m2, h, mul2(two, fma2(gi, gj, cc))); };
        const float2 e00 = H(h00, g0, g0, q3), e11 = H(h11, g1, g1, q2), e22 = H(h22, g2, g2, q1);
        const float2 e33 = H(h33, g3, g3, q0);
        const float2 e01 = H(h01, g0, g1, neg2(p23)), e02 = H(h02, g0, g2, neg2(p13));
        const float2 e13 = H(h13, g1, g3, neg2(p02)), e23 = H(h23, g2, g3, neg2(p01));
        const float2 e03 = add2(H(h03, g0, g3, u), dm2), e12 = sub2(H(h12, g1, g2, v), dm2);
        h00 = e00;
        h11 = e11;
        h22 = e22;
        h33 = e33;
        h01 = e01;
        h02 = e02;
        h13 = e13;
        h23 = e23;
        h03 = e03;
        h12 = e12;
        const float2 ng0 = fma2(m2, g0, mul2(dm2, t3)), ng1 = fma2(m2, g1, mul2(neg2(dm2), t2));
        const float2 ng2 = fma2(m2, g2, mul2(neg2(dm2), t1)), ng3 = fma2(m2, g3, mul2(dm2, t0));
        g0 = ng0;
        g1 = ng1;
        g2 = ng2;
        g3 = ng3;
    }
    const float2 ss = mul2(s0, s1), ss2 = add2(ss, ss);
    o.r1[0] = mul2(s0, g0);
    o.r1[1] = mul2(s0, g2);
    o.r1[2] = h00;
    o.r1[3] = h02;
    o.r1[4] = h22;
    o.r2[0] = mul2(s1, g1);
    o.r2[1] = mul2(s1, g3);
    o.r2[2] = h11;
    o.r2[3] = h13;
    o.r2[4] = h33;
    o.r0[0] = neg2(add2(o.r1[0], o.r2[0]));
    o.r0[1] = neg2(add2(o.r1[1], o.r2[1]));
    o.r0[2] = fma2(ss2, h01, add2(h00, h11));
    o.r0[3] = fma2(ss, add2(h03, h12), add2(h02, h13));
    o.r0[4] = fma2(ss2, h23, add2(h22, h33));
}

// Metric change of two trial samples (one per lane) from their current s, D
// and the exact increments ds, dD of a rank-one move (det dT = 0):
// dmu2_from of metric.cuh in two lanes.  m2 = 2 s f(D) = s/D (shape_size only).
template <int KIND>
X2_HD float2 dmu2_pair(float2 s, float2 D, float2 twoD, float2 m2, float2 ds, float2 dD, float delta, float2& dn)
{
    dn = add2(D, dD);
    if constexpr (KIND == kUntangle) {
        float ax, ay;
        const float rx = dmu2_from<float>(kUntangle, s.x, D.x, ds.x, dD.x, delta, ax);
        const float ry = dmu2_from<float>(kUntangle, s.y, D.y, ds.y, dD.y, delta, ay);
        return make_float2(rx, ry);
    } else {
        const float2 num = fma2(ds, D, mul2(neg2(s), dD));
        const float2 dm = ldiv2(num, mul2(twoD, dn));
        if constexpr (KIND == kShape) { return dm; }
        // d(m^2) + d((D-1)^2) = dm (2m + dm) + dD (D' + D - 2)
        return fma2(dm, add2(m2, dm), mul2(dD, add2(add2(dn, D), p2(-2.0f))));
    }
}

}  // namespace egg_b200
