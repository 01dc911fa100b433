// 3D TMOP metrics (host + device).
//
//   shape       mu = |T|^2 |cof T|^2 / (9 D^2) - 1                 (src/metric.hpp:199-275)
//   shape_size  mu_shape + (D - 1)^2                               (src/metric.hpp:241-246)
//   untangle    D -> Dh = (D + sqrt(D^2 + 4 delta^2)) / 2          (src/metric.hpp:250-262)
//
// vec(T) row-major, T = A W_inv, A[:,k] = s_k (nbr_k - corner).  Written as
//   mu + 1 = s q F(D) / 9,  s = |T|^2,  C = cof T,  q = |C|^2,  F = 1/D^2 | 1/Dh^2.
//
// A node of a sample moves T along rank-one directions B_i = e_i v^T (row i of
// T changes by v; v = -W^T s for the corner, s_ax W[ax,:] for the axis-ax
// neighbour, src/patch.hpp:204-233).  Along such directions the second
// derivative of det T and of the cofactor vanish (two equal rows), leaving
//   a = T v, c = C v, w_r = T_r x v (row r of T),
//   k_i = C_{i+1}.w_{i+2} - C_{i+2}.w_{i+1},  m_ii = |w_{i+1}|^2 + |w_{i+2}|^2,
//   m_{i,i+1} = -w_i.w_{i+1}  (indices mod 3),
// and with s' = 2a, q' = 2k, q'' = 2m, F' = F_D c, F'' = F_DD c c^T:
//   dmu/dx_i      = (2 a_i q F + 2 s k_i F + s q F_D c_i) / 9
//   d2mu/dx_i dx_j = (2 d_ij |v|^2 q F + 2 s m_ij F + s q F_DD c_i c_j
//                    + 4F (a_i k_j + a_j k_i) + 2 q F_D (a_i c_j + a_j c_i)
//                    + 2 s F_D (k_i c_j + k_j c_i)) / 9
// (+ 2(D-1) c_i and + 2 c_i c_j for shape_size).  This is the node gradient
// and J_b^T H J_b contraction of the reference (src/metric.hpp:756-808 forms
// it by six directional second derivatives) without the 81-entry Hessian.
#pragma once

#include "metric.cuh"

namespace egg_b200
{

template <class R> struct Shared3 {
    R t[9];
    R C[9];
    R D, s, q, F, FD, FDD;
};

template <class R> EGG_HD R det3(const R t[9])
{
    return t[0] * (t[4] * t[8] - t[5] * t[7]) - t[1] * (t[3] * t[8] - t[5] * t[6]) +
           t[2] * (t[3] * t[7] - t[4] * t[6]);
}

template <class R> EGG_HD void cof3(const R t[9], R C[9])
{
    C[0] = t[4] * t[8] - t[5] * t[7];
    C[1] = t[5] * t[6] - t[3] * t[8];
    C[2] = t[3] * t[7] - t[4] * t[6];
    C[3] = t[2] * t[7] - t[1] * t[8];
    C[4] = t[0] * t[8] - t[2] * t[6];
    C[5] = t[1] * t[6] - t[0] * t[7];
    C[6] = t[1] * t[5] - t[2] * t[4];
    C[7] = t[2] * t[3] - t[0] * t[5];
    C[8] = t[0] * t[4] - t[1] * t[3];
}

template <class R> EGG_HD void shared3(int kind, const R t[9], R delta, Shared3<R>& o)
{
    R s = R(0), q = R(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        o.t[i] = t[i];
        s += t[i] * t[i];
    }
    cof3<R>(t, o.C);
#pragma unroll
    for (int i = 0; i < 9; ++i) { q += o.C[i] * o.C[i]; }
    const R D = t[0] * o.C[0] + t[1] * o.C[1] + t[2] * o.C[2];
    o.D = D;
    o.s = s;
    o.q = q;
    if (kind == kUntangle) {
        const R r = sqrt(D * D + R(4) * delta * delta);
        const R Dh = R(0.5) * (D + r);
        const R d1 = Dh / r, d2 = R(2) * delta * delta / (r * r * r);
        const R inv = R(1) / Dh;
        const R inv2 = inv * inv;
        o.F = inv2;
        o.FD = R(-2) * d1 * inv2 * inv;
        o.FDD = R(6) * d1 * d1 * inv2 * inv2 - R(2) * d2 * inv2 * inv;
    } else {
        const R inv = R(1) / D;
        const R inv2 = inv * inv;
        o.F = inv2;
        o.FD = R(-2) * inv2 * inv;
        o.FDD = R(6) * inv2 * inv2;
    }
}

template <class R> EGG_HD R mu3_from(int kind, const Shared3<R>& S)
{
    R mu = S.s * S.q * S.F * R(1.0 / 9.0) - R(1);
    if (kind == kShapeSize) { mu += (S.D - R(1)) * (S.D - R(1)); }
    return mu;
}

template <class R> EGG_HD R mu3_value(int kind, const R t[9], R delta, R& det)
{
    Shared3<R> S;
    shared3<R>(kind, t, delta, S);
    det = S.D;
    return mu3_from<R>(kind, S);
}

// x.v over the entries where v may be nonzero: all three, or only entry ax
// when the caller knows v = v[ax] e_ax.  A known-zero entry is left out of
// the sum rather than multiplied by 0, which IEEE arithmetic would not let
// the compiler drop (ax is a constant once the caller's loop is unrolled).
template <class R> EGG_HD R dot_ax(R x0, R x1, R x2, const R v[3], int ax)
{
    if (ax == 0) { return x0 * v[0]; }
    if (ax == 1) { return x1 * v[1]; }
    if (ax == 2) { return x2 * v[2]; }
    return x0 * v[0] + x1 * v[1] + x2 * v[2];
}

// x.y with entry `skip` of y known to be zero (skip < 0: none).
template <class R> EGG_HD R dot_skip(const R* x, const R* y, int skip)
{
    if (skip == 0) { return x[1] * y[1] + x[2] * y[2]; }
    if (skip == 1) { return x[0] * y[0] + x[2] * y[2]; }
    if (skip == 2) { return x[0] * y[0] + x[1] * y[1]; }
    return x[0] * y[0] + x[1] * y[1] + x[2] * y[2];
}

// Node gradient g[3] and contracted Hessian h[6] = (xx, xy, xz, yy, yz, zz)
// of one sample along the rank-one directions e_i v^T.  ax >= 0 states that
// v = v[ax] e_ax (an axis neighbour with W_inv = I): then w_r = T_r x v has
// a zero entry ax and the terms with zero factors are left out.
template <class R> EGG_HD void role3(int kind, const Shared3<R>& S, const R v[3], R g[3], R h[6], int ax = -1)
{
    const R* t = S.t;
    const R* C = S.C;
    R a[3], c[3], w[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const R* tr = t + 3 * i;
        a[i] = dot_ax(tr[0], tr[1], tr[2], v, ax);
        c[i] = dot_ax(C[3 * i], C[3 * i + 1], C[3 * i + 2], v, ax);
        // w = T_r x v; with v = v[ax] e_ax, entry ax is zero and each other
        // entry keeps its one term in v[ax]
        if (ax == 0) {
            w[i][0] = R(0);
            w[i][1] = tr[2] * v[0];
            w[i][2] = -(tr[1] * v[0]);
        } else if (ax == 1) {
            w[i][0] = -(tr[2] * v[1]);
            w[i][1] = R(0);
            w[i][2] = tr[0] * v[1];
        } else if (ax == 2) {
            w[i][0] = tr[1] * v[2];
            w[i][1] = -(tr[0] * v[2]);
            w[i][2] = R(0);
        } else {
            w[i][0] = tr[1] * v[2] - tr[2] * v[1];
            w[i][1] = tr[2] * v[0] - tr[0] * v[2];
            w[i][2] = tr[0] * v[1] - tr[1] * v[0];
        }
    }
    R k[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
        k[i] = dot_skip(C + 3 * i1, w[i2], ax) - dot_skip(C + 3 * i2, w[i1], ax);
    }
    const R W00 = dot_skip(w[0], w[0], ax), W11 = dot_skip(w[1], w[1], ax), W22 = dot_skip(w[2], w[2], ax);
    const R W01 = dot_skip(w[0], w[1], ax), W12 = dot_skip(w[1], w[2], ax), W02 = dot_skip(w[0], w[2], ax);
    const R m[3][3] = {{W11 + W22, -W01, -W02}, {-W01, W00 + W22, -W12}, {-W02, -W12, W00 + W11}};
    const R vv = dot_ax(v[0], v[1], v[2], v, ax);
    const R s = S.s, q = S.q, F = S.F, FD = S.FD, FDD = S.FDD;
    const R n9 = R(1.0 / 9.0);
    const R dm1x2 = R(2) * (S.D - R(1));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        g[i] = (R(2) * a[i] * q * F + R(2) * s * k[i] * F + s * q * FD * c[i]) * n9;
        if (kind == kShapeSize) { g[i] += dm1x2 * c[i]; }
    }
    int e = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = i; j < 3; ++j) {
            R hij = R(2) * s * m[i][j] * F;
            if (i == j) { hij = R(2) * vv * q * F + hij; }
            hij = hij + s * q * FDD * c[i] * c[j] + R(4) * F * (a[i] * k[j] + a[j] * k[i]) +
                  R(2) * q * FD * (a[i] * c[j] + a[j] * c[i]) + R(2) * s * FD * (k[i] * c[j] + k[j] * c[i]);
            hij *= n9;
            if (kind == kShapeSize) { hij += R(2) * c[i] * c[j]; }
            h[e++] = hij;
        }
    }
}

// Full gradient over vec(T) and the Hessian-vector product H V along an
// arbitrary V (both 9 entries, row-major), from
//   d s = 2 T,  d q = 2 Q with Q = s T - T T^T T  (q = |cof T|^2 is the second
//   invariant of T^T T in 3D),  d D = C,
//   g = (q F ds + s F dq + s q F_D C) / 9,
// differentiated along V (s' = 2 T:V, q' = 2 Q:V, D' = C:V, dC = cof'(T)[V]).
// shape_size adds 2 (D - 1) C and 2 D' C + 2 (D - 1) dC.
template <class R> EGG_HD void mu3_grad(int kind, const Shared3<R>& S, R g[9])
{
    const R* t = S.t;
    R B[9];  // T^T T
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) { B[3 * i + j] = t[i] * t[j] + t[3 + i] * t[3 + j] + t[6 + i] * t[6 + j]; }
    }
    const R qF = S.q * S.F, sF = S.s * S.F, sqFD = S.s * S.q * S.FD;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const R TB = t[3 * i] * B[j] + t[3 * i + 1] * B[3 + j] + t[3 * i + 2] * B[6 + j];
            const R Q = S.s * t[3 * i + j] - TB;
            R v = (R(2) * qF * t[3 * i + j] + R(2) * sF * Q + sqFD * S.C[3 * i + j]) * R(1.0 / 9.0);
            if (kind == kShapeSize) { v += R(2) * (S.D - R(1)) * S.C[3 * i + j]; }
            g[3 * i + j] = v;
        }
    }
}

template <class R> EGG_HD void mu3_hvp(int kind, const Shared3<R>& S, const R V[9], R hv[9])
{
    const R* t = S.t;
    const R* C = S.C;
    R B[9], TtV[9];  // T^T T and T^T V
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            B[3 * i + j] = t[i] * t[j] + t[3 + i] * t[3 + j] + t[6 + i] * t[6 + j];
            TtV[3 * i + j] = t[i] * V[j] + t[3 + i] * V[3 + j] + t[6 + i] * V[6 + j];
        }
    }
    R Q[9], dC[9];
    R a = R(0), qd = R(0), Dd = R(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            const R TB = t[3 * i] * B[j] + t[3 * i + 1] * B[3 + j] + t[3 * i + 2] * B[6 + j];
            Q[3 * i + j] = S.s * t[3 * i + j] - TB;
            dC[3 * i + j] = V[3 * i1 + j1] * t[3 * i2 + j2] + t[3 * i1 + j1] * V[3 * i2 + j2] -
                            V[3 * i1 + j2] * t[3 * i2 + j1] - t[3 * i1 + j2] * V[3 * i2 + j1];
            a += t[3 * i + j] * V[3 * i + j];
            qd += Q[3 * i + j] * V[3 * i + j];
            Dd += C[3 * i + j] * V[3 * i + j];
        }
    }
    const R s = S.s, q = S.q, F = S.F, FD = S.FD, FDD = S.FDD;
    const R sd = R(2) * a;   // s'
    const R qdd = R(2) * qd; // q'
    const R c1 = R(2) * (qdd * F + q * FD * Dd);  // d(qF) * 2
    const R c2 = sd * F + s * FD * Dd;            // d(sF)
    const R c3 = sd * q * FD + s * qdd * FD + s * q * FDD * Dd;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            // (V T^T T + T V^T T + T T^T V)_ij
            R VB = R(0), TVtT = R(0), TTtV = R(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                VB += V[3 * i + k] * B[3 * k + j];
                TVtT += t[3 * i + k] * TtV[3 * j + k];
                TTtV += t[3 * i + k] * TtV[3 * k + j];
            }
            const R ddq = R(2) * (sd * t[3 * i + j] + s * V[3 * i + j] - VB - TVtT - TTtV);
            R v = c1 * t[3 * i + j] + R(2) * q * F * V[3 * i + j] + R(2) * c2 * Q[3 * i + j] + s * F * ddq +
                  c3 * C[3 * i + j] + s * q * FD * dC[3 * i + j];
            v *= R(1.0 / 9.0);
            if (kind == kShapeSize) { v += R(2) * Dd * C[3 * i + j] + R(2) * (S.D - R(1)) * dC[3 * i + j]; }
            hv[3 * i + j] = v;
        }
    }
}

// Change mu(T + dT) - mu(T) without subtracting metric values (see dmu2 in
// metric.cuh): with C = cof T, q = |C|^2 and the exact 3x3 expansions
//   cof(T + dT) = C + N(T, dT) + cof(dT)          (N the mixed cofactor)
//   det(T + dT) = D + C:dT + T:cof(dT) + det(dT),
// mu + 1 = s q F(D) / 9 changes by (d(sq) F' + s q dF) / 9 with
// d(sq) = ds q + s dq + ds dq and dF = F(D') - F(D) in product form.
template <class R> EGG_HD R dmu3(int kind, const R t[9], const R dt[9], R delta, R& dnew)
{
    R C[9], Cd[9];
    cof3<R>(t, C);
    cof3<R>(dt, Cd);
    R s = R(0), ds = R(0), q = R(0), dq = R(0), dD = R(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            const int k = 3 * i + j;
            const R N = dt[3 * i1 + j1] * t[3 * i2 + j2] + t[3 * i1 + j1] * dt[3 * i2 + j2] -
                        dt[3 * i1 + j2] * t[3 * i2 + j1] - t[3 * i1 + j2] * dt[3 * i2 + j1];
            const R dc = N + Cd[k];
            s += t[k] * t[k];
            ds += R(2) * t[k] * dt[k] + dt[k] * dt[k];
            q += C[k] * C[k];
            dq += R(2) * C[k] * dc + dc * dc;
            dD += C[k] * dt[k] + t[k] * Cd[k];
        }
    }
    dD += det3<R>(dt);
    const R D = t[0] * C[0] + t[1] * C[1] + t[2] * C[2];
    const R Dn = D + dD;
    dnew = Dn;
    R x = D, xn = Dn, dx = dD;  // the argument of F = 1/x^2
    if (kind == kUntangle) {
        const R d2 = R(4) * delta * delta;
        const R r = sqrt(D * D + d2), rn = sqrt(Dn * Dn + d2);
        x = untangle_dh_stable(D, r, delta);
        xn = untangle_dh_stable(Dn, rn, delta);
        dx = untangle_ddh(D, Dn, r, rn, dD, delta);
    }
    const R F = ls_div(R(1), x * x), Fn = ls_div(R(1), xn * xn);
    const R dF = -dx * (x + xn) * F * Fn;
    const R dsq = ds * q + s * dq + ds * dq;
    R dm = (dsq * Fn + s * q * dF) * R(1.0 / 9.0);
    if (kind == kShapeSize) { dm += dD * (Dn + D - R(2)); }
    return dm;
}

// A node move along a line changes T by the rank-one alpha u v^T (u the step
// direction, v the node's role vector), so along the line
//   det(T + a u v^T)    = D + a u.(C v)                   (exactly linear)
//   |T + a u v^T|^2     = s + a 2 u.(T v) + a^2 |u|^2 |v|^2
//   |cof(T + a u v^T)|^2 = q + a 2 C:N + a^2 |N|^2,  N = N(T, u v^T)
// (cof of a rank-one matrix vanishes).  LineSample3 holds these coefficients
// for one sample; dmu3_at gives mu(T + a u v^T) - mu(T) from them.
template <class R> struct LineSample3 {
    R D, D1, s, s1, s2, q, q1, q2;
    R n0[3], n1[3], n2[3];  // column norms^2 of T along the line: n0 + a n1 + a^2 n2
};

// ax >= 0 states that v = v[ax] e_ax (see role3): terms with zero factors
// are left out, and N's column ax vanishes.
template <class R>
EGG_HD void line_sample3(const R t[9], const R u[3], const R v[3], LineSample3<R>& L, int ax = -1)
{
    R C[9];
    cof3<R>(t, C);
    L.D = t[0] * C[0] + t[1] * C[1] + t[2] * C[2];
    R s = R(0), q = R(0);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        s += t[k] * t[k];
        q += C[k] * C[k];
    }
    L.s = s;
    L.q = q;
    R Tv[3], Cv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        Tv[i] = dot_ax(t[3 * i], t[3 * i + 1], t[3 * i + 2], v, ax);
        Cv[i] = dot_ax(C[3 * i], C[3 * i + 1], C[3 * i + 2], v, ax);
    }
    const R uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const R vv = dot_ax(v[0], v[1], v[2], v, ax);
    L.D1 = u[0] * Cv[0] + u[1] * Cv[1] + u[2] * Cv[2];
    L.s1 = R(2) * (u[0] * Tv[0] + u[1] * Tv[1] + u[2] * Tv[2]);
    L.s2 = uu * vv;
    R cn = R(0), nn = R(0);
    bool first = true;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (ax == j) { continue; }  // N[i][ax] = 0
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            R N;
            if (ax == j1) {
                N = u[i1] * v[j1] * t[3 * i2 + j2] - t[3 * i1 + j2] * u[i2] * v[j1];
            } else if (ax == j2) {
                N = t[3 * i1 + j1] * u[i2] * v[j2] - u[i1] * v[j2] * t[3 * i2 + j1];
            } else {
                N = u[i1] * v[j1] * t[3 * i2 + j2] + t[3 * i1 + j1] * u[i2] * v[j2] -
                    u[i1] * v[j2] * t[3 * i2 + j1] - t[3 * i1 + j2] * u[i2] * v[j1];
            }
            if (first) {
                cn = C[3 * i + j] * N;
                nn = N * N;
                first = false;
            } else {
                cn += C[3 * i + j] * N;
                nn += N * N;
            }
        }
    }
    L.q1 = R(2) * cn;
    L.q2 = nn;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const R tk2 = t[k] * t[k] + t[3 + k] * t[3 + k] + t[6 + k] * t[6 + k];
        L.n0[k] = tk2;
        if (ax >= 0 && k != ax) {  // column k of T does not move
            L.n1[k] = R(0);
            L.n2[k] = R(0);
            continue;
        }
        const R ut = u[0] * t[k] + u[1] * t[3 + k] + u[2] * t[6 + k];
        L.n1[k] = R(2) * v[k] * ut;
        L.n2[k] = v[k] * v[k] * uu;
    }
}

// mu(T + a u v^T) - mu(T) (difference form, as dmu3) and the new det.
template <class R> EGG_HD R dmu3_at(int kind, const LineSample3<R>& L, R a, R delta, R& dnew)
{
    const R dD = a * L.D1, ds = a * (L.s1 + a * L.s2), dq = a * (L.q1 + a * L.q2);
    const R D = L.D, Dn = D + dD;
    dnew = Dn;
    R x = D, xn = Dn, dx = dD;
    if (kind == kUntangle) {
        const R d2 = R(4) * delta * delta;
        const R r = sqrt(D * D + d2), rn = sqrt(Dn * Dn + d2);
        x = untangle_dh_stable(D, r, delta);
        xn = untangle_dh_stable(Dn, rn, delta);
        dx = untangle_ddh(D, Dn, r, rn, dD, delta);
    }
    const R F = ls_div(R(1), x * x), Fn = ls_div(R(1), xn * xn);
    const R dF = -dx * (x + xn) * F * Fn;
    const R dsq = ds * L.q + L.s * dq + ds * dq;
    R dm = (dsq * Fn + L.s * L.q * dF) * R(1.0 / 9.0);
    if (kind == kShapeSize) { dm += dD * (Dn + D - R(2)); }
    return dm;
}

// Column norms^2 of T + a u v^T (the guard's shape test); with ax >= 0 only
// column ax moves.
template <class R> EGG_HD void line_norms3(const LineSample3<R>& L, R a, R n[3], int ax = -1)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) { n[k] = (ax >= 0 && k != ax) ? L.n0[k] : L.n0[k] + a * (L.n1[k] + a * L.n2[k]); }
}

// Newton step -H^{-1} g for a symmetric 3x3 (packed xx, xy, xz, yy, yz, zz)
// with the reference fallbacks (src/solve.hpp:52-77).
template <class R> EGG_HD void solve3(const R h[6], const R g[3], R x[3])
{
    const R gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (gn < Tol<R>::znorm) {
        x[0] = x[1] = x[2] = R(0);
        return;
    }
    const R H[9] = {h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]};
    const R c00 = H[4] * H[8] - H[5] * H[7], c01 = -(H[3] * H[8] - H[5] * H[6]), c02 = H[3] * H[7] - H[4] * H[6];
    const R det = H[0] * c00 + H[1] * c01 + H[2] * c02;
    const R inv = R(1) / det;
    const R c10 = -(H[1] * H[8] - H[2] * H[7]), c11 = H[0] * H[8] - H[2] * H[6], c12 = -(H[0] * H[7] - H[1] * H[6]);
    const R c20 = H[1] * H[5] - H[2] * H[4], c21 = -(H[0] * H[5] - H[2] * H[3]), c22 = H[0] * H[4] - H[1] * H[3];
    x[0] = -inv * (c00 * g[0] + c10 * g[1] + c20 * g[2]);
    x[1] = -inv * (c01 * g[0] + c11 * g[1] + c21 * g[2]);
    x[2] = -inv * (c02 * g[0] + c12 * g[1] + c22 * g[2]);
    if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]))) {
        const R cc = R(-0.1) / gn;
        x[0] = cc * g[0];
        x[1] = cc * g[1];
        x[2] = cc * g[2];
    }
}

}  // namespace egg_b200
