// 3D sweep kernels of the egg_b200 core (sm_100a).
//
// Store: blocks are dense row-major (n0, n1, n2) node arrays, three doubles
// per node, packed back to back (same conventions as the 2D store).
//
// interior3_kernel: one CTA = a TI x TJ x TK tile of structured-interior DOFs;
// the (TI+2)(TJ+2)(TK+2) node window is staged in shared memory and each thread
// relaxes one DOF over its 64-occurrence patch (8 cells x 8 corner samples,
// src/structured_patch.hpp:89-258): for each of its four roles the 8 samples
// that move it contribute gradient and contracted Hessian (metric3.cuh), the
// 32 samples that do not move it contribute a constant energy and min det;
// then the 3x3 Newton step, <= 10 halvings on the 32 moving samples, omega
// blend (src/sweep.hpp:1534-1650).
#pragma once

#include "entity3.cuh"
#include "kernels2d.cuh"
#include "metric3.cuh"

namespace egg_b200
{

struct Tile3 {
    int32_t block;
    int32_t i0, j0, k0;  // first DOF (logical, >= 1)
};

// Corner-index bit of axis k (axis 0 most significant).
__host__ __device__ constexpr int bit3(int k) { return 4 >> k; }

template <int TI, int TJ, int TK> struct Win3 {
    static constexpr int WI = TI + 2, WJ = TJ + 2, WK = TK + 2;
    static constexpr int N = WI * WJ * WK;
    static constexpr int NC = (WI - 1) * (WJ - 1) * (WK - 1);  // cells of the window
    __device__ static int idx(int u, int v, int w) { return (u * WJ + v) * WK + w; }
    __device__ static int cidx(int u, int v, int w) { return (u * (WJ - 1) + v) * (WK - 1) + w; }
};

template <int TI, int TJ, int TK> struct Tile3Shared {
    double P[3][Win3<TI, TJ, TK>::N];  // node window, SoA per coordinate
};

// Edge vectors of sample b of the cell whose base is window node (bu, bv, bw);
// node `a` of the cell may be replaced by `trial` (a < 0: no substitution).
// A[i][k] = s_k (X[nbr_k] - X[corner])_i, returned row-major in t[9] (fp64).
template <int TI, int TJ, int TK>
__device__ __forceinline__ void edges3(const Tile3Shared<TI, TJ, TK>& sm, int bu, int bv, int bw, int b, int a,
                                       const double trial[3], double t[9])
{
    using W = Win3<TI, TJ, TK>;
    auto node = [&](int c, double p[3]) {
        if (c == a) {
            p[0] = trial[0];
            p[1] = trial[1];
            p[2] = trial[2];
        } else {
            const int id = W::idx(bu + (c >> 2), bv + ((c >> 1) & 1), bw + (c & 1));
            p[0] = sm.P[0][id];
            p[1] = sm.P[1][id];
            p[2] = sm.P[2][id];
        }
    };
    double pc[3];
    node(b, pc);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double pn[3];
        node(b ^ bit3(k), pn);
        const double sk = (b & bit3(k)) ? -1.0 : 1.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) { t[3 * i + k] = sk * (pn[i] - pc[i]); }
    }
}

// fp32 edge matrix of sample b from the window's fp32 forward edges
// fe[(3k + i) * N + node] = (X[node + e_k] - X[node])_i.  Column k of T is
// the forward edge along k at the corner with bit k cleared, so this is
// bitwise the fp32 rounding of edges3's fp64 column: the cache saves each
// sample 12 fp64 loads, 9 subtractions and 9 conversions.
template <int TI, int TJ, int TK>
__device__ __forceinline__ void edges3f(const float* __restrict__ fe, int bu, int bv, int bw, int b, float t[9])
{
    using W = Win3<TI, TJ, TK>;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int c = b & ~bit3(k);
        const int id = W::idx(bu + (c >> 2), bv + ((c >> 1) & 1), bw + (c & 1));
#pragma unroll
        for (int i = 0; i < 3; ++i) { t[3 * i + k] = fe[(3 * k + i) * W::N + id]; }
    }
}

template <class R> __device__ __forceinline__ bool below3(const R t[9], R det, R thr)
{
    R n[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { n[k] = t[k] * t[k] + t[3 + k] * t[3 + k] + t[6 + k] * t[6 + k]; }
    return !(det > R(0)) || det * det < thr * thr * n[0] * n[1] * n[2];
}

// Bit b set: sample b of the cell with base (bu, bv, bw) is inverted or
// badly shaped (below3 at kBadCell), from the fp32 edge cache; the det is
// formed as shared3 forms it (first cofactor row).
template <int TI, int TJ, int TK>
__device__ __forceinline__ unsigned cell_bad3(const float* __restrict__ fe, int bu, int bv, int bw)
{
    unsigned mask = 0u;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        float t[9];
        edges3f<TI, TJ, TK>(fe, bu, bv, bw, b, t);
        const float c0 = t[4] * t[8] - t[5] * t[7];
        const float c1 = t[5] * t[6] - t[3] * t[8];
        const float c2 = t[3] * t[7] - t[4] * t[6];
        const float D = t[0] * c0 + t[1] * c1 + t[2] * c2;
        if (below3<float>(t, D, float(kBadCell))) { mask |= 1u << b; }
    }
    return mask;
}

template <int KIND, class R>
__device__ __forceinline__ void sample3_shared(const double t64[9], double delta, Shared3<R>& S)
{
    R t[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) { t[i] = R(t64[i]); }
    shared3<R>(KIND, t, R(delta), S);
}

// Complete update of one interior DOF at window node (1+ti, 1+tj, 1+tk) in
// working precision R.  Returns false (and leaves `out` untouched) when R is
// float and the patch holds an inverted or badly shaped sample, so the caller
// redoes the DOF in fp64.
// fp64 metric change of one near-degenerate trial sample (cell base
// (bu, bv, bw), corner b, the DOF at corner a moved from pos by d), from the
// staged fp64 positions.  Out of line: it runs rarely and its fp64
// temporaries would otherwise weigh on the fp32 line search's registers.
template <int TI, int TJ, int TK, int KIND>
__device__ __noinline__ float dmu3_guard64(const Tile3Shared<TI, TJ, TK>& sm, int bu, int bv, int bw, int b, int a,
                                           const double pos[3], const double d[3], double delta, float& dn)
{
    const double none[3] = {0.0, 0.0, 0.0};
    const double trial[3] = {pos[0] + d[0], pos[1] + d[1], pos[2] + d[2]};
    double t0[9], t1[9], d0, d1;
    edges3<TI, TJ, TK>(sm, bu, bv, bw, b, -1, none, t0);
    edges3<TI, TJ, TK>(sm, bu, bv, bw, b, a, trial, t1);
    const double m0 = mu3_value<double>(KIND, t0, delta, d0);
    const double m1 = mu3_value<double>(KIND, t1, delta, d1);
    dn = d1 > 0.0 ? fmaxf(float(d1), 1e-38f) : (d1 < 0.0 ? fminf(float(d1), -1e-38f) : 0.0f);
    return float(m1 - m0);
}

template <int TI, int TJ, int TK, int KIND, class R>
__device__ bool dof3_update(const Tile3Shared<TI, TJ, TK>& sm, const float* __restrict__ fe,
                            const uint8_t* __restrict__ cbad, int ti, int tj, int tk, const double tau[3],
                            double delta, double omega, double out[3], bool grad_only = false)
{
    using W = Win3<TI, TJ, TK>;
    const int pid = W::idx(ti + 1, tj + 1, tk + 1);
    const double pos[3] = {sm.P[0][pid], sm.P[1][pid], sm.P[2][pid]};
    R g[3] = {R(0), R(0), R(0)};
    R h[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
    R e0 = R(0), econst = R(0);
    R mdconst = R(INFINITY);
    const double none[3] = {0.0, 0.0, 0.0};
    if constexpr (std::is_same_v<R, float>) {
        // Every sample of the DOF's 8 cells is in its patch (4 move it, 4 do
        // not).  If any is inverted or badly shaped the DOF relaxes in fp64;
        // otherwise the samples that do not move it have positive dets and
        // the fp32 accept test needs nothing else from them (it sums metric
        // changes, and their min det cannot decide the sign of the trial min).
        unsigned bad = 0u;
#pragma unroll
        for (int cell = 0; cell < 8; ++cell) {
            bad |= cbad[W::cidx(ti + (cell >> 2), tj + ((cell >> 1) & 1), tk + (cell & 1))];
        }
        if (bad) { return false; }
    } else {
    // Samples that do not move the DOF: constant energy and det.
#pragma unroll 1
    for (int cell = 0; cell < 8; ++cell) {
        const int ci = cell >> 2, cj = (cell >> 1) & 1, ck = cell & 1;
        const int a = ((1 - ci) << 2) | ((1 - cj) << 1) | (1 - ck);
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            const int b = a ^ (x == 0 ? 7 : (x == 1 ? 6 : (x == 2 ? 5 : 3)));
            Shared3<R> S;
            if constexpr (std::is_same_v<R, float>) {
                float tf[9];
                edges3f<TI, TJ, TK>(fe, ti + ci, tj + cj, tk + ck, b, tf);
                shared3<float>(KIND, tf, float(delta), S);
            } else {
                double t[9];
                edges3<TI, TJ, TK>(sm, ti + ci, tj + cj, tk + ck, b, -1, none, t);
                sample3_shared<KIND, R>(t, delta, S);
            }
            econst += mu3_from<R>(KIND, S);
            mdconst = fmin(mdconst, S.D);
        }
    }
    }
    // Samples that move it: role r (0 corner, 1+k axis-k neighbour).
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll 1
        for (int cell = 0; cell < 8; ++cell) {
            const int ci = cell >> 2, cj = (cell >> 1) & 1, ck = cell & 1;
            const int a = ((1 - ci) << 2) | ((1 - cj) << 1) | (1 - ck);
            const int b = r == 0 ? a : (a ^ bit3(r - 1));
            Shared3<R> S;
            if constexpr (std::is_same_v<R, float>) {
                float tf[9];
                edges3f<TI, TJ, TK>(fe, ti + ci, tj + cj, tk + ck, b, tf);
                shared3<float>(KIND, tf, float(delta), S);
            } else {
                double t[9];
                edges3<TI, TJ, TK>(sm, ti + ci, tj + cj, tk + ck, b, -1, none, t);
                sample3_shared<KIND, R>(t, delta, S);
            }
            e0 += mu3_from<R>(KIND, S);
            R v[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const R sk = (b & bit3(k)) ? R(-1) : R(1);
                v[k] = r == 0 ? -sk : (k == r - 1 ? sk : R(0));
            }
            R gg[3], hh[6];
            role3<R>(KIND, S, v, gg, hh, r - 1);  // r >= 1: v = sk e_(r-1)
#pragma unroll
            for (int q = 0; q < 3; ++q) { g[q] += gg[q]; }
#pragma unroll
            for (int q = 0; q < 6; ++q) { h[q] += hh[q]; }
        }
    }
    e0 += econst;
    const R gv[3] = {g[0] - R(tau[0]), g[1] - R(tau[1]), g[2] - R(tau[2])};
    if (grad_only) {  // gradient-only mode (FAS restriction / tau)
        out[0] = double(gv[0]);
        out[1] = double(gv[1]);
        out[2] = double(gv[2]);
        return true;
    }
    R dl[3];
    solve3<R>(h, gv, dl);
    R alpha = R(1);
    if constexpr (std::is_same_v<R, float>) {
        // fp32: accept on the summed metric changes of the 32 samples the DOF
        // moves, with the fp64 energy tolerance.  The move is rank one along
        // the line, so each sample reduces to a few coefficients
        // (line_sample3) and every step length costs a few flops; two step
        // lengths (alpha, alpha / 2) are tried per pass, in the reference's
        // order.  Near-degenerate trial samples are differenced in fp64.
        const float u[3] = {dl[0], dl[1], dl[2]};
        // pass 0 tries alpha = 1 alone (almost every DOF accepts it); later
        // passes try two step lengths each, 10 in all in the reference's order
        int tried = 0;
#pragma unroll 1
        for (int pass = 0; tried < 10; ++pass) {
            const int nt = (pass == 0 || tried == 9) ? 1 : 2;
            const float al[2] = {alpha, 0.5f * alpha};
            float dsum0 = 0.0f, dsum1 = 0.0f;
            float md0 = mdconst, md1 = mdconst;
            unsigned long long guard = 0ull;  // bit 2 * sample + trial
#pragma unroll
            for (int r = 0; r < 4; ++r) {
#pragma unroll 1
                for (int cell = 0; cell < 8; ++cell) {
                    const int ci = cell >> 2, cj = (cell >> 1) & 1, ck = cell & 1;
                    const int a = ((1 - ci) << 2) | ((1 - cj) << 1) | (1 - ck);
                    const int b = r == 0 ? a : (a ^ bit3(r - 1));
                    float tt[9], v[3];
                    edges3f<TI, TJ, TK>(fe, ti + ci, tj + cj, tk + ck, b, tt);
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float sk = (b & bit3(k)) ? -1.0f : 1.0f;
                        v[k] = r == 0 ? -sk : (k == r - 1 ? sk : 0.0f);
                    }
                    LineSample3<float> L;
                    line_sample3<float>(tt, u, v, L, r - 1);
#pragma unroll
                    for (int tr = 0; tr < 2; ++tr) {
                        if (tr >= nt) { break; }
                        float dn;
                        const float dm = dmu3_at<float>(KIND, L, al[tr], float(delta), dn);
                        float nrm[3];
                        line_norms3<float>(L, al[tr], nrm, r - 1);
                        if (!(fabsf(dn) > 0.0f) ||
                            dn * dn < float(kGuard * kGuard) * nrm[0] * nrm[1] * nrm[2]) {
                            guard |= 1ull << (2 * (r * 8 + cell) + tr);
                        } else if (tr == 0) {
                            dsum0 += dm;
                            md0 = fminf(md0, dn);
                        } else {
                            dsum1 += dm;
                            md1 = fminf(md1, dn);
                        }
                    }
                }
            }
#pragma unroll 1
            for (int bit = 0; guard != 0ull && bit < 64; ++bit) {
                if (!((guard >> bit) & 1ull)) { continue; }
                const int si = bit >> 1, tr = bit & 1;
                const int r = si >> 3, cell = si & 7;
                const int ci = cell >> 2, cj = (cell >> 1) & 1, ck = cell & 1;
                const int a = ((1 - ci) << 2) | ((1 - cj) << 1) | (1 - ck);
                const int b = r == 0 ? a : (a ^ bit3(r - 1));
                const double d3[3] = {double(al[tr] * u[0]), double(al[tr] * u[1]), double(al[tr] * u[2])};
                float dn;
                const float dm = dmu3_guard64<TI, TJ, TK, KIND>(sm, ti + ci, tj + cj, tk + ck, b, a, pos, d3, delta, dn);
                if (tr == 0) {
                    dsum0 += dm;
                    md0 = fminf(md0, dn);
                } else {
                    dsum1 += dm;
                    md1 = fminf(md1, dn);
                }
            }
#pragma unroll
            for (int tr = 0; tr < 2; ++tr) {
                if (tr >= nt) { break; }
                const float d3[3] = {al[tr] * u[0], al[tr] * u[1], al[tr] * u[2]};
                const float ds = tr == 0 ? dsum0 : dsum1, mdt = tr == 0 ? md0 : md1;
                const float dd = ds - (float(tau[0]) * d3[0] + float(tau[1]) * d3[1] + float(tau[2]) * d3[2]);
                if (isfinite(dd) && dd <= float(Tol<double>::energy) && (KIND == kUntangle || mdt > 0.0f)) {
                    out[0] = pos[0] + omega * double(d3[0]);
                    out[1] = pos[1] + omega * double(d3[1]);
                    out[2] = pos[2] + omega * double(d3[2]);
                    return true;
                }
            }
            tried += nt;
            alpha *= nt == 1 ? 0.5f : 0.25f;
        }
    } else {
#pragma unroll 1
    for (int it = 0; it < 10; ++it) {
        const double d[3] = {double(alpha * dl[0]), double(alpha * dl[1]), double(alpha * dl[2])};
        const double trial[3] = {pos[0] + d[0], pos[1] + d[1], pos[2] + d[2]};
        R e = econst;
        R md = mdconst;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
#pragma unroll 1
            for (int cell = 0; cell < 8; ++cell) {
                const int ci = cell >> 2, cj = (cell >> 1) & 1, ck = cell & 1;
                const int a = ((1 - ci) << 2) | ((1 - cj) << 1) | (1 - ck);
                const int b = r == 0 ? a : (a ^ bit3(r - 1));
                double t[9];
                edges3<TI, TJ, TK>(sm, ti + ci, tj + cj, tk + ck, b, a, trial, t);
                R tt[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) { tt[q] = R(t[q]); }
                R det;
                R m = mu3_value<R>(KIND, tt, R(delta), det);
                if constexpr (std::is_same_v<R, float>) {
                    // fp64 re-evaluation of near-degenerate trial samples: the
                    // barrier decision needs the sign of det exactly.
                    if (!(fabsf(det) > 0.0f) || below3<float>(tt, fabsf(det), float(kGuard))) {
                        double d64;
                        m = float(mu3_value<double>(KIND, t, delta, d64));
                        det = d64 > 0.0 ? fmaxf(float(d64), 1e-38f) : (d64 < 0.0 ? fminf(float(d64), -1e-38f) : 0.0f);
                    }
                }
                e += m;
                md = fmin(md, det);
            }
        }
        e -= R(tau[0]) * R(d[0]) + R(tau[1]) * R(d[1]) + R(tau[2]) * R(d[2]);
        if (isfinite(e) && e <= e0 + Tol<R>::energy && (KIND == kUntangle || md > R(0))) {
            out[0] = pos[0] + omega * d[0];
            out[1] = pos[1] + omega * d[1];
            out[2] = pos[2] + omega * d[2];
            return true;
        }
        alpha *= R(0.5);
    }
    }
    out[0] = pos[0];
    out[1] = pos[1];
    out[2] = pos[2];
    return true;
}

template <int TI, int TJ, int TK, int MINB, int KIND, class C>
__global__ void __launch_bounds__(TI* TJ* TK, MINB)
  interior3_kernel(const double* __restrict__ Xin, double* __restrict__ Xout, const Tile3* __restrict__ tiles,
                   const BlockInfo* __restrict__ blocks, const uint8_t* __restrict__ active,
                   const double* __restrict__ tau, double delta, double omega, double* __restrict__ grad_out)
{
    using W = Win3<TI, TJ, TK>;
    __shared__ Tile3Shared<TI, TJ, TK> sm;
    __shared__ float fe[std::is_same_v<C, float> ? 9 * W::N : 1];  // fp32 forward edges (mixed)
    __shared__ uint8_t cbad[std::is_same_v<C, float> ? W::NC : 1];  // per window cell: bad-sample bits (mixed)
    const Tile3 tile = tiles[blockIdx.x];
    const BlockInfo bi = blocks[tile.block];
    const int n0 = bi.n[0], n1 = bi.n[1], n2 = bi.n[2];
    const int u0 = tile.i0 - 1, v0 = tile.j0 - 1, w0 = tile.k0 - 1;
    constexpr int NT = TI * TJ * TK;
    for (int id = threadIdx.x; id < W::N; id += NT) {
        const int u = id / (W::WJ * W::WK), v = (id / W::WK) % W::WJ, w = id % W::WK;
        const int gi = u0 + u, gj = v0 + v, gk = w0 + w;
        double p0 = 0.0, p1 = 0.0, p2 = 0.0;
        if (gi < n0 && gj < n1 && gk < n2) {
            const int64_t node = bi.off + (int64_t(gi) * n1 + gj) * n2 + gk;
            p0 = Xin[3 * node];
            p1 = Xin[3 * node + 1];
            p2 = Xin[3 * node + 2];
        }
        sm.P[0][id] = p0;
        sm.P[1][id] = p1;
        sm.P[2][id] = p2;
    }
    __syncthreads();
    if constexpr (std::is_same_v<C, float>) {
        // forward edge along k of every window node that has a +k neighbour
        for (int id = threadIdx.x; id < W::N; id += NT) {
            const int cu = id / (W::WJ * W::WK), cv = (id / W::WK) % W::WJ, cw = id % W::WK;
            const bool has[3] = {cu + 1 < W::WI, cv + 1 < W::WJ, cw + 1 < W::WK};
            const int step[3] = {W::WJ * W::WK, W::WK, 1};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    fe[(3 * k + i) * W::N + id] = has[k] ? float(sm.P[i][id + step[k]] - sm.P[i][id]) : 0.0f;
                }
            }
        }
        __syncthreads();
        // each window cell's 8 samples checked once for the whole tile (a
        // DOF's patch covers all 8 samples of its 8 cells); cells reaching
        // past the block hold zero positions and are read by no DOF
        for (int c = threadIdx.x; c < W::NC; c += NT) {
            const int cu = c / ((W::WJ - 1) * (W::WK - 1)), cv = (c / (W::WK - 1)) % (W::WJ - 1), cw = c % (W::WK - 1);
            cbad[c] = uint8_t(cell_bad3<TI, TJ, TK>(fe, cu, cv, cw));
        }
        __syncthreads();
    }
    const int ti = threadIdx.x / (TJ * TK), tj = (threadIdx.x / TK) % TJ, tk = threadIdx.x % TK;
    const int gi = tile.i0 + ti, gj = tile.j0 + tj, gk = tile.k0 + tk;
    if (gi > n0 - 2 || gj > n1 - 2 || gk > n2 - 2) { return; }
    const int64_t slot = bi.off + (int64_t(gi) * n1 + gj) * n2 + gk;
    if (!active[slot]) { return; }
    double tv[3] = {0.0, 0.0, 0.0};
    if (tau != nullptr) {
        tv[0] = tau[3 * slot];
        tv[1] = tau[3 * slot + 1];
        tv[2] = tau[3 * slot + 2];
    }
    double out[3];
    const bool go = grad_out != nullptr;
    if (!dof3_update<TI, TJ, TK, KIND, C>(sm, fe, cbad, ti, tj, tk, tv, delta, omega, out, go)) {
        dof3_update<TI, TJ, TK, KIND, double>(sm, nullptr, nullptr, ti, tj, tk, tv, delta, omega, out, go);
    }
    double* dst = go ? grad_out : Xout;
    dst[3 * slot] = out[0];
    dst[3 * slot + 1] = out[1];
    dst[3 * slot + 2] = out[2];
}

// ---------------------------------------------------------------------------
// Stored-patch sweep, 3D (fp64, general W_inv): one thread per DOF.
// ---------------------------------------------------------------------------
struct StoredPatch3 {
    int64_t n;
    const int32_t* slot;
    const int64_t* off;
    const int32_t* gc;
    const int32_t* gn0;
    const int32_t* gn1;
    const int32_t* gn2;
    const int8_t* s0;
    const int8_t* s1;
    const int8_t* s2;
    const int32_t* role;
    const double* W;  // [occ*9] or [9]
    int32_t w_stride;
    const double* wt;
    int32_t wt_stride;
    const int8_t* etag;  // [n] entity tag of each DOF, or NULL (all Free)
    const double* epar;  // [n * EGG_B200_ENTITY_FIELDS] entity records
    int cold;            // first sweep of a run call: parametric entities project in world space
    SoftTable soft;      // directional terms per DOF (off == NULL: none)
    const double* arena; // entity arena (B-spline surfaces)
    double* seeds;       // [n * 2] last foot parameter of each B-spline-surface DOF (NaN: none)
};

__device__ __forceinline__ void assemble_T3(const double* X, int32_t ic, const int32_t in[3], const double s[3],
                                            const double* w, int32_t dslot, const double tr[3], double t[9],
                                            double& detA)
{
    auto ld = [&](int32_t n, double p[3]) {
        if (n == dslot) {
            p[0] = tr[0];
            p[1] = tr[1];
            p[2] = tr[2];
        } else {
            p[0] = X[3 * int64_t(n)];
            p[1] = X[3 * int64_t(n) + 1];
            p[2] = X[3 * int64_t(n) + 2];
        }
    };
    double c[3], A[9];
    ld(ic, c);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double p[3];
        ld(in[k], p);
#pragma unroll
        for (int i = 0; i < 3; ++i) { A[3 * i + k] = s[k] * (p[i] - c[i]); }
    }
    detA = det3(A);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            t[3 * i + k] = A[3 * i] * w[k] + A[3 * i + 1] * w[3 + k] + A[3 * i + 2] * w[6 + k];
        }
    }
}

// Stored-patch sweep, 3D, G lanes per DOF (see stored_patch_kernel): the
// lanes split the DOF's samples and reduce across the group.
template <int KIND, int G, bool CON>
__global__ void stored3_kernel(StoredPatch3 sp, const double* __restrict__ Xin, double* __restrict__ Xout,
                               const double* __restrict__ tau, double delta, double omega, double* __restrict__ grad_out)
{
    const int lane = threadIdx.x & (G - 1);
    const int64_t ngroups = (int64_t(gridDim.x) * blockDim.x) / G;
    const double none[3] = {0, 0, 0};
    for (int64_t d = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G; d < sp.n; d += ngroups) {
        const int32_t slot = sp.slot[d];
        const double pos[3] = {Xin[3 * int64_t(slot)], Xin[3 * int64_t(slot) + 1], Xin[3 * int64_t(slot) + 2]};
        const int64_t p0 = sp.off[d], p1 = sp.off[d + 1];
        double g[3] = {0, 0, 0}, h[6] = {0, 0, 0, 0, 0, 0}, e0 = 0.0;
        for (int64_t p = p0 + lane; p < p1; p += G) {
            const double* w = sp.W + p * sp.w_stride;
            const double s[3] = {double(sp.s0[p]), double(sp.s1[p]), double(sp.s2[p])};
            const int32_t in[3] = {sp.gn0[p], sp.gn1[p], sp.gn2[p]};
            double t[9], detA;
            assemble_T3(Xin, sp.gc[p], in, s, w, -1, none, t, detA);
            Shared3<double> S;
            shared3<double>(KIND, t, delta, S);
            const double wt = sp.wt[p * sp.wt_stride];
            e0 += wt * mu3_from<double>(KIND, S);
            const int role = sp.role[p];
            if (role < 0) { continue; }
            double v[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                v[c] = role == 0 ? -(s[0] * w[c] + s[1] * w[3 + c] + s[2] * w[6 + c]) : s[role - 1] * w[3 * (role - 1) + c];
            }
            double gg[3], hh[6];
            role3<double>(KIND, S, v, gg, hh);
#pragma unroll
            for (int q = 0; q < 3; ++q) { g[q] += wt * gg[q]; }
#pragma unroll
            for (int q = 0; q < 6; ++q) { h[q] += wt * hh[q]; }
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) { g[q] = group_sum<G>(g[q]); }
#pragma unroll
        for (int q = 0; q < 6; ++q) { h[q] = group_sum<G>(h[q]); }
        e0 = group_sum<G>(e0);
        // Directional soft terms (src/sweep.hpp:1307-1327,1491-1512), added
        // entry by entry to the full 3x3 Hessian.
        const int etag = (CON && sp.etag != nullptr) ? int(sp.etag[d]) : 0;
        if (sp.soft.off != nullptr) {
            double H9[9] = {h[0], h[1], h[2], h[1], h[3], h[4], h[2], h[4], h[5]};
            soft_dof_accumulate<3>(sp.soft, d, false, Xin, g, H9, e0);
            h[0] = H9[0];
            h[1] = H9[1];
            h[2] = H9[2];
            h[3] = H9[4];
            h[4] = H9[5];
            h[5] = H9[8];
        }
        double tv[3] = {0, 0, 0};
        if (tau != nullptr) {
            for (int q = 0; q < 3; ++q) { tv[q] = tau[3 * int64_t(slot) + q]; }
            for (int q = 0; q < 3; ++q) {
                g[q] -= tv[q];
                e0 -= tv[q] * pos[q];
            }
        }
        if (grad_out != nullptr) {
            if (lane == 0) {
                for (int q = 0; q < 3; ++q) { grad_out[3 * int64_t(slot) + q] = g[q]; }
            }
            continue;
        }
        // Constrained DOFs (src/sweep.hpp:1286-1403, 1718-1876): the step on
        // the entity's tangent space, damped by omega before the line
        // search, every trial on the entity; a parametric entity after the
        // first sweep of a run call searches in its parameters.
        // CON = false (a level without constrained DOFs) compiles none of it.
        const double* er = sp.epar + (etag != 0 ? d * EGG_B200_ENTITY_FIELDS : 0);
        // A B-spline surface carries its foot parameter from sweep to sweep
        // (src/sweep.hpp:1221-1265): the first sweep of a run call steps on
        // the seeded foot's frame and projects every trial from the seed,
        // which each projection advances; later sweeps search in its
        // parameters, every trial clamped onto the trim polygon
        // (src/sweep.hpp:1820-1832: the clamp applies inside the trim too).
        const bool bsurf = etag == EGG_B200_TAG_BSPLINESURF;
        double seed[2] = {NAN, NAN};
        if (bsurf) {
            seed[0] = sp.seeds[2 * d];
            seed[1] = sp.seeds[2 * d + 1];
        }
        const bool warm_param = (is_param3(etag) || (bsurf && isfinite(seed[0]))) && !sp.cold;
        double dl[3] = {0.0, 0.0, 0.0};
        double qs[2] = {0.0, 0.0}, dq[2] = {0.0, 0.0};
        if (etag == 0) {
            solve3<double>(h, g, dl);
        } else if (bsurf && warm_param) {
            bsurf_dof(kBsurfWarm, er, sp.arena, h, g, pos, omega, 0.0, seed, qs, dq, nullptr, nullptr);
        } else if (bsurf) {
            bsurf_dof(kBsurfCold, er, sp.arena, h, g, pos, omega, 0.0, seed, qs, dq, dl, nullptr);
            for (int q = 0; q < 3; ++q) { dl[q] *= omega; }
        } else if (warm_param) {
            param3_warm_step(etag, er, h, g, pos, omega, qs, dq);
        } else {
            entity3_newton_step(etag, er, h, g, pos, dl);
            for (int q = 0; q < 3; ++q) { dl[q] *= omega; }
        }
        double alpha = 1.0;
        double cur[3] = {pos[0], pos[1], pos[2]};
        for (int it = 0; it < 10; ++it) {
            double tr[3] = {pos[0] + alpha * dl[0], pos[1] + alpha * dl[1], pos[2] + alpha * dl[2]};
            if (bsurf) {
                bsurf_dof(warm_param ? kBsurfWarmTrial : kBsurfColdTrial, er, sp.arena, h, g, pos, omega, alpha,
                          seed, qs, dq, tr, nullptr);
            } else if (warm_param) {
                double qt[2] = {qs[0] + alpha * dq[0], qs[1] + alpha * dq[1]};
                p3_clamp(etag, er, qt);
                p3_eval(etag, er, qt, tr);
            } else if (etag != 0) {
                const double raw[3] = {tr[0], tr[1], tr[2]};
                entity3_project(etag, er, raw, tr);
            }
            double e = 0.0, md = INFINITY;
            for (int64_t p = p0 + lane; p < p1; p += G) {
                const double s[3] = {double(sp.s0[p]), double(sp.s1[p]), double(sp.s2[p])};
                const int32_t in[3] = {sp.gn0[p], sp.gn1[p], sp.gn2[p]};
                double t[9], detA;
                assemble_T3(Xin, sp.gc[p], in, s, sp.W + p * sp.w_stride, slot, tr, t, detA);
                double dd;
                e += sp.wt[p * sp.wt_stride] * mu3_value<double>(KIND, t, delta, dd);
                md = fmin(md, detA);
            }
            e = group_sum<G>(e);
            if (sp.soft.off != nullptr) { e += soft_dof_trial<3>(sp.soft, d, false, Xin, tr); }
            e -= tv[0] * tr[0] + tv[1] * tr[1] + tv[2] * tr[2];
            md = group_min<G>(md);
            if (isfinite(e) && e <= e0 + Tol<double>::energy && (KIND == kUntangle || md > 0.0)) {
                cur[0] = tr[0];
                cur[1] = tr[1];
                cur[2] = tr[2];
                break;
            }
            alpha *= 0.5;
        }
        if (lane == 0) {
            for (int q = 0; q < 3; ++q) {
                Xout[3 * int64_t(slot) + q] = etag != 0 ? cur[q] : pos[q] + omega * (cur[q] - pos[q]);
            }
            if (bsurf) {
                sp.seeds[2 * d] = seed[0];
                sp.seeds[2 * d + 1] = seed[1];
            }
        }
    }
}

// Owner -> non-owner copy refresh, three doubles per node.
__global__ void broadcast3_kernel(double* __restrict__ X, const int32_t* __restrict__ src,
                                  const int32_t* __restrict__ dst, int64_t n)
{
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t s = 3 * int64_t(src[e]), d = 3 * int64_t(dst[e]);
        X[d] = X[s];
        X[d + 1] = X[s + 1];
        X[d + 2] = X[s + 2];
    }
}

// Energy / min det over the canonical cell stencil of the blocks (3D).
template <int KIND>
__global__ void energy_structured3_kernel(EnergyStructured2 es, const double* __restrict__ X, double delta,
                                          double* part_s, double* part_c, double* part_m)
{
    Comp acc {0.0, 0.0};
    double mn = INFINITY;
    int64_t c_lo, c_hi;
    segment_range(es.seg, es.ncell, c_lo, c_hi);
    for (int64_t c = c_lo + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < c_hi;
         c += int64_t(gridDim.x) * blockDim.x) {
        int lo = 0, hi = es.nblocks - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (es.cell_off[mid] <= c) {
                lo = mid;
            } else {
                hi = mid - 1;
            }
        }
        const BlockInfo bi = es.blocks[lo];
        const int64_t lc = c - es.cell_off[lo];
        const int c1 = bi.n[1] - 1, c2 = bi.n[2] - 1;
        const int i = int(lc / (int64_t(c1) * c2)), j = int((lc / c2) % c1), k = int(lc % c2);
        const int32_t base = int32_t(bi.off + (int64_t(i) * bi.n[1] + j) * bi.n[2] + k);
        int32_t nd[8];
#pragma unroll
        for (int a = 0; a < 8; ++a) { nd[a] = base + ((a >> 2) * bi.n[1] + ((a >> 1) & 1)) * bi.n[2] + (a & 1); }
        const double none[3] = {0, 0, 0};
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const int64_t sid = c * 8 + b;
            const double s[3] = {(b & 4) ? -1.0 : 1.0, (b & 2) ? -1.0 : 1.0, (b & 1) ? -1.0 : 1.0};
            const int32_t in[3] = {nd[b ^ 4], nd[b ^ 2], nd[b ^ 1]};
            double t[9], detA;
            assemble_T3(X, nd[b], in, s, es.W + sid * es.w_stride, -1, none, t, detA);
            double dd;
            comp_add(acc, es.wt[sid * es.wt_stride] * mu3_value<double>(KIND, t, delta, dd));
            mn = fmin(mn, detA);
        }
    }
    block_reduce_store(acc, mn, part_s, part_c, part_m);
}

struct EnergyStored3 {
    int64_t n;
    const int32_t* gc;
    const int32_t* gn0;
    const int32_t* gn1;
    const int32_t* gn2;
    const int8_t* s0;
    const int8_t* s1;
    const int8_t* s2;
    const double* W;
    int32_t w_stride;
    const double* wt;
    int32_t wt_stride;
    const int64_t* seg = nullptr;  // per-mesh sample prefix offsets or null
};

template <int KIND>
__global__ void energy_stored3_kernel(EnergyStored3 es, const double* __restrict__ X, double delta, double* part_s,
                                      double* part_c, double* part_m)
{
    Comp acc {0.0, 0.0};
    double mn = INFINITY;
    const double none[3] = {0, 0, 0};
    int64_t i_lo, i_hi;
    segment_range(es.seg, es.n, i_lo, i_hi);
    for (int64_t i = i_lo + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < i_hi;
         i += int64_t(gridDim.x) * blockDim.x) {
        const double s[3] = {double(es.s0[i]), double(es.s1[i]), double(es.s2[i])};
        const int32_t in[3] = {es.gn0[i], es.gn1[i], es.gn2[i]};
        double t[9], detA;
        assemble_T3(X, es.gc[i], in, s, es.W + i * es.w_stride, -1, none, t, detA);
        double dd;
        comp_add(acc, es.wt[i * es.wt_stride] * mu3_value<double>(KIND, t, delta, dd));
        mn = fmin(mn, detA);
    }
    block_reduce_store(acc, mn, part_s, part_c, part_m);
}

// Device metric probe (tests): mu, gradient over vec(T) (9) and the contracted
// Hessian along e_i v^T (6) for n (t, v) pairs.
__global__ void metric3_probe_kernel(int kind, double delta, const double* t, const double* v, int64_t n,
                                     double* mu, double* g9, double* hv)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    Shared3<double> S;
    shared3<double>(kind, t + 9 * i, delta, S);
    mu[i] = mu3_from<double>(kind, S);
    for (int c = 0; c < 3; ++c) {
        const double e[3] = {c == 0 ? 1.0 : 0.0, c == 1 ? 1.0 : 0.0, c == 2 ? 1.0 : 0.0};
        double gg[3], hh[6];
        role3<double>(kind, S, e, gg, hh);
        for (int r = 0; r < 3; ++r) { g9[9 * i + 3 * r + c] = gg[r]; }
    }
    double gg[3];
    role3<double>(kind, S, v + 3 * i, gg, hv + 6 * i);
}

}  // namespace egg_b200
