// Packed-fp32 structured-interior sweep for mixed precision (sm_100a).
//
// Same tile, patch semantics and fp64 safety nets as interior_tile_kernel's
// fp32 path (kernels2d.cuh), rebuilt around Blackwell's two-lane fp32
// instructions (x2.cuh):
//   phase 1  the (CI+2) x (CJ+2) node window is staged in fp64 (for the fp64
//            fallbacks) and, relative to the window's first node, as fp32
//            hi + lo planes: hi holds the top 24 bits of the fp64 offset, lo
//            the rest, so an edge (hi_b - hi_a) + (lo_b - lo_a) is the fp64
//            edge rounded once more -- no fp64 arithmetic or conversion per
//            edge;
//   phase 2  one thread per cell (a second, partial round covers the cells
//            beyond the CTA's CI x CJ threads; one thread per cell in whole
//            warps measured slower, fewer CTAs fitting per SM) evaluates the
//            cell's four samples as two lane pairs (samples 0|1 and 2|3 share
//            their axis-0 edges) and stores the role contributions per
//            corner, the sample dets and the forward edges of its base node
//            for phase 3 -- the corner values in a layout shifted by one cell
//            (below) so that a DOF gathers each row of its cells with one
//            64-bit load;
//   phase 3  one thread per DOF sums its 4 corners, solves, and line-searches
//            its 12 moving samples as 6 lane pairs (cells (ci, 0) | (ci, 1),
//            same role), accepting on summed exact metric changes with the
//            fp64 tolerance.  Trial samples with |det| < kGuard |a0||a1| are
//            redone in fp64 from the fp64 window; DOFs next to a cell with an
//            inverted or badly shaped sample relax entirely in fp64.
// The sample semantics are src/structured_patch.hpp:89-258 and
// src/sweep.hpp:1534-1650, as for the scalar kernels.
#pragma once

#include "kernels2d.cuh"
#include "x2.cuh"

namespace egg_b200
{

template <int CI, int CJ, int NB = 1> struct TileSharedX2 {
    static constexpr int CH = CI + 1, CW = CJ + 1;  // cells staged
    static constexpr int NC = CH * CW;
    static constexpr int PW = CW + 1;                // window row length (nodes)
    static constexpr int PH = CH + 1;                // window rows
    static constexpr int NN = PH * PW;               // window nodes
    static constexpr int NT = CI * CJ;                // threads: one per DOF
    double2 P[NB][NN];                               // fp64 window(s)
    float hx[NN], hy[NN], lx[NN], ly[NN];            // offsets from the first node, hi + lo
    float f0x[NN], f0y[NN], f1x[NN], f1y[NN];        // forward edges along axis 0 / axis 1
    // Corner values of cell c, shifted: g[p][q][c] = (corner 2p+1 of cell c,
    // corner 2p of cell c+1), q = gx, gy, hxx, hxy, hyy; a DOF whose cells
    // are c00, c01 (row 0) and c10, c11 (row 1) takes corners 3 | 2 from
    // g[1][q][c00] and 1 | 0 from g[0][q][c10].
    float2 g[2][5][NC];
    // Sample dets, shifted alike: det[p][c] = (sample 2p of cell c, sample
    // 2p+1 of cell c+1); -inf for a cell with an inverted or badly shaped
    // sample, which sends every DOF around it to the fp64 path.
    float2 det[2][NC];
    uint64_t bar[NB];  // window-copy completion (persistent kernel)
};

// hi = the fp64 value with its mantissa cut to 24 bits (exact in fp32), lo =
// the rest rounded to fp32.
__device__ __forceinline__ void split_hl(double v, float& hi, float& lo)
{
    const double h = __hiloint2double(__double2hiint(v), __double2loint(v) & int(0xE0000000u));
    hi = __double2float_rn(h);
    lo = __double2float_rn(v - h);
}

// Phase 2 of a tile: thread t takes cells t, t + NT, ...  The cell
// (ci, cj) has its base at window node (ci, cj); (r0, c0) is the window's
// first node in the block, (n0, n1) the block's node counts.
template <class S, int KIND>
__device__ __forceinline__ void x2_cells(S& sm, int tid, int r0, int c0, int n0, int n1, float fdelta)
{
    constexpr int CW = S::CW, NC = S::NC, PW = S::PW;
    for (int cell = tid; cell < NC; cell += S::NT) {
        const int ci = cell / CW, cj = cell % CW;
        const bool valid = (r0 + ci <= n0 - 2) && (c0 + cj <= n1 - 2);
        const int a = ci * PW + cj, b = a + 1, c = a + PW, d = c + 1;  // nodes 00, 01, 10, 11
        // edges as lane pairs over the two sides: axis 0 (00->10 | 01->11), axis 1 (00->01 | 10->11)
        const float2 e0x = add2(sub2(make_float2(sm.hx[c], sm.hx[d]), make_float2(sm.hx[a], sm.hx[b])),
                                sub2(make_float2(sm.lx[c], sm.lx[d]), make_float2(sm.lx[a], sm.lx[b])));
        const float2 e0y = add2(sub2(make_float2(sm.hy[c], sm.hy[d]), make_float2(sm.hy[a], sm.hy[b])),
                                sub2(make_float2(sm.ly[c], sm.ly[d]), make_float2(sm.ly[a], sm.ly[b])));
        const float2 e1x = add2(sub2(make_float2(sm.hx[b], sm.hx[d]), make_float2(sm.hx[a], sm.hx[c])),
                                sub2(make_float2(sm.lx[b], sm.lx[d]), make_float2(sm.lx[a], sm.lx[c])));
        const float2 e1y = add2(sub2(make_float2(sm.hy[b], sm.hy[d]), make_float2(sm.hy[a], sm.hy[c])),
                                sub2(make_float2(sm.ly[b], sm.ly[d]), make_float2(sm.ly[a], sm.ly[c])));
        // forward edges for phase 3: the base node's, plus the last column's
        // axis-0 edge and the last row's axis-1 edge
        sm.f0x[a] = e0x.x;
        sm.f0y[a] = e0y.x;
        sm.f1x[a] = e1x.x;
        sm.f1y[a] = e1y.x;
        if (cj == CW - 1) {
            sm.f0x[b] = e0x.y;
            sm.f0y[b] = e0y.y;
        }
        if (ci == S::CH - 1) {
            sm.f1x[c] = e1x.y;
            sm.f1y[c] = e1y.y;
        }
        // shifted stores: lane y of pair p goes to slot cell (.x), lane x to
        // slot cell - 1 (.y), which no DOF reads when cj = 0
        float* gs = reinterpret_cast<float*>(&sm.g[0][0][0]);
        float* ds = reinterpret_cast<float*>(&sm.det[0][0]);
        auto put_g = [&](int p, int q, float2 v) {
            gs[2 * ((p * 5 + q) * NC + cell)] = v.y;
            if (cj > 0) { gs[2 * ((p * 5 + q) * NC + cell - 1) + 1] = v.x; }
        };
        auto put_det = [&](int p, float2 v) {
            ds[2 * (p * NC + cell)] = v.x;
            if (cj > 0) { ds[2 * (p * NC + cell - 1) + 1] = v.y; }
        };
        if (!valid) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                put_g(0, q, p2(0.0f));
                put_g(1, q, p2(0.0f));
            }
            put_det(0, p2(1.0f));
            put_det(1, p2(1.0f));
        } else {
        // corner c receives sample c in role 0, sample c^2 in role 1 and
        // sample c^1 in role 2.  Samples 0 | 1 first, folded at once into the
        // corner pairs 0 | 1 and 2 | 3 so that fewer values stay live.
        const float kb = float(kBadCell * kBadCell);
        float2 G01[5], G23[5], D01, D23;
        bool bad;
        {
            Roles2 P;  // columns (axis-0 side 0 | 1, axis-1 side 0)
            roles2<KIND>(e0x, p2(e1x.x), e0y, p2(e1y.x), p2(1.0f), make_float2(1.0f, -1.0f), fdelta, P);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                G01[q] = make_float2(P.r0[q].x + P.r2[q].y, P.r0[q].y + P.r2[q].x);
                G23[q] = P.r1[q];
            }
            // inverted or badly shaped sample (sine of a corner below kBadCell)
            const float2 bp = fma2(P.D, P.D, neg2(mul2(p2(kb), mul2(P.n0, P.n1))));
            bad = !(P.D.x > 0.0f) || !(P.D.y > 0.0f) || bp.x < 0.0f || bp.y < 0.0f;
            D01 = P.D;
        }
        {
            Roles2 Q;  // samples 2 | 3: columns (axis-0 side 0 | 1, axis-1 side 1)
            roles2<KIND>(e0x, p2(e1x.y), e0y, p2(e1y.y), p2(-1.0f), make_float2(1.0f, -1.0f), fdelta, Q);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                put_g(0, q, add2(G01[q], Q.r1[q]));
                const float2 B = add2(G23[q], Q.r0[q]);
                put_g(1, q, make_float2(B.x + Q.r2[q].y, B.y + Q.r2[q].x));
            }
            const float2 bq = fma2(Q.D, Q.D, neg2(mul2(p2(kb), mul2(Q.n0, Q.n1))));
            bad = bad || !(Q.D.x > 0.0f) || !(Q.D.y > 0.0f) || bq.x < 0.0f || bq.y < 0.0f;
            D23 = Q.D;
        }
        put_det(0, bad ? p2(-INFINITY) : D01);
        put_det(1, bad ? p2(-INFINITY) : D23);
        }
    }
}

// The fp64 fallbacks, out of line: they run for few DOFs, and inlined their
// fp64 temporaries would raise the register demand of the whole kernel.
template <int KIND>
__device__ __noinline__ double2 x2_dof_fp64(const double2* P, int PW, int ti, int tj, double tx, double ty,
                                            double delta, double omega, double2* gout)
{
    return dof_update_fp64<KIND>(P, PW, ti, tj, tx, ty, delta, omega, gout);
}

template <int KIND>
__device__ __noinline__ float x2_guard64(double2 qc, double2 q0, double2 q1, int role, double dx, double dy, double s0,
                                         double s1, double delta, float& dn)
{
    return dmu2_guard64<KIND>(qc, q0, q1, role, dx, dy, s0, s1, delta, dn);
}

// Phase 3 of a tile: the DOF at window node (ti + 1, tj + 1), store slot
// `slot`, from the tile's cell values and its fp64 window P; (txd, tyd) is
// its FAS shift tau (zero outside FAS).  Writes Xout[slot], or the gradient
// to grad_out[slot] in gradient-only mode.
template <class S, int KIND>
__device__ __forceinline__ void x2_dof(S& sm, const double2* __restrict__ P, int ti, int tj, int64_t slot,
                                       double txd, double tyd, double delta, double omega, float fdelta,
                                       double2* __restrict__ Xout, double2* __restrict__ grad_out)
{
    constexpr int CW = S::CW, PW = S::PW;
    const int c00 = ti * CW + tj, c10 = c00 + CW;
    // min det of the four samples the DOF does not move (sample a^3 of the
    // cell whose corner a it is); -inf flags a bad cell
    const float2 d0 = sm.det[0][c00], d1 = sm.det[1][c10];
    const float mdconst = fminf(fminf(d0.x, d0.y), fminf(d1.x, d1.y));
    if (mdconst == -INFINITY) {
        if (grad_out != nullptr) {
            x2_dof_fp64<KIND>(P, PW, ti, tj, txd, tyd, delta, omega, grad_out + slot);
        } else {
            Xout[slot] = x2_dof_fp64<KIND>(P, PW, ti, tj, txd, tyd, delta, omega, nullptr);
        }
        return;
    }
    // corner of each cell: (0,0) -> 3, (0,1) -> 2, (1,0) -> 1, (1,1) -> 0
    float gsum[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const float2 v = add2(sm.g[1][q][c00], sm.g[0][q][c10]);
        gsum[q] = v.x + v.y;
    }
    const float tx = float(txd), ty = float(tyd);
    const float gv[2] = {gsum[0] - tx, gsum[1] - ty};
    if (grad_out != nullptr) {
        grad_out[slot] = make_double2(double(gv[0]), double(gv[1]));
        return;
    }
    const float Hm[4] = {gsum[2], gsum[3], gsum[3], gsum[4]};
    float dlt[2];
    solve2<float>(Hm, gv, dlt);

    // The 12 moving samples as 6 lane pairs: row ci of cells, lanes (ci, 0) |
    // (ci, 1), role r.  A sample's columns are the forward edges F0 at (its
    // cell's base row, base column + (b & 1)) and F1 at (base row + (b >> 1),
    // base column); they are reloaded from shared memory on every trial, which
    // costs less than keeping six pairs' values live across the loop.
    const float kg = float(kGuard * kGuard);
    float alpha = 1.0f, ax_acc = 0.0f, ay_acc = 0.0f;
    bool accepted = false;
    for (int it = 0; it < 10 && !accepted; ++it) {
        const float dx = alpha * dlt[0], dy = alpha * dlt[1];
        const float2 DX = p2(dx), DY = p2(dy);
        const float2 dd = p2(dx * dx + dy * dy);
        float2 dsum2 = p2(0.0f);
        float md = mdconst;
        unsigned guard = 0u;
#pragma unroll
        for (int ci = 0; ci < 2; ++ci) {
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                // per-lane signs of the lane's sample
                float s0l[2], s1l[2];
#pragma unroll
                for (int cj = 0; cj < 2; ++cj) {
                    const int a = (1 - ci) * 2 + (1 - cj);
                    const int b = r == 0 ? a : (r == 1 ? (a ^ 2) : (a ^ 1));
                    s0l[cj] = (b & 2) ? -1.0f : 1.0f;
                    s1l[cj] = (b & 1) ? -1.0f : 1.0f;
                }
                int n0i[2], n1i[2];
#pragma unroll
                for (int cj = 0; cj < 2; ++cj) {
                    const int a = (1 - ci) * 2 + (1 - cj);
                    const int b = r == 0 ? a : (r == 1 ? (a ^ 2) : (a ^ 1));
                    n0i[cj] = (ti + ci) * PW + (tj + cj + (b & 1));
                    n1i[cj] = (ti + ci + (b >> 1)) * PW + (tj + cj);
                }
                // volatile: the loads stay inside the trial loop instead of
                // being hoisted out of it into 48 live registers
                const volatile float* F0x = sm.f0x;
                const volatile float* F0y = sm.f0y;
                const volatile float* F1x = sm.f1x;
                const volatile float* F1y = sm.f1y;
                const float2 t0 = make_float2(F0x[n0i[0]], F0x[n0i[1]]);
                const float2 t2 = make_float2(F0y[n0i[0]], F0y[n0i[1]]);
                const float2 t1 = make_float2(F1x[n1i[0]], F1x[n1i[1]]);
                const float2 t3 = make_float2(F1y[n1i[0]], F1y[n1i[1]]);
                const float2 N0 = fma2(t0, t0, mul2(t2, t2)), N1 = fma2(t1, t1, mul2(t3, t3));
                const float2 Sv = add2(N0, N1);
                const float2 D = fma2(t0, t3, neg2(mul2(t1, t2)));
                float2 ds, dD, n0t, n1t;
                if (r == 1) {  // column 0 += s0 d
                    const float2 k0 = make_float2(s0l[0], s0l[1]);
                    const float2 ex = mul2(k0, DX), ey = mul2(k0, DY);
                    ds = fma2(p2(2.0f), fma2(t0, ex, mul2(t2, ey)), dd);
                    dD = fma2(ex, t3, neg2(mul2(ey, t1)));
                    const float2 cx = add2(t0, ex), cy = add2(t2, ey);
                    n0t = fma2(cx, cx, mul2(cy, cy));
                    n1t = N1;
                } else if (r == 2) {  // column 1 += s1 d
                    const float2 k1 = make_float2(s1l[0], s1l[1]);
                    const float2 ex = mul2(k1, DX), ey = mul2(k1, DY);
                    ds = fma2(p2(2.0f), fma2(t1, ex, mul2(t3, ey)), dd);
                    dD = fma2(t0, ey, neg2(mul2(ex, t2)));
                    const float2 cx = add2(t1, ex), cy = add2(t3, ey);
                    n0t = N0;
                    n1t = fma2(cx, cx, mul2(cy, cy));
                } else {  // corner: column k -= s_k d (det dT = 0)
                    const float2 k0 = make_float2(-s0l[0], -s0l[1]), k1 = make_float2(-s1l[0], -s1l[1]);
                    const float2 e0x = mul2(k0, DX), e0y = mul2(k0, DY), e1x = mul2(k1, DX), e1y = mul2(k1, DY);
                    const float2 dot = add2(fma2(t0, e0x, mul2(t2, e0y)), fma2(t1, e1x, mul2(t3, e1y)));
                    ds = fma2(p2(2.0f), dot, add2(dd, dd));
                    dD = add2(fma2(e0x, t3, neg2(mul2(e0y, t1))), fma2(t0, e1y, neg2(mul2(e1x, t2))));
                    const float2 cx = add2(t0, e0x), cy = add2(t2, e0y), ex2 = add2(t1, e1x), ey2 = add2(t3, e1y);
                    n0t = fma2(cx, cx, mul2(cy, cy));
                    n1t = fma2(ex2, ex2, mul2(ey2, ey2));
                }
                const float2 M2 = KIND == kShapeSize ? ldiv2(Sv, D) : p2(0.0f);
                float2 dn;
                const float2 dm = dmu2_pair<KIND>(Sv, D, add2(D, D), M2, ds, dD, fdelta, dn);
                const float2 gq = fma2(dn, dn, neg2(mul2(p2(kg), mul2(n0t, n1t))));
                const bool gx = gq.x < 0.0f, gy = gq.y < 0.0f;
                if (gx) { guard |= 1u << (ci * 6 + 0 * 3 + r); }
                if (gy) { guard |= 1u << (ci * 6 + 1 * 3 + r); }
                dsum2 = add2(dsum2, make_float2(gx ? 0.0f : dm.x, gy ? 0.0f : dm.y));
                md = fminf(md, fminf(gx ? INFINITY : dn.x, gy ? INFINITY : dn.y));
            }
        }
        float dsum = dsum2.x + dsum2.y;
#pragma unroll 1
        for (int k = 0; guard && k < 12; ++k) {
            if (!((guard >> k) & 1u)) { continue; }
            const int ci = k / 6, cj = (k / 3) % 2, r = k % 3;
            const int a = (1 - ci) * 2 + (1 - cj);
            const int b = (r == 0) ? a : ((r == 1) ? (a ^ 2) : (a ^ 1));
            const int bn0 = b ^ 2, bn1 = b ^ 1;
            float dn;
            dsum += x2_guard64<KIND>(P[(ti + ci + (b >> 1)) * PW + (tj + cj + (b & 1))],
                                       P[(ti + ci + (bn0 >> 1)) * PW + (tj + cj + (bn0 & 1))],
                                       P[(ti + ci + (bn1 >> 1)) * PW + (tj + cj + (bn1 & 1))], r, double(dx),
                                       double(dy), (b & 2) ? -1.0 : 1.0, (b & 1) ? -1.0 : 1.0, delta, dn);
            md = fminf(md, dn);
        }
        dsum -= tx * dx + ty * dy;
        if (isfinite(dsum) && dsum <= float(Tol<double>::energy) && (KIND == kUntangle || md > 0.0f)) {
            ax_acc = dx;
            ay_acc = dy;
            accepted = true;
        } else {
            alpha *= 0.5f;
        }
    }
    double2 out = P[(ti + 1) * PW + (tj + 1)];
    if (accepted) {
        out.x += omega * double(ax_acc);
        out.y += omega * double(ay_acc);
    }
    Xout[slot] = out;
}

// The tile's window: fp64 into P and, relative to its first node, the fp32
// hi + lo planes (threads stride NT over the window nodes).
template <class S>
__device__ __forceinline__ void x2_planes(S& sm, const double2* P, int tid)
{
    const double2 org = P[0];
    for (int k = tid; k < S::NN; k += S::NT) {
        const double2 v = P[k];
        split_hl(v.x - org.x, sm.hx[k], sm.lx[k]);
        split_hl(v.y - org.y, sm.hy[k], sm.ly[k]);
    }
}

template <int CI, int CJ, int MINB, int KIND>
__global__ void __launch_bounds__(TileSharedX2<CI, CJ>::NT, MINB)
  interior_x2_kernel(const double2* __restrict__ Xin, double2* __restrict__ Xout, const Tile2* __restrict__ tiles,
                     const BlockInfo* __restrict__ blocks, const uint8_t* __restrict__ active,
                     const double2* __restrict__ tau, double delta, double omega, double2* __restrict__ grad_out)
{
    using S = TileSharedX2<CI, CJ>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S& sm = *reinterpret_cast<S*>(smem_raw);
    constexpr int NT = S::NT, PW = S::PW, NN = S::NN;
    const float fdelta = float(delta);

    const Tile2 tile = tiles[blockIdx.x];
    const BlockInfo bi = blocks[tile.block];
    const int n0 = bi.n[0], n1 = bi.n[1];
    const int r0 = tile.i0 - 1, c0 = tile.j0 - 1;  // window origin (always inside the block)
    const int tid = threadIdx.x;
    // This thread's DOF, its active flag and tau, read up front so that their
    // latency hides behind phases 1 and 2.
    const int ti = tid / CJ, tj = tid % CJ;
    const int gi = tile.i0 + ti, gj = tile.j0 + tj;
    const int64_t slot = bi.off + int64_t(gi) * n1 + gj;
    const bool mine = tid < CI * CJ && gi <= n0 - 2 && gj <= n1 - 2 && active[slot];
    double2 tv = make_double2(0.0, 0.0);
    if (mine && tau != nullptr) { tv = tau[slot]; }

    // Phase 1: window, fp64 and as fp32 offsets from its first node.
    const double2 org = Xin[bi.off + int64_t(r0) * n1 + c0];
    for (int k = tid; k < NN; k += NT) {
        const int r = k / PW, c = k % PW;
        const int wi = r0 + r, wj = c0 + c;
        double2 v = org;  // outside the block: never part of a valid cell
        if (wi < n0 && wj < n1) { v = Xin[bi.off + int64_t(wi) * n1 + wj]; }
        sm.P[0][k] = v;
        split_hl(v.x - org.x, sm.hx[k], sm.lx[k]);
        split_hl(v.y - org.y, sm.hy[k], sm.ly[k]);
    }
    __syncthreads();
    x2_cells<S, KIND>(sm, tid, r0, c0, n0, n1, fdelta);
    __syncthreads();
    if (mine) { x2_dof<S, KIND>(sm, sm.P[0], ti, tj, slot, tv.x, tv.y, delta, omega, fdelta, Xout, grad_out); }
}

// ---------------------------------------------------------------------------
// Persistent variant: each CTA walks the tile list with stride gridDim.x and
// double-buffers the fp64 window.  While a tile is computed, the TMA engine
// copies the next tile's window rows (cp.async.bulk, one per row, no tensor
// map: rows are contiguous in the store) into the other buffer, completing on
// that buffer's mbarrier.  Every wait is bounded: past kX2WaitLimit polls the
// kernel sets *err, drains its copies in flight (bounded as well) and stops.
// ---------------------------------------------------------------------------
constexpr long long kX2WaitLimit = 1ll << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
    return ok != 0;
}

// Polls until the phase with `parity` completes, at most kX2WaitLimit times.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    for (long long it = 0; it < kX2WaitLimit; ++it) {
        if (mbar_try_wait(bar, parity)) { return true; }
    }
    return false;
}

// One bulk copy global -> this CTA's shared memory, completing `bytes` on bar.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Thread 0: the window rows of tile t into buffer b.  Rows and columns past
// the block's last node are not copied (they feed only invalid cells).  Every
// row starts on a node (16 bytes) and copies whole nodes, as the bulk copy
// requires.
template <class S>
__device__ __forceinline__ void x2_issue_window(S& sm, int b, const double2* Xin, const Tile2* tiles,
                                                const BlockInfo* blocks, int t)
{
    const Tile2 tile = tiles[t];
    const BlockInfo bi = blocks[tile.block];
    const int r0 = tile.i0 - 1, c0 = tile.j0 - 1;
    const int rows = min(S::PH, bi.n[0] - r0), cols = min(S::PW, bi.n[1] - c0);
    const uint32_t row_bytes = uint32_t(cols) * uint32_t(sizeof(double2));
    // order this CTA's earlier generic reads of the buffer before the async writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&sm.bar[b], row_bytes * uint32_t(rows));
    for (int r = 0; r < rows; ++r) {
        bulk_copy_g2s(&sm.P[b][r * S::PW], Xin + bi.off + int64_t(r0 + r) * bi.n[1] + c0, row_bytes, &sm.bar[b]);
    }
}

template <int CI, int CJ, int MINB, int KIND>
__global__ void __launch_bounds__(TileSharedX2<CI, CJ, 2>::NT, MINB)
  interior_x2p_kernel(const double2* __restrict__ Xin, double2* __restrict__ Xout, const Tile2* __restrict__ tiles,
                      int ntiles, const BlockInfo* __restrict__ blocks, const uint8_t* __restrict__ active,
                      const double2* __restrict__ tau, double delta, double omega, double2* __restrict__ grad_out,
                      int* __restrict__ err)
{
    using S = TileSharedX2<CI, CJ, 2>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S& sm = *reinterpret_cast<S*>(smem_raw);
    const float fdelta = float(delta);
    const int tid = threadIdx.x;
    const int ti = tid / CJ, tj = tid % CJ;

    if (tid == 0) {
        mbar_init(&sm.bar[0], 1);
        mbar_init(&sm.bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int t = blockIdx.x;
    if (tid == 0 && t < ntiles) { x2_issue_window(sm, 0, Xin, tiles, blocks, t); }
    bool ok = true;
    int k = 0;
    for (; t < ntiles; t += gridDim.x, ++k) {
        const int b = k & 1;
        // the other buffer was released by the barrier that ended the last tile
        if (tid == 0 && t + int(gridDim.x) < ntiles) {
            x2_issue_window(sm, b ^ 1, Xin, tiles, blocks, t + gridDim.x);
        }
        const Tile2 tile = tiles[t];
        const BlockInfo bi = blocks[tile.block];
        const int n0 = bi.n[0], n1 = bi.n[1];
        const int gi = tile.i0 + ti, gj = tile.j0 + tj;
        const int64_t slot = bi.off + int64_t(gi) * n1 + gj;
        const bool mine = tid < CI * CJ && gi <= n0 - 2 && gj <= n1 - 2 && active[slot];
        double2 tv = make_double2(0.0, 0.0);
        if (mine && tau != nullptr) { tv = tau[slot]; }
        const bool landed = mbar_wait_bounded(&sm.bar[b], uint32_t(k >> 1) & 1u);
        if (landed) { x2_planes(sm, sm.P[b], tid); }
        // one decision for the whole CTA (a thread whose wait ran out must not
        // leave the others at a barrier)
        if (!__syncthreads_and(landed)) {
            ok = false;
            break;
        }
        x2_cells<S, KIND>(sm, tid, tile.i0 - 1, tile.j0 - 1, n0, n1, fdelta);
        __syncthreads();
        if (mine) { x2_dof<S, KIND>(sm, sm.P[b], ti, tj, slot, tv.x, tv.y, delta, omega, fdelta, Xout, grad_out); }
        __syncthreads();
    }
    if (!ok) {
        // a window copy did not complete: flag it and wait (bounded) for the
        // copies this CTA still has in flight before leaving
        if (tid == 0) { atomicExch(err, 1); }
        const int b = k & 1;
        mbar_wait_bounded(&sm.bar[b], uint32_t(k >> 1) & 1u);
        if (t + int(gridDim.x) < ntiles) { mbar_wait_bounded(&sm.bar[b ^ 1], uint32_t((k + 1) >> 1) & 1u); }
    }
}

}  // namespace egg_b200
