// 2D sweep kernels of the egg_b200 core (sm_100a).
//
// Store layout: every block is a dense row-major (n0, n1) array of nodes with
// the two coordinates interleaved (double2 per node); blocks are packed back to
// back.  No ghost ring: cross-block reads go to owner slots (stored-patch DOFs)
// or to the block's own refreshed copies of shared interface nodes.
//
// One block-Jacobi sweep (src/sweep.hpp:1938 jacobi_sweep_once) is
//   broadcast_kernel     owner -> non-owner copies on the read buffer
//   interior_tile_kernel structured-interior DOFs (patch synthesized, W_inv = I)
//   stored_patch_kernel  every other moving DOF (ragged stored patch)
// Both sweep kernels read X_in (frozen snapshot) and write X_out.
#pragma once

#include "entity2.cuh"
#include "metric.cuh"
#include "soft.cuh"

#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>

namespace egg_b200
{

struct BlockInfo {
    int64_t off;  // first node slot of the block in the packed store
    int32_t n[3]; // node counts per axis (n[2] = 1 in 2D)
    int32_t pad;
};

struct Tile2 {
    int32_t block;
    int32_t i0;  // first DOF row (logical, >= 1)
    int32_t j0;  // first DOF column
    int32_t pad;
};

// Relative threshold of the fp64 guard in mixed precision: a sample whose
// |det A| < kGuard * |a0| |a1| (sine of the corner angle below 1e-3) is
// re-evaluated in fp64.
constexpr double kGuard = 1e-3;

__device__ __forceinline__ double2 ld2(const double2* p) { return *p; }

// ---------------------------------------------------------------------------
// One sample from its two edge vectors e0 = s0 (n0 - c), e1 = s1 (n1 - c)
// (already signed).  vec(T) = [e0.x, e1.x, e0.y, e1.y] (A[:,k] = e_k, W = I).
// ---------------------------------------------------------------------------
template <class C> struct SampleOut {
    C mu, det;
    C g[4];
    C H[16];
};

template <int KIND, class C>
__device__ __forceinline__ void sample_full_c(C ax, C bx, C ay, C by, C delta, SampleOut<C>& o)
{
    const C t[4] = {ax, bx, ay, by};
    mu_eval<C>(KIND, t, delta, o.mu, o.g, o.H);
    o.det = det2(t);
}

// Full per-sample evaluation from fp64 edge vectors, in working precision C
// (fp64 re-evaluation for near-degenerate samples when C = float).
template <int KIND, class C>
__device__ __forceinline__ void sample_full(double ax, double bx, double ay, double by, double delta,
                                            SampleOut<C>& o)
{
    if constexpr (std::is_same_v<C, double>) {
        sample_full_c<KIND, double>(ax, bx, ay, by, delta, o);
    } else {
        const float fax = float(ax), fbx = float(bx), fay = float(ay), fby = float(by);
        const float d = fax * fby - fbx * fay;
        const float n0 = fax * fax + fay * fay, n1 = fbx * fbx + fby * fby;
        if (d * d < float(kGuard * kGuard) * n0 * n1) {
            SampleOut<double> od;
            sample_full_c<KIND, double>(ax, bx, ay, by, delta, od);
            o.mu = float(od.mu);
            o.det = float(od.det);
            for (int i = 0; i < 4; ++i) { o.g[i] = float(od.g[i]); }
            for (int i = 0; i < 16; ++i) { o.H[i] = float(od.H[i]); }
        } else {
            sample_full_c<KIND, float>(fax, fbx, fay, fby, float(delta), o);
        }
    }
}

// Value + det only (line-search trials), working precision C with fp64 guard.
template <int KIND, class C>
__device__ __forceinline__ C sample_mu_c(C ax, C bx, C ay, C by, C delta, C& det)
{
    const C t[4] = {ax, bx, ay, by};
    det = det2(t);
    return mu_value<C>(KIND, t, delta);
}

// Per-sample contributions to the three nodes a sample moves, without forming
// the full 4x4 metric Hessian: only its 10 distinct entries enter
//   role 1 (axis-0 neighbour)  grad s0 (g0, g2),  jhj (H00, H02, H22)
//   role 2 (axis-1 neighbour)  grad s1 (g1, g3),  jhj (H11, H13, H33)
//   role 0 (corner)            grad -(role1 + role2),
//                              jhj  role1 + role2 + s0 s1 (2 H01, H03 + H12, 2 H23)
// (role_Jb / accumulate_sample of src/patch.hpp:204-320 with W_inv = I).
template <class C> struct RoleOut {
    C mu, det;
    C r[3][5];  // [role 0, 1, 2][gx, gy, hxx, hxy, hyy]
};

template <int KIND, class C>
__device__ __forceinline__ void sample_roles_c(C a, C b, C c, C d, C s0, C s1, C delta, RoleOut<C>& o)
{
    const C t[4] = {a, b, c, d};
    const C cof[4] = {d, -c, -b, a};
    const C D = a * d - b * c;
    const C s = a * a + b * b + c * c + d * d;
    ScaleFn<C> sf = (KIND == kUntangle) ? untangle_scale(D, delta) : shape_scale(D);
    const C m = s * sf.f;
    C g2[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) { g2[i] = C(2) * sf.f * t[i] + s * sf.fp * cof[i]; }
    const C dm1 = D - C(1);
    auto P = [](int i, int j) -> C {
        const int k = i * 4 + j;
        return (k == 3 || k == 12) ? C(1) : ((k == 6 || k == 9) ? C(-1) : C(0));
    };
    // i, j are constants after inlining: the terms whose factor is an exact
    // zero (off-diagonal 2f, P(i, j) = 0) are left out rather than multiplied
    // by 0, which IEEE arithmetic would not let the compiler drop.
    auto H = [&](int i, int j) -> C {
        const C p = P(i, j);
        C h2 = C(2) * sf.fp * (t[i] * cof[j] + cof[i] * t[j]);
        if (i == j) { h2 = C(2) * sf.f + h2; }
        h2 = h2 + s * sf.fpp * cof[i] * cof[j];
        if (p != C(0)) { h2 = h2 + s * sf.fp * p; }
        if (KIND != kShapeSize) { return h2; }
        C h = C(2) * g2[i] * g2[j] + C(2) * m * h2 + C(2) * cof[i] * cof[j];
        if (p != C(0)) { h = h + C(2) * dm1 * p; }
        return h;
    };
    C g[4];
    if (KIND == kShapeSize) {
        o.mu = m * m - C(1) + dm1 * dm1;
#pragma unroll
        for (int i = 0; i < 4; ++i) { g[i] = C(2) * m * g2[i] + C(2) * dm1 * cof[i]; }
    } else {
        o.mu = m - C(1);
#pragma unroll
        for (int i = 0; i < 4; ++i) { g[i] = g2[i]; }
    }
    o.det = D;
    const C h00 = H(0, 0), h01 = H(0, 1), h02 = H(0, 2), h03 = H(0, 3), h11 = H(1, 1);
    const C h12 = H(1, 2), h13 = H(1, 3), h22 = H(2, 2), h23 = H(2, 3), h33 = H(3, 3);
    o.r[1][0] = s0 * g[0];
    o.r[1][1] = s0 * g[2];
    o.r[1][2] = h00;
    o.r[1][3] = h02;
    o.r[1][4] = h22;
    o.r[2][0] = s1 * g[1];
    o.r[2][1] = s1 * g[3];
    o.r[2][2] = h11;
    o.r[2][3] = h13;
    o.r[2][4] = h33;
    const C ss = s0 * s1;
    o.r[0][0] = -(o.r[1][0] + o.r[2][0]);
    o.r[0][1] = -(o.r[1][1] + o.r[2][1]);
    o.r[0][2] = h00 + h11 + C(2) * ss * h01;
    o.r[0][3] = h02 + h13 + ss * (h03 + h12);
    o.r[0][4] = h22 + h33 + C(2) * ss * h23;
}

// Role contributions from fp64 edge vectors in working precision C, with the
// fp64 re-evaluation of near-degenerate samples when C = float.
template <int KIND, class C>
__device__ __forceinline__ void sample_roles(double ax, double bx, double ay, double by, double s0, double s1,
                                             double delta, RoleOut<C>& o)
{
    if constexpr (std::is_same_v<C, double>) {
        sample_roles_c<KIND, double>(ax, bx, ay, by, s0, s1, delta, o);
    } else {
        const float fax = float(ax), fbx = float(bx), fay = float(ay), fby = float(by);
        const float d = fax * fby - fbx * fay;
        const float n0 = fax * fax + fay * fay, n1 = fbx * fbx + fby * fby;
        if (d * d < float(kGuard * kGuard) * n0 * n1) {
            RoleOut<double> od;
            sample_roles_c<KIND, double>(ax, bx, ay, by, s0, s1, delta, od);
            o.mu = float(od.mu);
            o.det = float(od.det);
#pragma unroll
            for (int r = 0; r < 3; ++r) {
#pragma unroll
                for (int q = 0; q < 5; ++q) { o.r[r][q] = float(od.r[r][q]); }
            }
        } else {
            sample_roles_c<KIND, float>(fax, fbx, fay, fby, float(s0), float(s1), float(delta), o);
        }
    }
}

// ---------------------------------------------------------------------------
// Owner -> non-owner copy refresh (src/structured_halo.hpp:197 fused_halo_broadcast).
// ---------------------------------------------------------------------------
__global__ void broadcast2_kernel(double2* __restrict__ X, const int32_t* __restrict__ src,
                                  const int32_t* __restrict__ dst, int64_t n)
{
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
         e += int64_t(gridDim.x) * blockDim.x) {
        X[dst[e]] = X[src[e]];
    }
}

// ---------------------------------------------------------------------------
// Fused structured-interior sweep.  One CTA = one tile of (CI-1) x (CJ-1)
// DOFs; CI*CJ threads.  Phase 1 stages the (CI+1) x (CJ+1) node window in
// shared memory; phase 2 evaluates each of the CI*CJ cells' four corner
// samples ONCE (value, det, gradient and the role-contracted Hessian for the
// three nodes each sample moves) - the reference re-evaluates every sample
// for each of the 4 DOFs that share it; phase 3 gathers the 16-occurrence
// patch of each DOF from its 4 cells, takes the 2x2 Newton step, backtracks
// (<= 10 halvings) on the patch energy with the node substituted, applies
// the omega blend and writes X_out.  Patch semantics follow
// src/structured_patch.hpp:89-258 and src/sweep.hpp:1534-1650.
// ---------------------------------------------------------------------------
// Whether the fp32 line search reads T from phase 2's cell edges.  Measured
// on B200: faster for shape (+1-2%) and untangle; shape_size runs 4-5%
// slower with it (its line search keeps more values live, and the hoisted
// edge loads spill), so it forms T from the staged positions instead.
template <int KIND, class C> constexpr bool kEdgeCache2 = std::is_same_v<C, float> && KIND != kShapeSize;

template <int CI, int CJ, class C, int KIND> struct TileShared2 {
    static constexpr int NC = CI * CJ;
    // fp32 cell edges for the mixed line search (one slot otherwise)
    static constexpr int NE = kEdgeCache2<KIND, C> ? NC : 1;
    // sample values: only the fp64 accept test reads them (one slot otherwise)
    static constexpr int NM = std::is_same_v<C, double> ? NC : 1;
    double2 P[(CI + 1) * (CJ + 1)];
    C mu[4][NM];
    C det[4][NC];
    C gh[4][5][NC];  // per local corner a: gx, gy, hxx, hxy, hyy
    float2 E[4][NE];  // axis-0 edge at column side 0, 1; axis-1 edge at row side 0, 1
    uint8_t bad[NC]; // cell holds an inverted or badly shaped sample
};

// Mixed precision: a DOF whose patch touches a cell with an inverted sample or
// a corner angle below asin(kBadCell) is relaxed entirely in fp64 (patch,
// Newton step and line search), since accept/reject decisions next to such
// cells are ill-conditioned in fp32.
constexpr double kBadCell = 0.1;

// Complete fp64 update of the DOF at window node (ti+1, tj+1): 16-occurrence
// patch (W_inv = I) evaluated from the staged positions, 2x2 Newton step,
// <= 10 halvings, omega blend.  Same semantics as the shared-sample path.
template <int KIND>
__device__ double2 dof_update_fp64(const double2* __restrict__ P, int PW, int ti, int tj, double tx, double ty,
                                   double delta, double omega, double2* gout = nullptr)
{
    const double2 pos = P[(ti + 1) * PW + (tj + 1)];
    double g0 = 0, g1 = 0, hxx = 0, hxy = 0, hyy = 0, e0 = 0;
    auto node = [&](int u, int v) { return P[(ti + u) * PW + (tj + v)]; };
#pragma unroll 1
    for (int cell = 0; cell < 4; ++cell) {
        const int ci = cell >> 1, cj = cell & 1;
        const int a = (1 - ci) * 2 + (1 - cj);
#pragma unroll 1
        for (int b = 0; b < 4; ++b) {
            const double s0 = (b & 2) ? -1.0 : 1.0, s1 = (b & 1) ? -1.0 : 1.0;
            const double2 pc = node(ci + (b >> 1), cj + (b & 1));
            const int b0 = b ^ 2, b1 = b ^ 1;
            const double2 p0 = node(ci + (b0 >> 1), cj + (b0 & 1));
            const double2 p1 = node(ci + (b1 >> 1), cj + (b1 & 1));
            SampleOut<double> o;
            sample_full_c<KIND, double>(s0 * (p0.x - pc.x), s1 * (p1.x - pc.x), s0 * (p0.y - pc.y),
                                        s1 * (p1.y - pc.y), delta, o);
            e0 += o.mu;
            if (b == a) {
                g0 -= s0 * o.g[0] + s1 * o.g[1];
                g1 -= s0 * o.g[2] + s1 * o.g[3];
                hxx += o.H[0] + o.H[5] + s0 * s1 * (o.H[1] + o.H[4]);
                hxy += o.H[2] + o.H[7] + s0 * s1 * (o.H[3] + o.H[6]);
                hyy += o.H[10] + o.H[15] + s0 * s1 * (o.H[11] + o.H[14]);
            } else if (b0 == a) {
                g0 += s0 * o.g[0];
                g1 += s0 * o.g[2];
                hxx += o.H[0];
                hxy += o.H[2];
                hyy += o.H[10];
            } else if (b1 == a) {
                g0 += s1 * o.g[1];
                g1 += s1 * o.g[3];
                hxx += o.H[5];
                hxy += o.H[7];
                hyy += o.H[15];
            }
        }
    }
    const double gv[2] = {g0 - tx, g1 - ty};
    if (gout != nullptr) {
        *gout = make_double2(gv[0], gv[1]);
        return pos;
    }
    const double Hm[4] = {hxx, hxy, hxy, hyy};
    double dl[2];
    solve2<double>(Hm, gv, dl);
    double alpha = 1.0;
#pragma unroll 1
    for (int it = 0; it < 10; ++it) {
        const double dx = alpha * dl[0], dy = alpha * dl[1];
        const double2 tr = make_double2(pos.x + dx, pos.y + dy);
        double e = 0.0, md = INFINITY;
#pragma unroll 1
        for (int cell = 0; cell < 4; ++cell) {
            const int ci = cell >> 1, cj = cell & 1;
            const int a = (1 - ci) * 2 + (1 - cj);
#pragma unroll 1
            for (int b = 0; b < 4; ++b) {
                const double s0 = (b & 2) ? -1.0 : 1.0, s1 = (b & 1) ? -1.0 : 1.0;
                const int b0 = b ^ 2, b1 = b ^ 1;
                const double2 pc = (b == a) ? tr : node(ci + (b >> 1), cj + (b & 1));
                const double2 p0 = (b0 == a) ? tr : node(ci + (b0 >> 1), cj + (b0 & 1));
                const double2 p1 = (b1 == a) ? tr : node(ci + (b1 >> 1), cj + (b1 & 1));
                double d;
                e += sample_mu_c<KIND, double>(s0 * (p0.x - pc.x), s1 * (p1.x - pc.x), s0 * (p0.y - pc.y),
                                               s1 * (p1.y - pc.y), delta, d);
                md = fmin(md, d);
            }
        }
        e -= tx * dx + ty * dy;
        if (isfinite(e) && e <= e0 + Tol<double>::energy && (KIND == kUntangle || md > 0.0)) {
            return make_double2(pos.x + omega * dx, pos.y + omega * dy);
        }
        alpha *= 0.5;
    }
    return pos;
}

// fp64 metric change of one near-degenerate trial sample, from the staged
// fp64 positions of its corner qc and neighbours q0, q1; the moving node
// (role 0 corner, 1 axis-0 neighbour, 2 axis-1 neighbour) is displaced by
// (dx, dy).  Called from a separate loop after the fp32 pass, so its fp64
// temporaries do not weigh on the fp32 line search's registers.
template <int KIND>
__device__ float dmu2_guard64(double2 qc, double2 q0, double2 q1, int role, double dx, double dy,
                                           double s0, double s1, double delta, float& dn)
{
    double d0, d1;
    const double m0 = sample_mu_c<KIND, double>(s0 * (q0.x - qc.x), s1 * (q1.x - qc.x), s0 * (q0.y - qc.y),
                                                s1 * (q1.y - qc.y), delta, d0);
    if (role == 0) {
        qc.x += dx;
        qc.y += dy;
    } else if (role == 1) {
        q0.x += dx;
        q0.y += dy;
    } else {
        q1.x += dx;
        q1.y += dy;
    }
    const double m1 = sample_mu_c<KIND, double>(s0 * (q0.x - qc.x), s1 * (q1.x - qc.x), s0 * (q0.y - qc.y),
                                                s1 * (q1.y - qc.y), delta, d1);
    dn = d1 > 0.0 ? fmaxf(float(d1), 1e-38f) : (d1 < 0.0 ? fminf(float(d1), -1e-38f) : 0.0f);
    return float(m1 - m0);
}

template <int CI, int CJ, int MINB, int KIND, class C, int FD>
__global__ void __launch_bounds__(CI* CJ, MINB)
  interior_tile_kernel(const double2* __restrict__ Xin, double2* __restrict__ Xout,
                       const Tile2* __restrict__ tiles, const BlockInfo* __restrict__ blocks,
                       const uint8_t* __restrict__ active, const double2* __restrict__ tau,
                       double delta, double omega, double2* __restrict__ grad_out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // FD = 0: CI x CJ cells per CTA, one per thread, for their (CI-1) x (CJ-1)
    // interior DOFs.  FD = 1: CI x CJ DOFs per CTA, one per thread, over the
    // (CI+1) x (CJ+1) cells around them, so no thread idles in phase 3.
    constexpr int NT = CI * CJ;
    constexpr int CH = FD ? CI + 1 : CI, CW = FD ? CJ + 1 : CJ;  // cells staged
    using S = TileShared2<CH, CW, C, KIND>;
    S& sm = *reinterpret_cast<S*>(smem_raw);
    constexpr int NC = CH * CW;
    constexpr int PW = CW + 1;

    const Tile2 tile = tiles[blockIdx.x];
    const BlockInfo bi = blocks[tile.block];
    const int n0 = bi.n[0], n1 = bi.n[1];
    const int r0 = tile.i0 - 1, c0 = tile.j0 - 1;  // node window origin
    const int tid = threadIdx.x;

    // Phase 1: node window.
    for (int k = tid; k < (CH + 1) * PW; k += NT) {
        const int r = k / PW, c = k % PW;
        const int gi = r0 + r, gj = c0 + c;
        double2 v = make_double2(0.0, 0.0);
        if (gi < n0 && gj < n1) { v = Xin[bi.off + int64_t(gi) * n1 + gj]; }
        sm.P[k] = v;
    }
    __syncthreads();

    // Phase 2: cell (ci, cj) with base node window (ci, cj); thread = cell
    // (a second round for the extra cells of an FD tile).  Each thread
    // accumulates the role contributions of its cell's four samples per
    // corner in registers and stores them once to column `cell` of the shared
    // cell arrays.
    for (int cell = tid; cell < NC; cell += NT) {
        const int ci = cell / CW, cj = cell % CW;
        const bool valid = (r0 + ci <= n0 - 2) && (c0 + cj <= n1 - 2);
        bool bad = false;
        C acc[4][5];  // role contributions per cell corner, stored once below
#pragma unroll
        for (int a = 0; a < 4; ++a) {
#pragma unroll
            for (int q = 0; q < 5; ++q) { acc[a][q] = C(0); }
            if constexpr (std::is_same_v<C, double>) { sm.mu[a][cell] = C(0); }
            sm.det[a][cell] = C(1);
        }
        if (valid) {
            // The cell's four edges.  Sample b's columns are the axis-0 edge on
            // side (b & 1) and the axis-1 edge on side (b >> 1): the sample
            // signs cancel the edge orientation exactly, so T is bitwise the
            // per-sample s_k (n_k - c).
            const double2 p00 = sm.P[ci * PW + cj], p01 = sm.P[ci * PW + cj + 1];
            const double2 p10 = sm.P[(ci + 1) * PW + cj], p11 = sm.P[(ci + 1) * PW + cj + 1];
            const double e0x[2] = {p10.x - p00.x, p11.x - p01.x}, e0y[2] = {p10.y - p00.y, p11.y - p01.y};
            const double e1x[2] = {p01.x - p00.x, p11.x - p10.x}, e1y[2] = {p01.y - p00.y, p11.y - p10.y};
            if constexpr (kEdgeCache2<KIND, C>) {
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    sm.E[k][cell] = make_float2(float(e0x[k]), float(e0y[k]));
                    sm.E[2 + k][cell] = make_float2(float(e1x[k]), float(e1y[k]));
                }
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const double s0 = (b & 2) ? -1.0 : 1.0;
                const double s1 = (b & 1) ? -1.0 : 1.0;
                const double ax = e0x[b & 1], bx = e1x[b >> 1];
                const double ay = e0y[b & 1], by = e1y[b >> 1];
                if constexpr (std::is_same_v<C, float>) {
                    // the fp32 / fp64 split needs only a coarse shape test
                    const float fax = float(ax), fbx = float(bx), fay = float(ay), fby = float(by);
                    const float dd = fax * fby - fbx * fay;
                    const float nn = (fax * fax + fay * fay) * (fbx * fbx + fby * fby);
                    bad = bad || !(dd > 0.0f) || dd * dd < float(kBadCell * kBadCell) * nn;
                }
                RoleOut<C> o;
                sample_roles<KIND, C>(ax, bx, ay, by, s0, s1, delta, o);
                if constexpr (std::is_same_v<C, double>) { sm.mu[b][cell] = o.mu; }  // fp32 accepts on differences
                sm.det[b][cell] = o.det;
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    acc[b][q] += o.r[0][q];
                    acc[b ^ 2][q] += o.r[1][q];
                    acc[b ^ 1][q] += o.r[2][q];
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
#pragma unroll
            for (int q = 0; q < 5; ++q) { sm.gh[a][q][cell] = acc[a][q]; }
        }
        sm.bad[cell] = bad ? 1 : 0;
    }
    __syncthreads();

    // Phase 3: DOFs.
    constexpr int DI = FD ? CI : CI - 1, DJ = FD ? CJ : CJ - 1;
    if (tid >= DI * DJ) { return; }
    const int ti = tid / DJ, tj = tid % DJ;
    const int gi = tile.i0 + ti, gj = tile.j0 + tj;
    if (gi > n0 - 2 || gj > n1 - 2) { return; }
    const int64_t slot = bi.off + int64_t(gi) * n1 + gj;
    if (!active[slot]) { return; }

    C g0 = 0, g1 = 0, hxx = 0, hxy = 0, hyy = 0, e0 = 0, econst = 0;
    C mdconst = C(INFINITY);
#pragma unroll
    for (int ci = 0; ci < 2; ++ci) {
#pragma unroll
        for (int cj = 0; cj < 2; ++cj) {
            const int cell = (ti + ci) * CW + (tj + cj);
            const int a = (1 - ci) * 2 + (1 - cj);
            g0 += sm.gh[a][0][cell];
            g1 += sm.gh[a][1][cell];
            hxx += sm.gh[a][2][cell];
            hxy += sm.gh[a][3][cell];
            hyy += sm.gh[a][4][cell];
            if constexpr (std::is_same_v<C, double>) {  // energies: the fp64 accept test only
                e0 += (sm.mu[0][cell] + sm.mu[1][cell]) + (sm.mu[2][cell] + sm.mu[3][cell]);
                econst += sm.mu[a ^ 3][cell];
            }
            mdconst = fmin(mdconst, sm.det[a ^ 3][cell]);
        }
    }
    C tx = 0, ty = 0;
    double txd = 0.0, tyd = 0.0;
    if (tau != nullptr) {
        const double2 tv = tau[slot];
        txd = tv.x;
        tyd = tv.y;
        tx = C(tv.x);
        ty = C(tv.y);
    }
    if constexpr (std::is_same_v<C, float>) {
        const int c00 = ti * CW + tj;
        if (sm.bad[c00] | sm.bad[c00 + 1] | sm.bad[c00 + CW] | sm.bad[c00 + CW + 1]) {
            if (grad_out != nullptr) {
                dof_update_fp64<KIND>(sm.P, PW, ti, tj, txd, tyd, delta, omega, grad_out + slot);
            } else {
                Xout[slot] = dof_update_fp64<KIND>(sm.P, PW, ti, tj, txd, tyd, delta, omega);
            }
            return;
        }
    }
    const C gv[2] = {g0 - tx, g1 - ty};
    if (grad_out != nullptr) {  // gradient-only mode (FAS restriction / tau)
        grad_out[slot] = make_double2(double(gv[0]), double(gv[1]));
        return;
    }
    const C Hm[4] = {hxx, hxy, hxy, hyy};
    C dlt[2];
    solve2<C>(Hm, gv, dlt);

    // Neighbour offsets relative to the DOF, in working precision.
    const double2 pos = sm.P[(ti + 1) * PW + (tj + 1)];
    C rx[3][3], ry[3][3];
#pragma unroll
    for (int u = 0; u < 3; ++u) {
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double2 q = sm.P[(ti + u) * PW + (tj + v)];
            rx[u][v] = C(q.x - pos.x);
            ry[u][v] = C(q.y - pos.y);
        }
    }

    C alpha = C(1);
    C ax_acc = C(0), ay_acc = C(0);
    bool accepted = false;
    if constexpr (std::is_same_v<C, float>) {
        // fp32: accept on the summed metric changes of the 12 samples the DOF
        // moves (dmu2, free of the cancellation of e' - e0 where mu ~ 1), with
        // the fp64 energy tolerance; near-degenerate trial samples are
        // differenced in fp64.
        for (int it = 0; it < 10 && !accepted; ++it) {
            const float dx = alpha * dlt[0], dy = alpha * dlt[1];
            float dsum = 0.0f;
            float md = mdconst;
            unsigned guard = 0u;
#pragma unroll
            for (int ci = 0; ci < 2; ++ci) {
#pragma unroll
                for (int cj = 0; cj < 2; ++cj) {
                    const int a = (1 - ci) * 2 + (1 - cj);
                    const int cell = (ti + ci) * CW + (tj + cj);
#pragma unroll
                    for (int r = 0; r < 3; ++r) {
                        const int b = (r == 0) ? a : ((r == 1) ? (a ^ 2) : (a ^ 1));
                        const float s0 = (b & 2) ? -1.0f : 1.0f;
                        const float s1 = (b & 1) ? -1.0f : 1.0f;
                        float t[4];
                        if constexpr (kEdgeCache2<KIND, C>) {
                            // T of sample b: the cell's fp32 edges from phase 2
                            // (each rounded once from its fp64 difference)
                            const float2 ea = sm.E[b & 1][cell], eb = sm.E[2 + (b >> 1)][cell];
                            t[0] = ea.x;
                            t[1] = eb.x;
                            t[2] = ea.y;
                            t[3] = eb.y;
                        } else {
                            const int bn0 = b ^ 2, bn1 = b ^ 1;
                            const int cu = ci + (b >> 1), cv = cj + (b & 1);
                            const int u0 = ci + (bn0 >> 1), v0 = cj + (bn0 & 1);
                            const int u1 = ci + (bn1 >> 1), v1 = cj + (bn1 & 1);
                            t[0] = s0 * (rx[u0][v0] - rx[cu][cv]);
                            t[1] = s1 * (rx[u1][v1] - rx[cu][cv]);
                            t[2] = s0 * (ry[u0][v0] - ry[cu][cv]);
                            t[3] = s1 * (ry[u1][v1] - ry[cu][cv]);
                        }
                        // r = 0 moves both columns of T; r = 1 (2) moves column
                        // 0 (1) only, whose change forms skip the zero entries.
                        float dn, dm, ax, bx, ay, by;
                        if (r == 0) {
                            const float dt[4] = {-s0 * dx, -s1 * dx, -s0 * dy, -s1 * dy};
                            dm = dmu2<float>(KIND, t, dt, float(delta), dn);
                            ax = t[0] + dt[0];
                            bx = t[1] + dt[1];
                            ay = t[2] + dt[2];
                            by = t[3] + dt[3];
                        } else if (r == 1) {
                            const float ex = s0 * dx, ey = s0 * dy;
                            dm = dmu2_col<float, 0>(KIND, t, ex, ey, float(delta), dn);
                            ax = t[0] + ex;
                            bx = t[1];
                            ay = t[2] + ey;
                            by = t[3];
                        } else {
                            const float ex = s1 * dx, ey = s1 * dy;
                            dm = dmu2_col<float, 1>(KIND, t, ex, ey, float(delta), dn);
                            ax = t[0];
                            bx = t[1] + ex;
                            ay = t[2];
                            by = t[3] + ey;
                        }
                        if (dn * dn < float(kGuard * kGuard) * (ax * ax + ay * ay) * (bx * bx + by * by)) {
                            guard |= 1u << (ci * 6 + cj * 3 + r);  // redone in fp64 below
                        } else {
                            dsum += dm;
                            md = fminf(md, dn);
                        }
                    }
                }
            }
#pragma unroll 1
            for (int k = 0; guard && k < 12; ++k) {
                if (!((guard >> k) & 1u)) { continue; }
                const int ci = k / 6, cj = (k / 3) % 2, r = k % 3;
                const int a = (1 - ci) * 2 + (1 - cj);
                const int b = (r == 0) ? a : ((r == 1) ? (a ^ 2) : (a ^ 1));
                const int bn0 = b ^ 2, bn1 = b ^ 1;
                float dn;
                dsum += dmu2_guard64<KIND>(sm.P[(ti + ci + (b >> 1)) * PW + (tj + cj + (b & 1))],
                                           sm.P[(ti + ci + (bn0 >> 1)) * PW + (tj + cj + (bn0 & 1))],
                                           sm.P[(ti + ci + (bn1 >> 1)) * PW + (tj + cj + (bn1 & 1))], r, double(dx),
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
    } else {
    for (int it = 0; it < 10 && !accepted; ++it) {
        const C dx = alpha * dlt[0], dy = alpha * dlt[1];
        C e = econst;
        C md = mdconst;
#pragma unroll
        for (int ci = 0; ci < 2; ++ci) {
#pragma unroll
            for (int cj = 0; cj < 2; ++cj) {
                const int a = (1 - ci) * 2 + (1 - cj);
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const int b = (r == 0) ? a : ((r == 1) ? (a ^ 2) : (a ^ 1));
                    const int bn0 = b ^ 2, bn1 = b ^ 1;
                    // node window coords of corner / neighbours (cell base (ci, cj))
                    const int cu = ci + (b >> 1), cv = cj + (b & 1);
                    const int u0 = ci + (bn0 >> 1), v0 = cj + (bn0 & 1);
                    const int u1 = ci + (bn1 >> 1), v1 = cj + (bn1 & 1);
                    const C pcx = (b == a) ? dx : rx[cu][cv];
                    const C pcy = (b == a) ? dy : ry[cu][cv];
                    const C p0x = (bn0 == a) ? dx : rx[u0][v0];
                    const C p0y = (bn0 == a) ? dy : ry[u0][v0];
                    const C p1x = (bn1 == a) ? dx : rx[u1][v1];
                    const C p1y = (bn1 == a) ? dy : ry[u1][v1];
                    const C s0 = (b & 2) ? C(-1) : C(1);
                    const C s1 = (b & 1) ? C(-1) : C(1);
                    C ax = s0 * (p0x - pcx), bx = s1 * (p1x - pcx);
                    C ay = s0 * (p0y - pcy), by = s1 * (p1y - pcy);
                    C d;
                    C m;
                    if constexpr (std::is_same_v<C, float>) {
                        const float dd = ax * by - bx * ay;
                        const float nn0 = ax * ax + ay * ay, nn1 = bx * bx + by * by;
                        if (dd * dd < float(kGuard * kGuard) * nn0 * nn1) {
                            // fp64 re-evaluation from the staged fp64 positions
                            const double2 qc = sm.P[(ti + cu) * PW + (tj + cv)];
                            const double2 q0 = sm.P[(ti + u0) * PW + (tj + v0)];
                            const double2 q1 = sm.P[(ti + u1) * PW + (tj + v1)];
                            const double tX = pos.x + double(dx), tY = pos.y + double(dy);
                            const double cX = (b == a) ? tX : qc.x, cY = (b == a) ? tY : qc.y;
                            const double X0 = (bn0 == a) ? tX : q0.x, Y0 = (bn0 == a) ? tY : q0.y;
                            const double X1 = (bn1 == a) ? tX : q1.x, Y1 = (bn1 == a) ? tY : q1.y;
                            double dd64;
                            const double m64 = sample_mu_c<KIND, double>(
                              double(s0) * (X0 - cX), double(s1) * (X1 - cX), double(s0) * (Y0 - cY),
                              double(s1) * (Y1 - cY), delta, dd64);
                            m = float(m64);
                            d = float(dd64);
                        } else {
                            m = sample_mu_c<KIND, float>(ax, bx, ay, by, float(delta), d);
                        }
                    } else {
                        m = sample_mu_c<KIND, double>(ax, bx, ay, by, delta, d);
                    }
                    e += m;
                    md = fmin(md, d);
                }
            }
        }
        e -= tx * dx + ty * dy;
        const bool ok = isfinite(e) && (e <= e0 + Tol<C>::energy) &&
                        (KIND == kUntangle || md > C(0));
        if (ok) {
            ax_acc = dx;
            ay_acc = dy;
            accepted = true;
        } else {
            alpha *= C(0.5);
        }
    }
    }
    double2 out = pos;
    if (accepted) {
        out.x = pos.x + omega * double(ax_acc);
        out.y = pos.y + omega * double(ay_acc);
    }
    Xout[slot] = out;
}

// ---------------------------------------------------------------------------
// Stored-patch sweep (fp64): one thread per DOF over its ragged occurrence
// slice; general W_inv, per-sample weights and the FAS tau shift.  Mirrors
// src/patch.hpp:325 patch_eval + src/sweep.hpp:1534 interior_update_kernel.
// ---------------------------------------------------------------------------
struct StoredPatch2 {
    int64_t n;              // DOFs
    const int32_t* slot;    // [n] owner slot of each DOF
    const int64_t* off;     // [n+1] occurrence ranges
    const int32_t* gc;      // [occ] owner slots
    const int32_t* gn0;
    const int32_t* gn1;
    const int8_t* s0;       // [occ] +-1
    const int8_t* s1;
    const int32_t* role;    // [occ]
    const double* W;        // [occ*4] or [4]
    int32_t w_stride;       // 4 or 0
    const double* wt;       // [occ] or [1]
    int32_t wt_stride;      // 1 or 0
    const int8_t* etag;     // [n] entity tag of each DOF, or NULL (all Free)
    const double* epar;     // [n * EGG_B200_ENTITY_FIELDS] entity records (constrained DOFs)
    int cold;               // first sweep of a run call: trimmed arcs project in world space
    const double* arena;    // entity arena (B-spline knots, control points, weights)
    double* seeds;          // [n] last foot parameter of each B-spline DOF (NaN: none)
    SoftTable soft;         // directional / curvature terms per DOF (off == NULL: none)
};

__device__ __forceinline__ void assemble_T(const double2 c, const double2 n0, const double2 n1,
                                           double s0, double s1, const double* w, double t[4],
                                           double& detA)
{
    const double A00 = s0 * (n0.x - c.x), A01 = s1 * (n1.x - c.x);
    const double A10 = s0 * (n0.y - c.y), A11 = s1 * (n1.y - c.y);
    detA = A00 * A11 - A01 * A10;
    t[0] = A00 * w[0] + A01 * w[2];
    t[1] = A00 * w[1] + A01 * w[3];
    t[2] = A10 * w[0] + A11 * w[2];
    t[3] = A10 * w[1] + A11 * w[3];
}

template <int KIND>
__device__ void stored_patch_eval(const StoredPatch2& sp, const double2* X, int64_t d, double delta,
                                  double g[2], double h[4], double& e0, double& mdet)
{
    g[0] = g[1] = 0.0;
    h[0] = h[1] = h[2] = h[3] = 0.0;
    e0 = 0.0;
    mdet = INFINITY;
    for (int64_t p = sp.off[d]; p < sp.off[d + 1]; ++p) {
        const double* w = sp.W + p * sp.w_stride;
        const double s0 = sp.s0[p], s1 = sp.s1[p];
        double t[4], detA;
        assemble_T(X[sp.gc[p]], X[sp.gn0[p]], X[sp.gn1[p]], s0, s1, w, t, detA);
        mdet = fmin(mdet, detA);
        const double wt = sp.wt[p * sp.wt_stride];
        const int role = sp.role[p];
        double mu, gg[4], H[16];
        mu_eval<double>(KIND, t, delta, mu, gg, H);
        e0 += wt * mu;
        if (role < 0) { continue; }
        // Jb (4x2): row a = (i, c): column i holds v_c, v = -(s0 w[0,c] + s1 w[1,c])
        // for the corner, s_ax w[ax, c] for an axis-ax neighbour.
        double v[2];
        for (int c = 0; c < 2; ++c) {
            v[c] = (role == 0) ? -(s0 * w[0 * 2 + c] + s1 * w[1 * 2 + c])
                               : ((role == 1) ? s0 * w[0 * 2 + c] : s1 * w[1 * 2 + c]);
        }
        for (int i = 0; i < 2; ++i) {
            g[i] += wt * (gg[i * 2 + 0] * v[0] + gg[i * 2 + 1] * v[1]);
            for (int j = 0; j < 2; ++j) {
                double acc = 0.0;
                for (int c = 0; c < 2; ++c) {
                    for (int c2 = 0; c2 < 2; ++c2) { acc += v[c] * H[(i * 2 + c) * 4 + (j * 2 + c2)] * v[c2]; }
                }
                h[i * 2 + j] += wt * acc;
            }
        }
    }
}

template <int KIND>
__device__ void stored_trial(const StoredPatch2& sp, const double2* X, int64_t d, int32_t dslot,
                             double2 trial, double delta, double& e, double& md)
{
    e = 0.0;
    md = INFINITY;
    for (int64_t p = sp.off[d]; p < sp.off[d + 1]; ++p) {
        const double* w = sp.W + p * sp.w_stride;
        const int32_t ic = sp.gc[p], i0 = sp.gn0[p], i1 = sp.gn1[p];
        const double2 c = (ic == dslot) ? trial : X[ic];
        const double2 n0 = (i0 == dslot) ? trial : X[i0];
        const double2 n1 = (i1 == dslot) ? trial : X[i1];
        double t[4], detA;
        assemble_T(c, n0, n1, double(sp.s0[p]), double(sp.s1[p]), w, t, detA);
        e += sp.wt[p * sp.wt_stride] * mu_value<double>(KIND, t, delta);
        md = fmin(md, detA);
    }
}

// Reductions over an aligned group of G lanes (G a power of two <= 32) by
// xor butterfly: every lane of the group ends with the same value (each step
// adds a pair in both orders, and fp addition commutes), so the lanes of a
// group take identical Newton steps and accept decisions.
template <int G> __device__ __forceinline__ unsigned group_mask()
{
    if constexpr (G == 32) {
        return 0xffffffffu;
    } else {
        return ((1u << G) - 1u) << ((threadIdx.x & 31u) & ~unsigned(G - 1));
    }
}

template <int G> __device__ __forceinline__ double group_sum(double v)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) { v += __shfl_xor_sync(group_mask<G>(), v, o, G); }
    return v;
}

template <int G> __device__ __forceinline__ double group_min(double v)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) { v = fmin(v, __shfl_xor_sync(group_mask<G>(), v, o, G)); }
    return v;
}

// Lanes per DOF of the stored-patch sweeps: the widest group (32, 8, 2 or 1)
// whose threads over all stored DOFs stay within a budget.  Few stored DOFs
// (a small multi-block mesh) get a warp each, so the patch is a few rounds of
// parallel work; many (a batch of meshes) get narrow groups, which spend
// fewer issue slots on per-lane redundancy (the solve, the reductions) while
// the interior tiles run beside them.  A 3D patch has 64 samples to split,
// so its budget is larger.  Measured on B200: 256 meshes with 139 k stored
// DOFs run best at 2 lanes (a warp each: -15%); the 7-block 129^3 sphere's
// FAS levels best at 8 lanes on the fine level.
constexpr int64_t kStoredFillThreads2 = 148 * 4096;
constexpr int64_t kStoredFillThreads3 = 148 * 16384;

// Stored-patch sweep, G lanes per DOF: the lanes split the DOF's samples
// (gradient, contracted Hessian, energy; then each line-search trial) and
// reduce across the group, so a ragged patch of 16-64 gathered samples can be
// a few rounds of parallel work instead of one thread's serial loop.
template <int KIND, int G, bool CON>
__global__ void stored_patch_kernel(StoredPatch2 sp, const double2* __restrict__ Xin,
                                    double2* __restrict__ Xout, const double2* __restrict__ tau,
                                    double delta, double omega, double2* __restrict__ grad_out)
{
    const int lane = threadIdx.x & (G - 1);
    const int64_t ngroups = (int64_t(gridDim.x) * blockDim.x) / G;
    for (int64_t d = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) / G; d < sp.n; d += ngroups) {
        const int32_t slot = sp.slot[d];
        const double2 pos = Xin[slot];
        const int64_t p0 = sp.off[d], p1 = sp.off[d + 1];
        double g0 = 0.0, g1 = 0.0, h00 = 0.0, h01 = 0.0, h10 = 0.0, h11 = 0.0, e0 = 0.0;
        for (int64_t p = p0 + lane; p < p1; p += G) {
            const double* w = sp.W + p * sp.w_stride;
            const double s0 = sp.s0[p], s1 = sp.s1[p];
            double t[4], detA;
            assemble_T(Xin[sp.gc[p]], Xin[sp.gn0[p]], Xin[sp.gn1[p]], s0, s1, w, t, detA);
            const double wt = sp.wt[p * sp.wt_stride];
            const int role = sp.role[p];
            double mu, gg[4], H[16];
            mu_eval<double>(KIND, t, delta, mu, gg, H);
            e0 += wt * mu;
            if (role < 0) { continue; }
            double v[2];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                v[c] = (role == 0) ? -(s0 * w[c] + s1 * w[2 + c]) : ((role == 1) ? s0 * w[c] : s1 * w[2 + c]);
            }
            double gl[2], hl[4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                gl[i] = gg[i * 2] * v[0] + gg[i * 2 + 1] * v[1];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    double acc = 0.0;
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
#pragma unroll
                        for (int c2 = 0; c2 < 2; ++c2) { acc += v[c] * H[(i * 2 + c) * 4 + (j * 2 + c2)] * v[c2]; }
                    }
                    hl[i * 2 + j] = acc;
                }
            }
            g0 += wt * gl[0];
            g1 += wt * gl[1];
            h00 += wt * hl[0];
            h01 += wt * hl[1];
            h10 += wt * hl[2];
            h11 += wt * hl[3];
        }
        double g[2] = {group_sum<G>(g0), group_sum<G>(g1)};
        double h[4] = {group_sum<G>(h00), group_sum<G>(h01), group_sum<G>(h10), group_sum<G>(h11)};
        e0 = group_sum<G>(e0);
        // Soft terms fold into the Newton system and the baseline energy
        // (src/sweep.hpp:1461-1512; constrained DOFs take the directional
        // samples only, src/sweep.hpp:1307-1327).  Every lane of the group
        // adds them alike.
        const int etag = (CON && sp.etag != nullptr) ? int(sp.etag[d]) : 0;
        soft_dof_accumulate<2>(sp.soft, d, etag == 0, reinterpret_cast<const double*>(Xin), g, h, e0);
        double tx = 0.0, ty = 0.0;
        if (tau != nullptr) {
            tx = tau[slot].x;
            ty = tau[slot].y;
            g[0] -= tx;
            g[1] -= ty;
            e0 -= tx * pos.x + ty * pos.y;
        }
        if (grad_out != nullptr) {
            if (lane == 0) { grad_out[slot] = make_double2(g[0], g[1]); }
            continue;
        }
        // A constrained DOF (src/sweep.hpp:1286-1403): the Newton step reduced
        // onto its entity's tangent, damped by omega before the line search,
        // and every trial projected onto the entity, so the accepted point
        // stays on the geometry.  A Free DOF: the full step, omega blend after.
        // A trimmed curve after the first sweep of a run call searches in its
        // parameter instead (src/sweep.hpp:1718-1876): trials q* + alpha dq,
        // clamped onto the trim and evaluated on the curve.
        // CON = false (a level without constrained DOFs) compiles none of it.
        const double* er = sp.epar + (etag != 0 ? d * EGG_B200_ENTITY_FIELDS : 0);
        const bool warm_arc = is_tcurve(etag) && !sp.cold;
        // B-spline DOFs carry a seed (their last foot parameter): every seeded
        // projection starts its Newton solve there and stores its result
        // (src/sweep.hpp:1219-1265).
        const bool bsp = etag == EGG_B200_TAG_BSPLINE;
        const bool comp = etag == EGG_B200_TAG_COMPOSITE;
        const double* cslice = comp ? sp.arena + int64_t(er[6]) : nullptr;  // the path's arena slice
        const double* crec = comp ? cslice + int64_t(er[1]) : nullptr;
        const int cseg = comp ? int(er[0]) : 0;
        double seed = bsp ? sp.seeds[d] : 0.0;
        BSplineCurve bc {};
        if (bsp) { bc = bspline_view(er, sp.arena); }
        double dl[2] = {0.0, 0.0};
        double qstar = 0.0, dq = 0.0;
        if (etag == 0) {
            solve2<double>(h, g, dl);
        } else if (comp) {  // one path for every sweep: step on the nearest segment's tangent
            composite_newton_step(cslice, crec, cseg, h, g, pos.x, pos.y, dl);
            dl[0] *= omega;
            dl[1] *= omega;
        } else if (bsp) {
            if (sp.cold) {
                bspline_cold_step(bc, h, g, pos.x, pos.y, seed, dl);
                dl[0] *= omega;
                dl[1] *= omega;
            } else {
                bspline_warm_step(bc, h, g, pos.x, pos.y, omega, seed, qstar, dq);
            }
        } else if (warm_arc) {
            tc_warm_step(etag, er, h, g, pos.x, pos.y, omega, qstar, dq);
        } else {
            entity_newton_step(etag, er, h, g, pos.x, pos.y, dl);
            dl[0] *= omega;
            dl[1] *= omega;
        }
        double alpha = 1.0;
        double2 cur = pos;
        for (int it = 0; it < 10; ++it) {
            double2 trial = make_double2(pos.x + alpha * dl[0], pos.y + alpha * dl[1]);
            if (comp) {
                double tx, ty;
                composite_frame(cslice, crec, cseg, trial.x, trial.y, trial.x, trial.y, tx, ty);
            } else if (bsp) {
                if (sp.cold) {
                    bspline_project_seeded(bc, trial.x, trial.y, seed, trial.x, trial.y);
                } else {
                    bspline_point(bc, bspline_clamp(bc, qstar + alpha * dq), 0, trial.x, trial.y);
                }
            } else if (warm_arc) {
                tc_eval(etag, er, tc_clamp(etag, er, qstar + alpha * dq), 0, trial.x, trial.y);
            } else if (etag != 0) {
                entity_project(etag, er, trial.x, trial.y, trial.x, trial.y);
            }
            double e = 0.0, md = INFINITY;
            for (int64_t p = p0 + lane; p < p1; p += G) {
                const double* w = sp.W + p * sp.w_stride;
                const int32_t ic = sp.gc[p], i0 = sp.gn0[p], i1 = sp.gn1[p];
                const double2 c = (ic == slot) ? trial : Xin[ic];
                const double2 n0 = (i0 == slot) ? trial : Xin[i0];
                const double2 n1 = (i1 == slot) ? trial : Xin[i1];
                double t[4], detA;
                assemble_T(c, n0, n1, double(sp.s0[p]), double(sp.s1[p]), w, t, detA);
                e += sp.wt[p * sp.wt_stride] * mu_value<double>(KIND, t, delta);
                md = fmin(md, detA);
            }
            e = group_sum<G>(e);
            if (sp.soft.off != nullptr) {
                const double tr[2] = {trial.x, trial.y};
                e += soft_dof_trial<2>(sp.soft, d, etag == 0, reinterpret_cast<const double*>(Xin), tr);
            }
            e -= tx * trial.x + ty * trial.y;
            md = group_min<G>(md);
            if (isfinite(e) && e <= e0 + Tol<double>::energy && (KIND == kUntangle || md > 0.0)) {
                cur = trial;
                break;
            }
            alpha *= 0.5;
        }
        if (etag == 0 && omega != 1.0) {
            cur.x = pos.x + omega * (cur.x - pos.x);
            cur.y = pos.y + omega * (cur.y - pos.y);
        }
        if (bsp && lane == 0) { sp.seeds[d] = seed; }
        if (lane == 0) { Xout[slot] = cur; }
    }
}

// ---------------------------------------------------------------------------
// Energy / min-det reductions (fp64, compensated, deterministic two-pass).
// ---------------------------------------------------------------------------
struct Comp {
    double s, c;
};

__device__ __forceinline__ void comp_add(Comp& a, double x)
{
    const double t = a.s + x;
    if (fabs(a.s) >= fabs(x)) {
        a.c += (a.s - t) + x;
    } else {
        a.c += (x - t) + a.s;
    }
    a.s = t;
}

__device__ __forceinline__ Comp comp_merge(Comp a, Comp b)
{
    Comp r = a;
    comp_add(r, b.s);
    r.c += b.c;
    return r;
}

// Block-level reduction of (compensated sum, min); thread 0 returns true and
// holds the block's result in acc / mn.
__device__ __forceinline__ bool block_reduce(Comp& acc, double& mn)
{
    __shared__ double ss[32], sc[32], sm[32];
    for (int o = 16; o > 0; o >>= 1) {
        Comp other;
        other.s = __shfl_down_sync(0xffffffffu, acc.s, o);
        other.c = __shfl_down_sync(0xffffffffu, acc.c, o);
        const double om = __shfl_down_sync(0xffffffffu, mn, o);
        acc = comp_merge(acc, other);
        mn = fmin(mn, om);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        ss[wid] = acc.s;
        sc[wid] = acc.c;
        sm[wid] = mn;
    }
    __syncthreads();
    if (wid != 0) { return false; }
    const int nw = (blockDim.x + 31) >> 5;
    Comp a {0.0, 0.0};
    double m = INFINITY;
    if (lane < nw) {
        a.s = ss[lane];
        a.c = sc[lane];
        m = sm[lane];
    }
    for (int o = 16; o > 0; o >>= 1) {
        Comp other;
        other.s = __shfl_down_sync(0xffffffffu, a.s, o);
        other.c = __shfl_down_sync(0xffffffffu, a.c, o);
        const double om = __shfl_down_sync(0xffffffffu, m, o);
        a = comp_merge(a, other);
        m = fmin(m, om);
    }
    acc = a;
    mn = m;
    return lane == 0;
}

// Block reduction into partial slot blockIdx.y * gridDim.x + blockIdx.x
// (blockIdx.y = segment of a segmented reduction, 0 otherwise).
__device__ __forceinline__ void block_reduce_store(Comp acc, double mn, double* part_s,
                                                   double* part_c, double* part_m)
{
    if (block_reduce(acc, mn)) {
        const int64_t slot = int64_t(blockIdx.y) * gridDim.x + blockIdx.x;
        part_s[slot] = acc.s;
        part_c[slot] = acc.c;
        part_m[slot] = mn;
    }
}

// Item range of this CTA row: segment blockIdx.y of `seg` (prefix offsets),
// or [0, n) without segments.
__device__ __forceinline__ void segment_range(const int64_t* seg, int64_t n, int64_t& lo, int64_t& hi)
{
    lo = seg ? seg[blockIdx.y] : 0;
    hi = seg ? seg[blockIdx.y + 1] : n;
}

struct EnergyStructured2 {
    int32_t nblocks;
    const BlockInfo* blocks;
    const int64_t* cell_off;  // [nblocks+1] prefix of (n0-1)(n1-1)
    int64_t ncell;
    const double* W;          // [4] or [ncell*4*4]
    int32_t w_stride;         // 0 or 4 (per sample)
    const double* wt;         // [1] or [ncell*4]
    int32_t wt_stride;
    const int64_t* seg = nullptr;  // per-mesh cell prefix offsets (segmented reduction) or null
};

template <int KIND>
__global__ void energy_structured2_kernel(EnergyStructured2 es, const double2* __restrict__ X,
                                          double delta, double* part_s, double* part_c,
                                          double* part_m)
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
        const int cw = bi.n[1] - 1;
        const int i = int(lc / cw), j = int(lc % cw);
        const int64_t base = bi.off + int64_t(i) * bi.n[1] + j;
        const double2 p[4] = {X[base], X[base + 1], X[base + bi.n[1]], X[base + bi.n[1] + 1]};
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int64_t sid = c * 4 + b;
            const double* w = es.W + sid * es.w_stride;
            double t[4], detA;
            assemble_T(p[b], p[b ^ 2], p[b ^ 1], (b & 2) ? -1.0 : 1.0, (b & 1) ? -1.0 : 1.0, w, t,
                       detA);
            comp_add(acc, es.wt[sid * es.wt_stride] * mu_value<double>(KIND, t, delta));
            mn = fmin(mn, detA);
        }
    }
    block_reduce_store(acc, mn, part_s, part_c, part_m);
}

struct EnergyStored2 {
    int64_t n;
    const int32_t* gc;
    const int32_t* gn0;
    const int32_t* gn1;
    const int8_t* s0;
    const int8_t* s1;
    const double* W;
    int32_t w_stride;
    const double* wt;
    int32_t wt_stride;
    const int64_t* seg = nullptr;  // per-mesh sample prefix offsets or null
};

template <int KIND>
__global__ void energy_stored2_kernel(EnergyStored2 es, const double2* __restrict__ X, double delta,
                                      double* part_s, double* part_c, double* part_m)
{
    Comp acc {0.0, 0.0};
    double mn = INFINITY;
    int64_t i_lo, i_hi;
    segment_range(es.seg, es.n, i_lo, i_hi);
    for (int64_t i = i_lo + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < i_hi;
         i += int64_t(gridDim.x) * blockDim.x) {
        double t[4], detA;
        assemble_T(X[es.gc[i]], X[es.gn0[i]], X[es.gn1[i]], double(es.s0[i]), double(es.s1[i]),
                   es.W + i * es.w_stride, t, detA);
        comp_add(acc, es.wt[i * es.wt_stride] * mu_value<double>(KIND, t, delta));
        mn = fmin(mn, detA);
    }
    block_reduce_store(acc, mn, part_s, part_c, part_m);
}

// Single-CTA final pass over the partials, fixed order: out[0] = energy, out[1] = min det.
__global__ void reduce_finalize_kernel(const double* part_s, const double* part_c,
                                       const double* part_m, int n, double* out_e, double* out_m)
{
    Comp acc {0.0, 0.0};
    double mn = INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        acc = comp_merge(acc, Comp {part_s[i], part_c[i]});
        mn = fmin(mn, part_m[i]);
    }
    if (block_reduce(acc, mn)) {
        *out_e = acc.s + acc.c;
        *out_m = mn;
    }
}

// Adds the whole-sample directional total to a finished energy report
// (src/directional.hpp:281-299, src/sweep.hpp:1921): one CTA, compensated,
// fixed order, so the reported energy is the composed objective.
template <int D>
__global__ void soft_energy_add_kernel(const SoftTerm* __restrict__ terms, int64_t n, double eps,
                                       const double* __restrict__ X, double* out_e)
{
    Comp acc {0.0, 0.0};
    double mn = INFINITY;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const SoftTerm t = terms[i];
        double p[4][3];
        soft_load<D>(t, X, p);
        comp_add(acc, soft_energy<D>(t, p, eps));
    }
    if (block_reduce(acc, mn)) { *out_e += acc.s + acc.c; }
}

// Per-mesh directional totals of a batch: CTA m adds the sum over terms
// [seg[m], seg[m+1]) to out[2m], the mesh's reported energy.
template <int D>
__global__ void soft_energy_add_seg_kernel(const SoftTerm* __restrict__ terms, const int64_t* __restrict__ seg,
                                           double eps, const double* __restrict__ X, double* out)
{
    Comp acc {0.0, 0.0};
    double mn = INFINITY;
    for (int64_t i = seg[blockIdx.x] + threadIdx.x; i < seg[blockIdx.x + 1]; i += blockDim.x) {
        const SoftTerm t = terms[i];
        double p[4][3];
        soft_load<D>(t, X, p);
        comp_add(acc, soft_energy<D>(t, p, eps));
    }
    if (block_reduce(acc, mn)) { out[2 * int64_t(blockIdx.x)] += acc.s + acc.c; }
}

// Segmented final pass: CTA m folds partials [m n, (m+1) n) into
// out[2m] = energy and out[2m+1] = min det of segment m.
__global__ void reduce_finalize_seg_kernel(const double* part_s, const double* part_c,
                                           const double* part_m, int n, double* out)
{
    const int64_t base = int64_t(blockIdx.x) * n;
    Comp acc {0.0, 0.0};
    double mn = INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        acc = comp_merge(acc, Comp {part_s[base + i], part_c[base + i]});
        mn = fmin(mn, part_m[base + i]);
    }
    if (block_reduce(acc, mn)) {
        out[2 * int64_t(blockIdx.x)] = acc.s + acc.c;
        out[2 * int64_t(blockIdx.x) + 1] = mn;
    }
}

}  // namespace egg_b200
