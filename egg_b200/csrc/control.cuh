// Control-net reduced Gauss-Newton kernels (src/control_net.hpp:486-1106,
// src/control_solve.hpp:533-820).
//
// A net drives one block of the store: X = M C + b with M the tensor product
// of per-axis clamped B-spline bases (banded: node i of axis k reads controls
// off_k[i] .. off_k[i] + k_supp - 1 with weights wt_k[i, :]).  Several nets
// (one per mesh of a batch) are stacked: net-node, lattice and free-control
// spaces are concatenations indexed through per-net offsets.
//
// Per-node work runs over a net's block nodes and reads the block's canonical
// cell stencil directly (cells of the block around the node, 2^D corner
// samples each, the node's role in each), so no membership tables are stored
// and each sample's metric work is fused with the node gather:
//   grad  y_n = sum_p wt_p J_b(n,p)^T dmu/dT(T_p)
//   hvp   y_n = sum_p wt_p J_b(n,p)^T H(T_p) dT_p,  dT_p assembled from corr
//   hess  h_n = sum_p wt_p J_b^T H(T_p) J_b          (Jacobi preconditioner)
// J_b(n,p) is rank one, e_i v^T: v = -W^T s for the corner, s_k W[k,:] for
// the axis-k neighbour.
#pragma once

#include "kernels3d.cuh"

namespace egg_b200
{

struct CtlNet {
    int32_t block;
    int32_t k_supp;
    int32_t node_shape[3];
    int32_t ctrl_shape[3];
    int32_t ctrl_stride[3];
    int32_t pad;
    int64_t node_off;  // store slot of the block's first node
    int64_t cell_off;  // first canonical energy-stencil cell of the block
    int64_t n_off;     // first net node (b and node-space buffers)
    int64_t c_off;     // first lattice control
    int64_t f_off;     // first free control
    int64_t n_nodes, n_ctrl, n_free;
    int64_t ax_off[3];   // into the concatenated per-axis off / wt tables (nodes)
    int64_t sup_base[3]; // into the concatenated support CSR offsets (controls + 1)
};

struct CtlTables {
    int32_t n_nets;
    const CtlNet* nets;
    const int64_t* node_pfx;  // [n_nets + 1] net-node prefix
    const int64_t* ctrl_pfx;  // [n_nets + 1] lattice prefix
    const int64_t* free_pfx;  // [n_nets + 1] free-control prefix
    const int32_t* off;       // per-axis first support control per node
    const double* wt;         // per-axis basis weights [node * k_supp]
    const int32_t* sup_off;   // per-axis support CSR offsets (relative to sup entries of the net axis)
    const int32_t* sup_node;  // support nodes
    const double* sup_w;      // support weights
    const int32_t* free_idx;  // [free] lattice index within the net
    const int32_t* free_midx; // [free * D] multi-index
    const int32_t* free_of;   // [lattice] stacked free index or -1
};

// Per-net PCG state (device resident; thread 0 of the per-net reduction CTA
// updates it, kernels skip nets whose `done` is set).
struct PcgState {
    double b_norm2, stop2, r_norm2, rz, alpha, beta, lam, pad;
    int32_t it, its, done, max_iter, active, pad2;
};

__device__ __forceinline__ int net_of(const int64_t* pfx, int n, int64_t i)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pfx[mid] <= i) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

template <int D> __device__ __forceinline__ void unravel_node(const CtlNet& n, int64_t f, int L[3])
{
    L[2] = 0;
    if (D == 3) {
        L[2] = int(f % n.node_shape[2]);
        f /= n.node_shape[2];
    }
    L[1] = int(f % n.node_shape[1]);
    L[0] = int(f / n.node_shape[1]);
}

// X (store) = M C + b, or a net-node field out = M C (b == null, node_space).
template <int D>
__global__ void ctl_eval_kernel(CtlTables T, int64_t total_nodes, const double* __restrict__ C,
                                const double* __restrict__ b, double* __restrict__ out, bool node_space,
                                const PcgState* __restrict__ st)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_nodes;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.node_pfx, T.n_nets, g);
        if (st && st[ni].done) { continue; }
        const CtlNet n = T.nets[ni];
        const int64_t f = g - n.n_off;
        int L[3];
        unravel_node<D>(n, f, L);
        const int ks = n.k_supp;
        double acc[D];
#pragma unroll
        for (int c = 0; c < D; ++c) { acc[c] = 0.0; }
        const int32_t* off0 = T.off + n.ax_off[0];
        const int32_t* off1 = T.off + n.ax_off[1];
        const double* wt0 = T.wt + n.ax_off[0] * ks;
        const double* wt1 = T.wt + n.ax_off[1] * ks;
        const double* Cn = C + n.c_off * D;
        if (D == 2) {
            for (int t0 = 0; t0 < ks; ++t0) {
                const double w0 = wt0[L[0] * ks + t0];
                const int64_t r0 = int64_t(off0[L[0]] + t0) * n.ctrl_stride[0];
                for (int t1 = 0; t1 < ks; ++t1) {
                    const double w = 1.0 * w0 * wt1[L[1] * ks + t1];
                    const int64_t ci = r0 + int64_t(off1[L[1]] + t1) * n.ctrl_stride[1];
#pragma unroll
                    for (int c = 0; c < D; ++c) { acc[c] += w * Cn[ci * D + c]; }
                }
            }
        } else {
            const int32_t* off2 = T.off + n.ax_off[2];
            const double* wt2 = T.wt + n.ax_off[2] * ks;
            for (int t0 = 0; t0 < ks; ++t0) {
                const double w0 = wt0[L[0] * ks + t0];
                const int64_t r0 = int64_t(off0[L[0]] + t0) * n.ctrl_stride[0];
                for (int t1 = 0; t1 < ks; ++t1) {
                    const double w01 = 1.0 * w0 * wt1[L[1] * ks + t1];
                    const int64_t r1 = r0 + int64_t(off1[L[1]] + t1) * n.ctrl_stride[1];
                    for (int t2 = 0; t2 < ks; ++t2) {
                        const double w = w01 * wt2[L[2] * ks + t2];
                        const int64_t ci = r1 + int64_t(off2[L[2]] + t2) * n.ctrl_stride[2];
#pragma unroll
                        for (int c = 0; c < D; ++c) { acc[c] += w * Cn[ci * D + c]; }
                    }
                }
            }
        }
        if (node_space) {
#pragma unroll
            for (int c = 0; c < D; ++c) { out[g * D + c] = acc[c]; }
        } else {
            const int64_t slot = n.node_off + f;
#pragma unroll
            for (int c = 0; c < D; ++c) { out[slot * D + c] = acc[c] + (b ? b[g * D + c] : 0.0); }
        }
    }
}

// C_dir[lattice] = v[free] on free controls, 0 elsewhere.
template <int D>
__global__ void ctl_scatter_kernel(CtlTables T, int64_t total_ctrl, const double* __restrict__ v,
                                   double* __restrict__ Cdir, const PcgState* __restrict__ st)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_ctrl;
         g += int64_t(gridDim.x) * blockDim.x) {
        if (st && st[net_of(T.ctrl_pfx, T.n_nets, g)].done) { continue; }
        const int32_t f = T.free_of[g];
#pragma unroll
        for (int c = 0; c < D; ++c) { Cdir[g * D + c] = f >= 0 ? v[int64_t(f) * D + c] : 0.0; }
    }
}

enum { kCtlGrad = 0, kCtlHvp = 1, kCtlHess = 2 };

// Rank-one direction of node role r in a sample (v = -W^T s or s_k W[k,:]).
template <int D> __device__ __forceinline__ void role_dir(int role, const double* w, const double s[3], double v[3])
{
#pragma unroll
    for (int j = 0; j < D; ++j) {
        if (role == 0) {
            double a = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) { a -= s[k] * w[k * D + j]; }
            v[j] = a;
        } else {
            v[j] = s[role - 1] * w[(role - 1) * D + j];
        }
    }
}

// The directional soft terms' nodal gradient added into the net-node
// gradient y (src/directional.hpp:343-379, src/control_solve.hpp:556-559):
// every node of every sample, at its owner slot; a slot inside a net's block
// adds to that net's node.  The control's Newton model and preconditioner
// stay the shape term's, as in the reference.
template <int D>
__global__ void ctl_dir_scatter_kernel(CtlTables T, const SoftTerm* __restrict__ terms, int64_t n, double eps,
                                       const double* __restrict__ X, double* __restrict__ y)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        SoftTerm t = terms[i];
        const int ar = soft_arity(t.kind);
        for (int m = 0; m < ar; ++m) {
            const int64_t slot = t.node[m];
            int ni = -1;
            for (int q = 0; q < T.n_nets && ni < 0; ++q) {
                if (slot >= T.nets[q].node_off && slot < T.nets[q].node_off + T.nets[q].n_nodes) { ni = q; }
            }
            if (ni < 0) { continue; }
            t.slot = m;
            double g[D], H[D * D], e = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) { g[k] = 0.0; }
#pragma unroll
            for (int k = 0; k < D * D; ++k) { H[k] = 0.0; }
            soft_accumulate<D>(t, X, eps, g, H, e);
            const int64_t row = T.nets[ni].n_off + (slot - T.nets[ni].node_off);
#pragma unroll
            for (int k = 0; k < D; ++k) { atomicAdd(&y[row * D + k], g[k]); }
        }
    }
}

// Per-node gradient / Hessian-vector product / contracted Hessian over the
// block's canonical cell stencil (see the file comment).
template <int D, int KIND, int MODE>
__global__ void ctl_node_kernel(CtlTables T, int64_t total_nodes, EnergyStructured2 es, const double* __restrict__ X,
                                const double* __restrict__ corr, double* __restrict__ out,
                                const PcgState* __restrict__ st)
{
    constexpr int NC = 1 << D;  // corners per cell
    constexpr int OUTW = MODE == kCtlHess ? D * D : D;
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_nodes;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.node_pfx, T.n_nets, g);
        if (st && st[ni].done) { continue; }
        const CtlNet n = T.nets[ni];
        const int64_t f = g - n.n_off;
        int L[3];
        unravel_node<D>(n, f, L);
        const int n0 = n.node_shape[0], n1 = n.node_shape[1], n2 = D == 3 ? n.node_shape[2] : 1;
        const int c1 = n1 - 1, c2 = D == 3 ? n2 - 1 : 1;
        double acc[OUTW];
#pragma unroll
        for (int i = 0; i < OUTW; ++i) { acc[i] = 0.0; }
        // cells around the node in ascending cell order
        for (int cc = 0; cc < NC; ++cc) {
            int cl[3] = {L[0] - 1 + ((cc >> (D - 1)) & 1), L[1] - 1 + ((cc >> (D - 2)) & 1),
                         D == 3 ? L[2] - 1 + (cc & 1) : 0};
            if (cl[0] < 0 || cl[0] > n0 - 2 || cl[1] < 0 || cl[1] > n1 - 2) { continue; }
            if (D == 3 && (cl[2] < 0 || cl[2] > n2 - 2)) { continue; }
            // node's corner index inside the cell (axis 0 most significant)
            int q = 0;
#pragma unroll
            for (int k = 0; k < D; ++k) { q = (q << 1) | (L[k] - cl[k]); }
            const int64_t lc = (int64_t(cl[0]) * c1 + cl[1]) * c2 + (D == 3 ? cl[2] : 0);
            const int64_t cell = n.cell_off + lc;
            const int64_t base = n.node_off + (int64_t(cl[0]) * n1 + cl[1]) * n2 + (D == 3 ? cl[2] : 0);
            for (int b = 0; b < NC; ++b) {
                int role = -1;
                if (q == b) {
                    role = 0;
                } else {
#pragma unroll
                    for (int k = 0; k < D; ++k) {
                        if (q == (b ^ (1 << (D - 1 - k)))) { role = k + 1; }
                    }
                }
                if (role < 0) { continue; }
                const int64_t sid = cell * NC + b;
                const double* w = es.W + sid * es.w_stride;
                const double wt = es.wt[sid * es.wt_stride];
                double s[3];
#pragma unroll
                for (int k = 0; k < D; ++k) { s[k] = (b & (1 << (D - 1 - k))) ? -1.0 : 1.0; }
                auto corner_slot = [&](int a) {
                    if (D == 2) { return base + int64_t((a >> 1) & 1) * n1 + (a & 1); }
                    return base + (int64_t((a >> 2) & 1) * n1 + ((a >> 1) & 1)) * n2 + (a & 1);
                };
                double v[3];
                role_dir<D>(role, w, s, v);
                if constexpr (D == 2) {
                    const int64_t sc = corner_slot(b), sa = corner_slot(b ^ 2), sb = corner_slot(b ^ 1);
                    const double2* X2 = reinterpret_cast<const double2*>(X);
                    double t[4], detA;
                    assemble_T(X2[sc], X2[sa], X2[sb], s[0], s[1], w, t, detA);
                    double mu, gT[4], H[16];
                    mu_eval<double>(KIND, t, 0.0, mu, gT, H);
                    if constexpr (MODE == kCtlGrad) {
#pragma unroll
                        for (int i = 0; i < 2; ++i) { acc[i] += wt * (gT[2 * i] * v[0] + gT[2 * i + 1] * v[1]); }
                    } else if constexpr (MODE == kCtlHvp) {
                        // dT from corr at the same corners (net-node indexed)
                        const int64_t gc = n.n_off + (sc - n.node_off), ga = n.n_off + (sa - n.node_off),
                                      gb = n.n_off + (sb - n.node_off);
                        const double2 dc = make_double2(corr[2 * gc], corr[2 * gc + 1]);
                        const double2 da = make_double2(corr[2 * ga], corr[2 * ga + 1]);
                        const double2 db = make_double2(corr[2 * gb], corr[2 * gb + 1]);
                        double dt[4], dd;
                        assemble_T(dc, da, db, s[0], s[1], w, dt, dd);
                        double hv[4];
#pragma unroll
                        for (int a = 0; a < 4; ++a) {
                            hv[a] = H[4 * a] * dt[0] + H[4 * a + 1] * dt[1] + H[4 * a + 2] * dt[2] + H[4 * a + 3] * dt[3];
                        }
#pragma unroll
                        for (int i = 0; i < 2; ++i) { acc[i] += wt * (hv[2 * i] * v[0] + hv[2 * i + 1] * v[1]); }
                    } else {
#pragma unroll
                        for (int i = 0; i < 2; ++i) {
#pragma unroll
                            for (int j = 0; j < 2; ++j) {
                                double h = 0.0;
#pragma unroll
                                for (int a = 0; a < 2; ++a) {
#pragma unroll
                                    for (int c = 0; c < 2; ++c) { h += H[(2 * i + a) * 4 + 2 * j + c] * v[a] * v[c]; }
                                }
                                acc[2 * i + j] += wt * h;
                            }
                        }
                    }
                } else {
                    const int32_t ic = int32_t(corner_slot(b));
                    const int32_t in[3] = {int32_t(corner_slot(b ^ 4)), int32_t(corner_slot(b ^ 2)),
                                           int32_t(corner_slot(b ^ 1))};
                    const double none[3] = {0, 0, 0};
                    double t[9], detA;
                    assemble_T3(X, ic, in, s, w, -1, none, t, detA);
                    Shared3<double> S3;
                    shared3<double>(KIND, t, 0.0, S3);
                    if constexpr (MODE == kCtlGrad) {
                        double gT[9];
                        mu3_grad<double>(KIND, S3, gT);
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            acc[i] += wt * (gT[3 * i] * v[0] + gT[3 * i + 1] * v[1] + gT[3 * i + 2] * v[2]);
                        }
                    } else if constexpr (MODE == kCtlHvp) {
                        // corr is net-node indexed: shift store slots into the net-node space
                        const int64_t sh = n.n_off - n.node_off;
                        const int32_t icn = int32_t(ic + sh);
                        const int32_t inn[3] = {int32_t(in[0] + sh), int32_t(in[1] + sh), int32_t(in[2] + sh)};
                        double dt[9], dd;
                        assemble_T3(corr, icn, inn, s, w, -1, none, dt, dd);
                        double hv[9];
                        mu3_hvp<double>(KIND, S3, dt, hv);
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            acc[i] += wt * (hv[3 * i] * v[0] + hv[3 * i + 1] * v[1] + hv[3 * i + 2] * v[2]);
                        }
                    } else {
                        double gg[3], h6[6];
                        role3<double>(KIND, S3, v, gg, h6);
                        const double hm[9] = {h6[0], h6[1], h6[2], h6[1], h6[3], h6[4], h6[2], h6[4], h6[5]};
#pragma unroll
                        for (int i = 0; i < 9; ++i) { acc[i] += wt * hm[i]; }
                    }
                }
            }
        }
#pragma unroll
        for (int i = 0; i < OUTW; ++i) { out[g * OUTW + i] = acc[i]; }
    }
}

// Tensor support of one control: per axis the CSR list of (node, weight).
template <int D> struct Support {
    const int32_t* node[3];
    const double* w[3];
    int len[3];
};

template <int D>
__device__ __forceinline__ Support<D> support_of(const CtlTables& T, const CtlNet& n, const int a[3])
{
    Support<D> sp;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int32_t* so = T.sup_off + n.sup_base[k];
        const int32_t b0 = so[a[k]], b1 = so[a[k] + 1];
        sp.node[k] = T.sup_node + b0;
        sp.w[k] = T.sup_w + b0;
        sp.len[k] = b1 - b0;
    }
    return sp;
}

// Free-control pullback out_f = sum_{n in supp(f)} w_n y_n (+ lam v_f), or the
// Jacobi block P_f = sum w_n^2 h_n (PRECOND).
template <int D, bool PRECOND>
__global__ void ctl_pullback_kernel(CtlTables T, int64_t total_free, const double* __restrict__ y,
                                    double* __restrict__ out, const double* __restrict__ v,
                                    const PcgState* __restrict__ st)
{
    constexpr int W = PRECOND ? D * D : D;
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_free;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.free_pfx, T.n_nets, g);
        if (st && !PRECOND && st[ni].done) { continue; }
        const CtlNet n = T.nets[ni];
        int a[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < D; ++k) { a[k] = T.free_midx[g * D + k]; }
        const Support<D> sp = support_of<D>(T, n, a);
        double acc[W];
#pragma unroll
        for (int i = 0; i < W; ++i) { acc[i] = 0.0; }
        const int l2 = D == 3 ? sp.len[2] : 1;
        for (int t0 = 0; t0 < sp.len[0]; ++t0) {
            for (int t1 = 0; t1 < sp.len[1]; ++t1) {
                for (int t2 = 0; t2 < l2; ++t2) {
                    double w = 1.0 * sp.w[0][t0] * sp.w[1][t1];
                    int64_t nd = int64_t(sp.node[0][t0]) * n.node_shape[1] + sp.node[1][t1];
                    if (D == 3) {
                        w *= sp.w[2][t2];
                        nd = nd * n.node_shape[2] + sp.node[2][t2];
                    }
                    const int64_t gn = n.n_off + nd;
                    if (PRECOND) {
                        const double w2 = w * w;
#pragma unroll
                        for (int i = 0; i < W; ++i) { acc[i] += w2 * y[gn * W + i]; }
                    } else {
#pragma unroll
                        for (int i = 0; i < W; ++i) { acc[i] += w * y[gn * W + i]; }
                    }
                }
            }
        }
        if (!PRECOND && st && st[ni].lam > 0.0) {
#pragma unroll
            for (int i = 0; i < W; ++i) { acc[i] += st[ni].lam * v[g * W + i]; }
        }
#pragma unroll
        for (int i = 0; i < W; ++i) { out[g * W + i] = acc[i]; }
    }
}

// z_f = (P_f + lam I)^{-1} r_f with the Newton-solve fallbacks (src/solve.hpp).
template <int D>
__global__ void ctl_precond_apply_kernel(CtlTables T, int64_t total_free, const double* __restrict__ prec,
                                         const double* __restrict__ r, double* __restrict__ z,
                                         const PcgState* __restrict__ st)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_free;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.free_pfx, T.n_nets, g);
        if (st[ni].done) { continue; }
        const double lam = st[ni].lam;
        const double* P = prec + g * D * D;
        double rhs[3], x[3];
#pragma unroll
        for (int i = 0; i < D; ++i) { rhs[i] = -r[g * D + i]; }
        if (D == 2) {
            const double H[4] = {P[0] + lam, P[1], P[2], P[3] + lam};
            solve2<double>(H, rhs, x);
        } else {
            const double h6[6] = {P[0] + lam, P[1], P[2], P[4] + lam, P[5], P[8] + lam};
            solve3<double>(h6, rhs, x);
        }
#pragma unroll
        for (int i = 0; i < D; ++i) { z[g * D + i] = x[i]; }
    }
}

// Per-net reductions over the stacked free vector (one CTA row per net, fixed
// order, compensated), with the PCG scalar step of the reduction folded into
// thread 0 (src/control_solve.hpp:761-819):
enum {
    kRedStore = 0,   // out[net] = x . y
    kRedAmax,        // out[net] = max |x|
    kRedTrace,       // out[net] = sum of diagonals of the D x D blocks of x
    kRedInit,        // r.r:   b_norm2, stop2 = rtol^2 b, r_norm2; done when b == 0
    kRedRz0,         // r.z:   rz
    kRedPap,         // p.Ap:  stop on non-positive curvature, else alpha = rz / pAp
    kRedRr,          // r.r:   r_norm2; stop when <= stop2 (its = it + 1)
    kRedRz,          // r.z:   beta = rz_new / rz, rz = rz_new, ++it, stop at max_iter
};

template <int D, int OP>
__global__ void ctl_reduce_kernel(CtlTables T, const double* __restrict__ x, const double* __restrict__ y,
                                  double* __restrict__ out, PcgState* __restrict__ st, double rtol)
{
    const int ni = blockIdx.x;
    const bool skip = (OP >= kRedPap) && st[ni].done;
    if (skip) { return; }  // uniform across the CTA
    const int64_t W = OP == kRedTrace ? D * D : D;
    const int64_t lo = T.free_pfx[ni] * W, hi = T.free_pfx[ni + 1] * W;
    Comp acc {0.0, 0.0};
    double mx = 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        if (OP == kRedAmax) {
            mx = fmax(mx, fabs(x[i]));
        } else if (OP == kRedTrace) {
            const int64_t e = i - lo;
            if ((e % (D * D)) % (D + 1) == 0) { comp_add(acc, x[i]); }
        } else {
            comp_add(acc, x[i] * y[i]);
        }
    }
    // max via the min slot of the shared reducer
    double mn = -mx;
    if (!block_reduce(acc, mn)) { return; }
    const double v = OP == kRedAmax ? -mn : acc.s + acc.c;
    PcgState& s = st[ni];
    switch (OP) {
    case kRedStore:
    case kRedAmax:
    case kRedTrace: out[ni] = v; break;
    case kRedInit:
        s.b_norm2 = v;
        s.r_norm2 = v;
        {
            // rtol < 0: the per-net relative tolerance was preloaded into stop2
            const double rt = rtol >= 0.0 ? rtol : s.stop2;
            s.stop2 = rt * rt * v;
        }
        s.it = 0;
        s.its = 0;
        s.done = (v == 0.0 || !s.active || s.max_iter <= 0) ? 1 : 0;
        break;
    case kRedRz0: s.rz = v; break;
    case kRedPap:
        if (!(v > 0.0)) {
            s.its = s.it;
            s.done = 1;
        } else {
            s.alpha = s.rz / v;
        }
        break;
    case kRedRr:
        s.r_norm2 = v;
        if (v <= s.stop2) {
            s.its = s.it + 1;
            s.done = 1;
        }
        break;
    case kRedRz:
        s.beta = v / s.rz;
        s.rz = v;
        s.it += 1;
        if (s.it >= s.max_iter) {
            s.its = s.it;
            s.done = 1;
        }
        break;
    }
}

// PCG vector updates over the stacked free vector (skipping finished nets).
enum { kVecInit = 0, kVecAxpy2, kVecXpay, kVecCopy };

template <int D, int OP>
__global__ void ctl_vec_kernel(CtlTables T, int64_t total_free, double* __restrict__ a, double* __restrict__ b,
                               const double* __restrict__ c, const double* __restrict__ d,
                               const PcgState* __restrict__ st)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_free;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.free_pfx, T.n_nets, g);
        if (OP == kVecInit ? !st[ni].active : st[ni].done) { continue; }
#pragma unroll
        for (int i = 0; i < D; ++i) {
            const int64_t e = g * D + i;
            if (OP == kVecInit) {          // a = dC = 0, b = r = -G (c)
                a[e] = 0.0;
                b[e] = -c[e];
            } else if (OP == kVecAxpy2) {  // a = dC += alpha p (c); b = r -= alpha Ap (d)
                const double al = st[ni].alpha;
                a[e] += al * c[e];
                b[e] -= al * d[e];
            } else if (OP == kVecXpay) {   // a = p = z (c) + beta p
                a[e] = c[e] + st[ni].beta * a[e];
            } else {                       // a = p = z (c)
                a[e] = c[e];
            }
        }
    }
}

// Trial / commit on the net nodes: out[slot] = X[slot] + alpha[net] corr[node]
// (out may alias X for the commit).
template <int D>
__global__ void ctl_step_kernel(CtlTables T, int64_t total_nodes, const double* X, const double* __restrict__ corr,
                                const double* __restrict__ alpha, double* out)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_nodes;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.node_pfx, T.n_nets, g);
        const double al = alpha[ni];
        if (al == 0.0) { continue; }
        const CtlNet n = T.nets[ni];
        const int64_t slot = n.node_off + (g - n.n_off);
#pragma unroll
        for (int c = 0; c < D; ++c) { out[slot * D + c] = X[slot * D + c] + al * corr[g * D + c]; }
    }
}

// C[lattice(free)] += alpha[net] dC[free].
template <int D>
__global__ void ctl_commit_c_kernel(CtlTables T, int64_t total_free, const double* __restrict__ dC,
                                    const double* __restrict__ alpha, double* __restrict__ C)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_free;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.free_pfx, T.n_nets, g);
        const double al = alpha[ni];
        if (al == 0.0) { continue; }
        const CtlNet n = T.nets[ni];
        const int64_t ci = n.c_off + T.free_idx[g];
#pragma unroll
        for (int c = 0; c < D; ++c) { C[ci * D + c] += al * dC[g * D + c]; }
    }
}

}  // namespace egg_b200
