// Reduced control solves: the layer that couples per-block nets in a
// multi-block topology (src/control_solve.hpp:1585-2610 ControlTopoSessionT,
// src/control_net.hpp:776-1106) and carries a single net's sliding walls
// (src/control_solve.hpp:820-1545).  The per-net kernels of control.cuh evaluate every net, gather
// per-node gradients / Hessian-vector products / Hessian blocks over each
// block's own cells and pull them back onto that net's lattice; here:
//   * alias sums over the copies of a shared node (the owner's net node takes
//     the group's total, the other copies are zeroed: the adjoint of the
//     owner -> copy broadcast) and alias broadcasts (copies take the owner's
//     value, as the store's owner -> copy refresh does for positions);
//   * CSR products for the reduction dC = R dq over the stacked lattice
//     components, its transpose Rᵀ (a gather CSR), and penalty rows
//     1/2 sum_j w_j (P_j C)^2 with their transpose;
//   * the scalar Jacobi diagonal of the reduced system, d_c = sum over the
//     controls of R's column c of a^T P_ctrl a;
//   * vector updates and reductions over the reduced (q) space.  The dots
//     run in one CTA in a fixed order, so every run reduces alike.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "control.cuh"

namespace egg_b200
{

// Scalars of the reduced-system PCG, resident on the device: the reduction
// CTAs advance them and set `done`, the update kernels skip once it is set,
// so a CG iteration needs no host round trip.  `its` follows the reference's
// count (src/control_solve.hpp:2565-2610): a breakdown (p.Ap <= 0) stops
// before the iteration counts, reaching the tolerance counts it, and
// max_iter caps it.
struct TopoPcg {
    double b_norm2, stop2, r_norm2, rz, alpha, beta, rtol, pad;
    int32_t it, its, done, max_iter;
};

// out[f] = C[lattice(f)] over the stacked free controls (D reals each).
template <int D>
__global__ void ctl_gather_free_kernel(CtlTables T, int64_t total_free, const double* __restrict__ C,
                                       double* __restrict__ out)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_free;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.free_pfx, T.n_nets, g);
        const int64_t ci = T.nets[ni].c_off + T.free_idx[g];
#pragma unroll
        for (int c = 0; c < D; ++c) { out[g * D + c] = C[ci * D + c]; }
    }
}

// out[i] = sum_e coef[e] v[col[e]] over row i's entries.
__global__ void topo_csr_apply_kernel(int64_t n_rows, const int32_t* __restrict__ off, const int32_t* __restrict__ col,
                                      const double* __restrict__ coef, const double* __restrict__ v,
                                      double* __restrict__ out)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_rows; i += int64_t(gridDim.x) * blockDim.x) {
        double acc = 0.0;
        for (int32_t e = off[i]; e < off[i + 1]; ++e) { acc += coef[e] * v[col[e]]; }
        out[i] = acc;
    }
}

// out[i] += sum_e coef[e] w[row[e]] r[row[e]] (Pᵀ W r over the transpose CSR).
__global__ void topo_csrT_accum_kernel(int64_t n_rows, const int32_t* __restrict__ off, const int32_t* __restrict__ row,
                                       const double* __restrict__ coef, const double* __restrict__ w,
                                       const double* __restrict__ r, double* __restrict__ out)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_rows; i += int64_t(gridDim.x) * blockDim.x) {
        double acc = 0.0;
        for (int32_t e = off[i]; e < off[i + 1]; ++e) { acc += coef[e] * w[row[e]] * r[row[e]]; }
        out[i] += acc;
    }
}

// Alias groups of net nodes (owner first).  SUM: the owner takes the group's
// total and the copies are zeroed; otherwise the copies take the owner's
// value.  ncomp reals per node.
template <bool SUM>
__global__ void topo_alias_kernel(int64_t n_groups, const int32_t* __restrict__ g_off, const int64_t* __restrict__ g_node,
                                  int ncomp, double* __restrict__ buf)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < n_groups; g += int64_t(gridDim.x) * blockDim.x) {
        const int64_t owner = g_node[g_off[g]];
        for (int c = 0; c < ncomp; ++c) {
            if (SUM) {
                double acc = 0.0;
                for (int32_t e = g_off[g]; e < g_off[g + 1]; ++e) { acc += buf[g_node[e] * ncomp + c]; }
                buf[owner * ncomp + c] = acc;
                for (int32_t e = g_off[g] + 1; e < g_off[g + 1]; ++e) { buf[g_node[e] * ncomp + c] = 0.0; }
            } else {
                const double v = buf[owner * ncomp + c];
                for (int32_t e = g_off[g] + 1; e < g_off[g + 1]; ++e) { buf[g_node[e] * ncomp + c] = v; }
            }
        }
    }
}

// Scalar Jacobi diagonal of the reduced system: for column c of R, the
// entries on one control (its D components are adjacent rows) form a; d_c
// adds a^T P_ctrl a over those controls (src/control_net.hpp:988-1020).
template <int D>
__global__ void topo_qdiag_build_kernel(int64_t nq, const int32_t* __restrict__ g_off, const int32_t* __restrict__ g_row,
                                        const double* __restrict__ g_coef, const double* __restrict__ prec,
                                        double* __restrict__ diag)
{
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < nq; c += int64_t(gridDim.x) * blockDim.x) {
        double d = 0.0;
        int32_t e = g_off[c];
        const int32_t e_end = g_off[c + 1];
        while (e < e_end) {
            const int32_t ctrl = g_row[e] / D;
            double a[D];
#pragma unroll
            for (int k = 0; k < D; ++k) { a[k] = 0.0; }
            while (e < e_end && g_row[e] / D == ctrl) {
                a[g_row[e] % D] = g_coef[e];
                ++e;
            }
            const double* P = prec + int64_t(ctrl) * D * D;
#pragma unroll
            for (int i = 0; i < D; ++i) {
#pragma unroll
                for (int j = 0; j < D; ++j) { d += a[i] * P[i * D + j] * a[j]; }
            }
        }
        diag[c] = d;
    }
}

// z = r / (d + lam) where d + lam > 0, else z = r.
__global__ void topo_qdiag_apply_kernel(int64_t nq, const double* __restrict__ diag, double lam,
                                        const double* __restrict__ r, double* __restrict__ z)
{
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < nq; c += int64_t(gridDim.x) * blockDim.x) {
        const double d = diag[c] + lam;
        z[c] = d > 0.0 ? r[c] / d : r[c];
    }
}

// The same inside the device-resident PCG (skipped once it has stopped).
__global__ void topo_qdiag_apply_pcg_kernel(int64_t nq, const double* __restrict__ diag, double lam,
                                            const double* __restrict__ r, double* __restrict__ z,
                                            const TopoPcg* __restrict__ st)
{
    if (st->done) { return; }
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < nq; c += int64_t(gridDim.x) * blockDim.x) {
        const double d = diag[c] + lam;
        z[c] = d > 0.0 ? r[c] / d : r[c];
    }
}

enum TopoVecOp : int {
    kTopoNeg = 0,   // a = -c
    kTopoAxpy = 1,  // a += s c
    kTopoXpay = 2,  // a = c + s a
    kTopoCopy = 3,  // a = c
    kTopoZero = 4,  // a = 0
};

template <int OP>
__global__ void topo_vec_kernel(int64_t n, double* __restrict__ a, const double* __restrict__ c, double s)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        if (OP == kTopoNeg) {
            a[i] = -c[i];
        } else if (OP == kTopoAxpy) {
            a[i] += s * c[i];
        } else if (OP == kTopoXpay) {
            a[i] = c[i] + s * a[i];
        } else if (OP == kTopoCopy) {
            a[i] = c[i];
        } else {
            a[i] = 0.0;
        }
    }
}

enum TopoRedOp : int {
    kTopoDot = 0,   // out = x . y
    kTopoAmax = 1,  // out = max |x|
};

// Fixed-order block reduction of x . y (compensated per thread) or max |x|
// over one CTA of 1024 threads: thread t takes items t, t + 1024, ... and a
// tree combines the threads; the result lands in part[0].
template <int OP>
__device__ __forceinline__ void topo_block_reduce(int64_t n, const double* __restrict__ x,
                                                  const double* __restrict__ y, double* part)
{
    const int t = threadIdx.x;
    double s = 0.0, comp = 0.0;
    for (int64_t i = t; i < n; i += 1024) {
        if (OP == kTopoDot) {
            const double v = x[i] * y[i] - comp;
            const double u = s + v;
            comp = (u - s) - v;
            s = u;
        } else {
            s = fmax(s, fabs(x[i]));
        }
    }
    part[t] = s;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if (t < w) { part[t] = OP == kTopoDot ? part[t] + part[t + w] : fmax(part[t], part[t + w]); }
        __syncthreads();
    }
}

template <int OP>
__global__ void __launch_bounds__(1024) topo_reduce_kernel(int64_t n, const double* __restrict__ x,
                                                           const double* __restrict__ y, double* __restrict__ out)
{
    __shared__ double part[1024];
    topo_block_reduce<OP>(n, x, y, part);
    if (threadIdx.x == 0) { *out = part[0]; }
}

// ---------------------------------------------------------------------------
// Jacobi-preconditioned CG on the reduced system (src/control_solve.hpp:
// 2565-2610 pcg_solve_q), its scalars in TopoPcg.

enum TopoPcgOp : int {
    kTopoPcgInit = 0,  // b_norm2 = r.r
    kTopoPcgRz0 = 1,   // rz = r.z
    kTopoPcgPap = 2,   // alpha = rz / p.Ap, or stop on breakdown
    kTopoPcgRr = 3,    // r_norm2 = r.r, stop at the tolerance
    kTopoPcgRz = 4,    // beta = r.z / rz; one iteration done
};

template <int OP>
__global__ void __launch_bounds__(1024) topo_pcg_reduce_kernel(int64_t n, const double* __restrict__ x,
                                                               const double* __restrict__ y, TopoPcg* __restrict__ st)
{
    __shared__ double part[1024];
    if (OP != kTopoPcgInit && OP != kTopoPcgRz0 && st->done) { return; }
    topo_block_reduce<kTopoDot>(n, x, y, part);
    if (threadIdx.x != 0) { return; }
    const double v = part[0];
    TopoPcg s = *st;
    if (OP == kTopoPcgInit) {
        s.b_norm2 = v;
        s.r_norm2 = v;
        s.stop2 = s.rtol * s.rtol * v;
        s.it = 0;
        s.its = 0;
        s.done = (v == 0.0 || s.max_iter <= 0) ? 1 : 0;
    } else if (OP == kTopoPcgRz0) {
        s.rz = v;
    } else if (OP == kTopoPcgPap) {
        if (!(v > 0.0)) {
            s.done = 1;
            s.its = s.it;
        } else {
            s.alpha = s.rz / v;
        }
    } else if (OP == kTopoPcgRr) {
        s.r_norm2 = v;
        if (v <= s.stop2) {
            s.done = 1;
            s.its = s.it + 1;
        }
    } else {
        s.beta = v / s.rz;
        s.rz = v;
        s.it += 1;
        if (s.it >= s.max_iter) {
            s.done = 1;
            s.its = s.it;
        }
    }
    *st = s;
}

// dq += alpha p, r -= alpha Ap.
__global__ void topo_pcg_step_kernel(int64_t n, double* __restrict__ dq, double* __restrict__ r,
                                     const double* __restrict__ p, const double* __restrict__ ap,
                                     const TopoPcg* __restrict__ st)
{
    if (st->done) { return; }
    const double a = st->alpha;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        dq[i] += a * p[i];
        r[i] -= a * ap[i];
    }
}

// p = z + beta p.
__global__ void topo_pcg_xpay_kernel(int64_t n, double* __restrict__ p, const double* __restrict__ z,
                                     const TopoPcg* __restrict__ st)
{
    if (st->done) { return; }
    const double b = st->beta;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        p[i] = z[i] + b * p[i];
    }
}

}  // namespace egg_b200
