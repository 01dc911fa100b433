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

// ---------------------------------------------------------------------------
// Sliding-wall frames of a topology (src/control_solve.hpp:126-300,
// src/control_net.hpp:320-470,1105-1300): projection of the sliding roots
// with their frozen tangents, the damped member move, the wall-face b
// re-extension, and the db/dC linearisation of that re-extension (the
// frozen -n n^T projector at each wall-face node, extended inward).
// ---------------------------------------------------------------------------

namespace egg_b200
{

// Foot of p on an entity blob of the frame wire and the dim - 1 unit
// tangents there (zero where the entity is not codim-1 or the chart is
// degenerate).  2D blobs: the fixed-size records, a B-spline curve
// (degree, n_ctrl, knot_off, ctrl_off, t0, t1, w_off, has_w) or a composite
// path (n_segs, rec_off), offsets into `arena`; 3D: the surface records.
// The tangents are those at the projection of the foot, as the reference's
// wall frame re-projects the foot (src/control_solve.hpp:66-90).
template <int D>
__device__ void frame_entity(int tag, const double* rec, const double* arena, const double* p, double* foot,
                             double t[2][3])
{
    for (int kt = 0; kt < 2; ++kt) { t[kt][0] = t[kt][1] = t[kt][2] = 0.0; }
    if (D == 2) {
        double fx, fy, tx = 0.0, ty = 0.0, gx, gy;
        if (tag == EGG_B200_TAG_COMPOSITE) {
            const double* recs = arena + int64_t(rec[1]);
            composite_frame(arena, recs, int(rec[0]), p[0], p[1], fx, fy, tx, ty);
            composite_frame(arena, recs, int(rec[0]), fx, fy, gx, gy, tx, ty);
        } else if (tag == EGG_B200_TAG_BSPLINE) {
            const BSplineCurve c = composite_bspline(rec, arena);
            double q = bspline_foot(c, p[0], p[1], INFINITY);
            if (!bspline_inside(c, q)) { q = bspline_clamp(c, q); }
            bspline_point(c, q, 0, fx, fy);
            double r = bspline_foot(c, fx, fy, INFINITY);
            if (!bspline_inside(c, r)) { r = bspline_clamp(c, r); }
            double jx, jy;
            bspline_point(c, r, 1, jx, jy);
            unit_or_e0(jx, jy, tx, ty);
        } else {
            entity_project(tag, rec, p[0], p[1], fx, fy);
            entity_tangent(tag, rec, fx, fy, tx, ty);
        }
        foot[0] = fx;
        foot[1] = fy;
        t[0][0] = tx;
        t[0][1] = ty;
    } else if (tag == EGG_B200_TAG_BSPLINESURF) {
        double io[3] = {p[0], p[1], p[2]}, B[6];
        bsurf_dof(kBsurfFrame, rec, arena, nullptr, nullptr, nullptr, 0.0, 0.0, nullptr, nullptr, nullptr, io, B);
        for (int k = 0; k < 3; ++k) { foot[k] = io[k]; }
        bsurf_dof(kBsurfFrame, rec, arena, nullptr, nullptr, nullptr, 0.0, 0.0, nullptr, nullptr, nullptr, io, B);
        for (int a = 0; a < 2; ++a) {
            for (int k = 0; k < 3; ++k) { t[a][k] = B[a * 3 + k]; }
        }
    } else {
        entity3_project(tag, rec, p, foot);
        if (is_surf3(tag)) {
            double q[2], J[2][3];
            p3_invert(tag, rec, foot, q);
            p3_clamp(tag, rec, q);
            p3_frame(tag, rec, q, J);
            p3_basis(tag, J, t);
        }
    }
    for (int kt = 0; kt < D - 1; ++kt) {
        double n = 0.0;
        for (int k = 0; k < D; ++k) { n += t[kt][k] * t[kt][k]; }
        n = sqrt(n);
        if (n > 0.0) {
            for (int k = 0; k < D; ++k) { t[kt][k] /= n; }
        }
    }
}

// Per sliding root: project the representative control, freeze the tangent
// frame (a degenerate tangent freezes the root), keep (foot, pos) and
// rewrite the root's reduction entries and their gather-CSR twins.
template <int D>
__global__ void topo_frame_slide_kernel(int n_slide, const int32_t* __restrict__ tag, const int32_t* __restrict__ rep,
                                        const double* __restrict__ params, int stride, const double* __restrict__ arena,
                                        const int32_t* __restrict__ entry_off, const int32_t* __restrict__ r_entry,
                                        const int32_t* __restrict__ kt, const int32_t* __restrict__ comp,
                                        const double* __restrict__ base, const int32_t* __restrict__ g_entry_of_r,
                                        const double* __restrict__ C, double* __restrict__ fp,
                                        double* __restrict__ r_coef, double* __restrict__ g_coef)
{
    const int si = blockIdx.x * blockDim.x + threadIdx.x;
    if (si >= n_slide) { return; }
    double pos[3] = {0.0, 0.0, 0.0}, foot[3] = {0.0, 0.0, 0.0}, t[2][3];
    for (int k = 0; k < D; ++k) { pos[k] = C[int64_t(rep[si]) * D + k]; }
    frame_entity<D>(tag[si], params + int64_t(si) * stride, arena, pos, foot, t);
    for (int a = 0; a < D - 1; ++a) {
        double n = 0.0;
        for (int k = 0; k < D; ++k) { n += t[a][k] * t[a][k]; }
        if (n < 1e-24) {
            for (int k = 0; k < D; ++k) { t[a][k] = 0.0; }
        }
    }
    for (int k = 0; k < D; ++k) {
        fp[int64_t(si) * 2 * D + k] = foot[k];
        fp[int64_t(si) * 2 * D + D + k] = pos[k];
    }
    for (int32_t e = entry_off[si]; e < entry_off[si + 1]; ++e) {
        const double v = base[e] * t[kt[e]][comp[e]];
        r_coef[r_entry[e]] = v;
        g_coef[g_entry_of_r[r_entry[e]]] = v;
    }
}

// C[row] += alpha * coef * (foot - pos) over every member row of every root
// (a row may belong to more than one root, hence the atomic adds).
template <int D>
__global__ void topo_member_move_kernel(int64_t n_members, const int32_t* __restrict__ members,
                                        const int32_t* __restrict__ mem_root, const double* __restrict__ mem_coef,
                                        const double* __restrict__ fp, double alpha, double* __restrict__ C)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n_members; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t row = members[i], si = mem_root[i];
        for (int k = 0; k < D; ++k) {
            const double diff = fp[si * 2 * D + k] - fp[si * 2 * D + D + k];
            atomicAdd(&C[row * D + k], alpha * mem_coef[i] * diff);
        }
    }
}

// Block-logical multi-index of net node f.
template <int D> __device__ __forceinline__ void net_unravel(const CtlNet& n, int64_t f, int L[3])
{
    L[0] = L[1] = L[2] = 0;
    for (int k = D - 1; k >= 0; --k) {
        L[k] = int(f % n.node_shape[k]);
        f /= n.node_shape[k];
    }
}

// Boolean-sum extension of a boundary field at net node f (delta in the
// net's node space): boundary rows pass through; interior rows take the sum
// over axes of the two faces' lerp minus (dim - 1) times the corner blend
// (src/control_net.hpp:322-375).
template <int D>
__device__ void tfi_ext_at(const CtlNet& n, const double* __restrict__ delta, int64_t f, const int L[3], double out[3])
{
    int64_t nstr[3];
    nstr[D - 1] = 1;
    for (int k = D - 2; k >= 0; --k) { nstr[k] = nstr[k + 1] * n.node_shape[k + 1]; }
    bool boundary = false;
    for (int k = 0; k < D; ++k) { boundary = boundary || L[k] == 0 || L[k] == n.node_shape[k] - 1; }
    if (boundary) {
        for (int c = 0; c < D; ++c) { out[c] = delta[f * D + c]; }
        return;
    }
    double xi[3];
    for (int k = 0; k < D; ++k) { xi[k] = double(L[k]) / double(n.node_shape[k] - 1); }
    for (int c = 0; c < D; ++c) { out[c] = 0.0; }
    for (int bits = 0; bits < (1 << D); ++bits) {
        double w = 1.0;
        int64_t cf = 0;
        for (int k = 0; k < D; ++k) {
            if (bits & (1 << k)) {
                w *= xi[k];
                cf += int64_t(n.node_shape[k] - 1) * nstr[k];
            } else {
                w *= 1.0 - xi[k];
            }
        }
        for (int c = 0; c < D; ++c) { out[c] -= double(D - 1) * w * delta[cf * D + c]; }
    }
    for (int ax = 0; ax < D; ++ax) {
        for (int side = 0; side < 2; ++side) {
            const int64_t fp = f + int64_t((side == 0 ? 0 : n.node_shape[ax] - 1) - L[ax]) * nstr[ax];
            const double w = side == 0 ? 1.0 - xi[ax] : xi[ax];
            for (int c = 0; c < D; ++c) { out[c] += w * delta[fp * D + c]; }
        }
    }
}

// Per node of every net with a wall face: the boundary delta of the b
// re-extension -- the entity's projection of the spline on the net's wall
// faces, X0 on its other outer faces, zero on seam faces and inside -- and,
// with the db/dC model on, the frozen -(I - sum t t^T) projector at listed
// wall-face nodes.  Xs, X0 and delta live in net-node space.
template <int D>
__global__ void topo_wall_delta_kernel(CtlTables T, int64_t total_nodes, const int32_t* __restrict__ net_has_wall,
                                       const int32_t* __restrict__ seam, const double* __restrict__ X0, int n_wf,
                                       const int32_t* __restrict__ wf_net, const int32_t* __restrict__ wf_axis,
                                       const int32_t* __restrict__ wf_side, const int32_t* __restrict__ wf_tag,
                                       const double* __restrict__ wf_params, int stride,
                                       const double* __restrict__ arena, const double* __restrict__ Xs, bool with_db,
                                       const int32_t* __restrict__ face_of_node, double* __restrict__ face_P,
                                       double* __restrict__ delta)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_nodes;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.node_pfx, T.n_nets, g);
        if (!net_has_wall[ni]) { continue; }
        const CtlNet n = T.nets[ni];
        int L[3];
        net_unravel<D>(n, g - n.n_off, L);
        bool boundary = false, on_seam = false;
        for (int k = 0; k < D; ++k) {
            const int side = L[k] == 0 ? 0 : (L[k] == n.node_shape[k] - 1 ? 1 : -1);
            if (side >= 0) {
                boundary = true;
                on_seam = on_seam || seam[ni * 2 * D + 2 * k + side] != 0;
            }
        }
        if (!boundary || on_seam) {
            for (int c = 0; c < D; ++c) { delta[g * D + c] = 0.0; }
            continue;
        }
        double xs[3] = {0.0, 0.0, 0.0}, exact[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < D; ++c) {
            xs[c] = Xs[g * D + c];
            exact[c] = X0[g * D + c];
        }
        for (int w = 0; w < n_wf; ++w) {
            if (wf_net[w] != ni) { continue; }
            const int end = wf_side[w] == 0 ? 0 : n.node_shape[wf_axis[w]] - 1;
            if (L[wf_axis[w]] != end) { continue; }
            double proj[3] = {0.0, 0.0, 0.0}, t[2][3];
            const double* rec = wf_params + int64_t(w) * stride;
            frame_entity<D>(wf_tag[w], rec, arena, xs, proj, t);
            for (int c = 0; c < D; ++c) { exact[c] = proj[c]; }
            if (with_db && face_of_node[g] >= 0) {
                // re-orthonormalise the tangents at the foot (degenerate ones
                // dropped); P = sum t t^T - I, or 0 without a tangent
                double on[2][3];
                int n_on = 0;
                for (int a = 0; a < D - 1; ++a) {
                    double v[3] = {t[a][0], t[a][1], t[a][2]};
                    for (int b = 0; b < n_on; ++b) {
                        double dp = 0.0;
                        for (int k = 0; k < D; ++k) { dp += on[b][k] * v[k]; }
                        for (int k = 0; k < D; ++k) { v[k] -= dp * on[b][k]; }
                    }
                    double nrm = 0.0;
                    for (int k = 0; k < D; ++k) { nrm += v[k] * v[k]; }
                    if (nrm > 1e-24) {
                        nrm = sqrt(nrm);
                        for (int k = 0; k < D; ++k) { on[n_on][k] = v[k] / nrm; }
                        ++n_on;
                    }
                }
                double* P = face_P + int64_t(face_of_node[g]) * D * D;
                for (int r = 0; r < D; ++r) {
                    for (int c = 0; c < D; ++c) {
                        double ttc = 0.0;
                        for (int b = 0; b < n_on; ++b) { ttc += on[b][r] * on[b][c]; }
                        double pv = n_on == 0 ? 0.0 : ttc;
                        if (r == c && n_on > 0) { pv -= 1.0; }
                        P[r * D + c] = pv;
                    }
                }
            }
        }
        for (int c = 0; c < D; ++c) { delta[g * D + c] = exact[c] - xs[c]; }
    }
}

// out = ext(delta) (ADD: out += ext(delta)) over the nodes of the nets whose
// flag is set (net-node space).
template <int D, bool ADD>
__global__ void topo_tfi_ext_kernel(CtlTables T, int64_t total_nodes, const int32_t* __restrict__ net_flag,
                                    const double* __restrict__ delta, double* __restrict__ out)
{
    for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < total_nodes;
         g += int64_t(gridDim.x) * blockDim.x) {
        const int ni = net_of(T.node_pfx, T.n_nets, g);
        if (!net_flag[ni]) { continue; }
        const CtlNet n = T.nets[ni];
        const int64_t f = g - n.n_off;
        int L[3];
        net_unravel<D>(n, f, L);
        double v[3];
        tfi_ext_at<D>(n, delta + n.n_off * D, f, L, v);
        for (int c = 0; c < D; ++c) { out[g * D + c] = (ADD ? out[g * D + c] : 0.0) + v[c]; }
    }
}

// db/dC forward at the wall-face nodes: delta(j) = P_j v(j).
template <int D>
__global__ void topo_db_delta_kernel(int64_t n_face, const int64_t* __restrict__ face_node,
                                     const double* __restrict__ face_P, const double* __restrict__ v,
                                     double* __restrict__ delta)
{
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n_face; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t g = face_node[j];
        const double* P = face_P + j * D * D;
        for (int r = 0; r < D; ++r) {
            double acc = 0.0;
            for (int c = 0; c < D; ++c) { acc += P[r * D + c] * v[g * D + c]; }
            delta[g * D + r] = acc;
        }
    }
}

// db/dC adjoint on the alias-summed node gradient: y(j) += P_j^T (ext^T
// y)(j).  ext^T at a face-interior node sums its own entry and the lerp
// weights along its axis line; at a block corner it subtracts (dim - 1)
// times the corner-blend moment of the interior; other nodes keep their own
// entry.  Only interior nodes and the face node itself are read, so face
// nodes update in place without a race (src/control_net.hpp:396-460).
template <int D>
__global__ void topo_db_adjoint_kernel(CtlTables T, int64_t n_face, const int64_t* __restrict__ face_node,
                                       const double* __restrict__ face_P, double* __restrict__ y)
{
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < n_face; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t g = face_node[j];
        const int ni = net_of(T.node_pfx, T.n_nets, g);
        const CtlNet n = T.nets[ni];
        int L[3];
        net_unravel<D>(n, g - n.n_off, L);
        int n_ext = 0, ext_ax = -1, ext_side = 0;
        for (int k = 0; k < D; ++k) {
            if (L[k] == 0) {
                ++n_ext;
                ext_ax = k;
                ext_side = 0;
            } else if (L[k] == n.node_shape[k] - 1) {
                ++n_ext;
                ext_ax = k;
                ext_side = 1;
            }
        }
        auto node = [&](const int* li) {
            int64_t f = 0;
            for (int k = 0; k < D; ++k) { f = f * n.node_shape[k] + li[k]; }
            return n.n_off + f;
        };
        double ds[3] = {0.0, 0.0, 0.0};
        for (int c = 0; c < D; ++c) { ds[c] = y[g * D + c]; }
        if (n_ext == 1) {
            int li[3] = {L[0], L[1], L[2]};
            for (int i = 1; i < n.node_shape[ext_ax] - 1; ++i) {
                li[ext_ax] = i;
                const double xi = double(i) / double(n.node_shape[ext_ax] - 1);
                const double w = ext_side == 0 ? 1.0 - xi : xi;
                const int64_t s = node(li);
                for (int c = 0; c < D; ++c) { ds[c] += w * y[s * D + c]; }
            }
        } else if (n_ext == D) {
            bool any = true;
            for (int k = 0; k < D; ++k) { any = any && n.node_shape[k] >= 3; }
            int li[3] = {1, 1, 1};
            while (any) {
                double w = 1.0;
                for (int k = 0; k < D; ++k) {
                    const double xi = double(li[k]) / double(n.node_shape[k] - 1);
                    w *= L[k] == 0 ? 1.0 - xi : xi;
                }
                const int64_t s = node(li);
                for (int c = 0; c < D; ++c) { ds[c] -= double(D - 1) * w * y[s * D + c]; }
                int k = D - 1;
                for (; k >= 0; --k) {
                    if (++li[k] < n.node_shape[k] - 1) { break; }
                    li[k] = 1;
                }
                if (k < 0) { break; }
            }
        }
        const double* P = face_P + j * D * D;
        for (int r = 0; r < D; ++r) {
            double acc = 0.0;
            for (int c = 0; c < D; ++c) { acc += P[c * D + r] * ds[c]; }
            y[g * D + r] += acc;
        }
    }
}

}  // namespace egg_b200
