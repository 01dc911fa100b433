// FAS (nonlinear multigrid) device kernels: transfers between a parent level
// and its coarse level, elementwise helpers, and the paired line-search
// reduction of the safeguarded coarse correction.  Both levels are packed
// per-block stores (dense row-major blocks, D doubles per node).
//
// Transfers follow src/mg_transfer.hpp:116-341:
//   inject         x_c(b, I) = x_p(b, I .* f)                     (all coarse nodes)
//   full weighting tau_c(b, I) = sum_o prod_k w(o_k) g_p(b, I .* f + o)
//                  w = 1/2 (o = 0), 1/4 (o = +-1) on factor-2 axes, identity on
//                  factor-1 axes; only free coarse nodes, zero elsewhere
//   prolongation   c_p(b, J) = mean of the 2^m coarse corners bracketing J
//                  (m = number of odd coordinates of J on factor-2 axes)
#pragma once

#include "kernels2d.cuh"

namespace egg_b200
{

// Block of a flat node index: the largest b with blocks[b].off <= node.
__device__ __forceinline__ int find_block(const BlockInfo* blocks, int nb, int64_t node)
{
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (blocks[mid].off <= node) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

__device__ __forceinline__ void unravel3(int64_t f, const int32_t n[3], int I[3])
{
    I[2] = int(f % n[2]);
    f /= n[2];
    I[1] = int(f % n[1]);
    I[0] = int(f / n[1]);
}

__device__ __forceinline__ int64_t ravel3(const int32_t n[3], int i, int j, int k)
{
    return (int64_t(i) * n[1] + j) * n[2] + k;
}

struct Transfer {
    int32_t nb;
    const BlockInfo* parent;  // parent level blocks (offset, shape)
    const BlockInfo* coarse;  // coarse level blocks
    const int32_t* factor;    // [nb * 3], 1 or 2 (axis >= D: 1)
    int64_t n_parent, n_coarse;
};

template <int D>
__global__ void inject_kernel(Transfer t, const double* __restrict__ xp, double* __restrict__ xc)
{
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < t.n_coarse;
         c += int64_t(gridDim.x) * blockDim.x) {
        const int b = find_block(t.coarse, t.nb, c);
        const BlockInfo cb = t.coarse[b], pb = t.parent[b];
        int I[3];
        unravel3(c - cb.off, cb.n, I);
        const int64_t p = pb.off + ravel3(pb.n, I[0] * t.factor[3 * b], I[1] * t.factor[3 * b + 1],
                                          I[2] * t.factor[3 * b + 2]);
#pragma unroll
        for (int k = 0; k < D; ++k) { xc[D * c + k] = xp[D * p + k]; }
    }
}

// Full weighting of the parent gradient onto free coarse nodes.  Interior
// coarse nodes read only their own block; interface coarse nodes (listed in
// `iface`, with `iface_src[node * 3^D + e]` giving the parent slot of
// stencil entry e, or -1 for an unused entry) read across the face.
template <int D>
__global__ void full_weight_kernel(Transfer t, const double* __restrict__ gp, double* __restrict__ tc,
                                   const uint8_t* __restrict__ cfree, const int32_t* __restrict__ iface_slot,
                                   const int32_t* __restrict__ iface_src, int64_t n_iface)
{
    constexpr int NO = D == 2 ? 9 : 27;
    for (int64_t c = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; c < t.n_coarse;
         c += int64_t(gridDim.x) * blockDim.x) {
        if (cfree[c] == 2) { continue; }  // free interface node: table path below
        double acc[D];
#pragma unroll
        for (int k = 0; k < D; ++k) { acc[k] = 0.0; }
        if (cfree[c] == 1) {  // free interior node
            const int b = find_block(t.coarse, t.nb, c);
            const BlockInfo cb = t.coarse[b], pb = t.parent[b];
            int I[3];
            unravel3(c - cb.off, cb.n, I);
            const int f[3] = {t.factor[3 * b], t.factor[3 * b + 1], t.factor[3 * b + 2]};
            for (int e = 0; e < NO; ++e) {
                int rem = e;
                int F[3] = {I[0] * f[0], I[1] * f[1], I[2] * f[2]};
                double w = 1.0;
                bool valid = true;
                for (int k = 0; k < D; ++k) {
                    const int o = rem % 3 - 1;
                    rem /= 3;
                    if (f[k] == 1) {
                        if (o != 0) { valid = false; }
                    } else {
                        w *= o == 0 ? 0.5 : 0.25;
                        F[k] += o;
                    }
                }
                if (!valid) { continue; }
                const int64_t p = pb.off + ravel3(pb.n, F[0], F[1], F[2]);
#pragma unroll
                for (int k = 0; k < D; ++k) { acc[k] += w * gp[D * p + k]; }
            }
        }
#pragma unroll
        for (int k = 0; k < D; ++k) { tc[D * c + k] = acc[k]; }
    }
    // Interface rows (few): one thread per row after the grid-stride pass.
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n_iface;
         r += int64_t(gridDim.x) * blockDim.x) {
        const int64_t c = iface_slot[r];
        const int b = find_block(t.coarse, t.nb, c);
        const int f[3] = {t.factor[3 * b], t.factor[3 * b + 1], t.factor[3 * b + 2]};
        double acc[D];
#pragma unroll
        for (int k = 0; k < D; ++k) { acc[k] = 0.0; }
        for (int e = 0; e < NO; ++e) {
            const int32_t p = iface_src[r * NO + e];
            if (p < 0) { continue; }
            int rem = e;
            double w = 1.0;
            for (int k = 0; k < D; ++k) {
                const int o = rem % 3 - 1;
                rem /= 3;
                if (f[k] == 2) { w *= o == 0 ? 0.5 : 0.25; }
            }
#pragma unroll
            for (int k = 0; k < D; ++k) { acc[k] += w * gp[D * int64_t(p) + k]; }
        }
#pragma unroll
        for (int k = 0; k < D; ++k) { tc[D * c + k] = acc[k]; }
    }
}

// Multilinear prolongation of a coarse correction onto every parent node.
template <int D>
__global__ void prolong_kernel(Transfer t, const double* __restrict__ cc, double* __restrict__ cp)
{
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < t.n_parent;
         p += int64_t(gridDim.x) * blockDim.x) {
        const int b = find_block(t.parent, t.nb, p);
        const BlockInfo cb = t.coarse[b], pb = t.parent[b];
        int J[3];
        unravel3(p - pb.off, pb.n, J);
        int c[3], r[3];
        double w0 = 1.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int f = t.factor[3 * b + k];
            c[k] = J[k] / f;
            r[k] = J[k] % f;
            if (r[k] != 0) { w0 *= 0.5; }
        }
        double acc[D];
#pragma unroll
        for (int k = 0; k < D; ++k) { acc[k] = 0.0; }
        for (int e = 0; e < (1 << D); ++e) {
            int C[3] = {c[0], c[1], c[2]};
            bool valid = true;
            for (int k = 0; k < D; ++k) {
                if (((e >> k) & 1) == 0) { continue; }
                if (r[k] == 0) {
                    valid = false;
                    break;
                }
                C[k] += 1;
            }
            if (!valid) { continue; }
            const int64_t q = cb.off + ravel3(cb.n, C[0], C[1], C[2]);
#pragma unroll
            for (int k = 0; k < D; ++k) { acc[k] += w0 * cc[D * q + k]; }
        }
#pragma unroll
        for (int k = 0; k < D; ++k) { cp[D * p + k] = acc[k]; }
    }
}

// out = x + a c at nodes with mask != 0 (every node when mask is null), x
// elsewhere (src/mg_transfer.hpp:300).
template <int D>
__global__ void masked_axpy_kernel(double* out, const double* x, const double* c, double a, const uint8_t* mask,
                                   int64_t n)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const double ai = (mask == nullptr || mask[i]) ? a : 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) { out[D * i + k] = x[D * i + k] + ai * c[D * i + k]; }
    }
}

template <int D> __global__ void zero_unmasked_kernel(double* buf, const uint8_t* mask, int64_t n)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        if (mask[i]) { continue; }
#pragma unroll
        for (int k = 0; k < D; ++k) { buf[D * i + k] = 0.0; }
    }
}

__global__ void vec_sub_kernel(double* out, const double* a, const double* b, int64_t n)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        out[i] = a[i] - b[i];
    }
}

}  // namespace egg_b200
