// egg_b200 device-side wire build: the bulk index arrays of the sweep-context
// wire, built by kernels from the blocks' global node ids.
//
// The wire is the reference's `build_flat_context`
// (egg/smoothing/flat_context.py:136-346, with its `cell_stencil` at :40-121):
//
//   * cells enumerated block by block in C order; corner b in [0, 2^D) packs
//     the per-axis offset bits, axis 0 most significant; sample id 2^D*cell+b
//     has corner C[cell, b], axis-k neighbour C[cell, b ^ bit_k] and sign +1
//     where bit k of b is clear, else -1 (flat_context.py:90-113);
//   * interior-eligible nodes (logical index in [1, n-2] on every axis of a
//     block whose axes are all >= 3 long) name (block, logical) and carry no
//     stored samples when the target is a uniform multiple of the identity
//     (flat_context.py:211-238); a later block overwrites an earlier one;
//   * membership rows (cell, a, b) -- node C[cell, a] meets sample (cell, b)
//     with role 0 (a == b), 1+k (a ^ b == bit_k) or -1 -- kept for moving,
//     non-interior nodes and stably sorted by node (flat_context.py:114-121,
//     240-260); P_of counts each moving DOF's rows (flat_context.py:262-272).
//
// Layout of the work: one thread per block slot (interior keys), per node
// (classification, DOF compaction), per cell (occurrence counts and fills,
// the energy stencil with vector stores) and per occurrence (rows).  The
// stable sort by node is a counting sort: an exclusive scan of the per-node
// occurrence counts gives each node's row range, the occurrences land there
// in any order, and one thread per node sorts its few (cell, corner) keys,
// which restores the (cell, a, b) order of the reference's stable argsort.
// Every output is therefore identical, bit for bit, to the NumPy builder's.
#include "egg_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace egg_b200
{
extern thread_local std::string g_last_error;  // session.cu

namespace wire
{

struct Fail : std::runtime_error {
    int code;
    Fail(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define WIRE_CK(call)                                                                                          \
    do {                                                                                                       \
        cudaError_t e__ = (call);                                                                              \
        if (e__ != cudaSuccess) {                                                                              \
            throw Fail(EGG_B200_ERUNTIME, std::string("CUDA error: ") + cudaGetErrorString(e__) + " at " +   \
                                            __FILE__ + ":" + std::to_string(__LINE__));                        \
        }                                                                                                      \
    } while (0)

template <class T> struct Buf {
    T* p = nullptr;
    size_t n = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() { reset(); }
    void reset()
    {
        if (p) { cudaFree(p); }
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count)
    {
        reset();
        if (count) { WIRE_CK(cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T))); }
        n = count;
    }
    void zero(cudaStream_t st)
    {
        if (n) { WIRE_CK(cudaMemsetAsync(p, 0, n * sizeof(T), st)); }
    }
    void upload(const T* h, size_t count, cudaStream_t st)
    {
        alloc(count);
        if (n) { WIRE_CK(cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, st)); }
    }
    void download(T* h, size_t count, cudaStream_t st) const
    {
        if (h && count) { WIRE_CK(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, st)); }
    }
};

// Block layout on the device: nodes per axis (3 entries, 1 past D), node and
// cell offsets of each block in the concatenated id array / cell list.
struct Blocks {
    int nb;
    int D;
    const int32_t* n;         // [3 nb]
    const int64_t* node_off;  // [nb + 1]
    const int64_t* cell_off;  // [nb + 1]
    const int64_t* ids;       // [node_off[nb]] global node ids
};

// Last b with off[b] <= i (off ascending, off[0] == 0, i < off[nb]); blocks
// without cells have off[b] == off[b + 1] and are skipped by the search.
__device__ __forceinline__ int find_block(const int64_t* off, int nb, int64_t i)
{
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

// Global ids of the 2^D corners of cell c (corner bit of axis 0 most significant).
__device__ __forceinline__ void cell_corners(const Blocks& B, int64_t c, int64_t* C)
{
    const int b = find_block(B.cell_off, B.nb, c);
    const int64_t lc = c - B.cell_off[b];
    const int64_t n1 = B.n[3 * b + 1], n2 = B.n[3 * b + 2];
    const int64_t* ids = B.ids + B.node_off[b];
    if (B.D == 2) {
        const int64_t i = lc / (n1 - 1), j = lc % (n1 - 1);
        const int64_t base = i * n1 + j;
        C[0] = ids[base];
        C[1] = ids[base + 1];
        C[2] = ids[base + n1];
        C[3] = ids[base + n1 + 1];
    } else {
        const int64_t c2 = n2 - 1, c1 = n1 - 1;
        const int64_t i = lc / (c1 * c2), j = (lc / c2) % c1, k = lc % c2;
        const int64_t base = (i * n1 + j) * n2 + k;
        for (int a = 0; a < 8; ++a) {
            C[a] = ids[base + (a >> 2) * n1 * n2 + ((a >> 1) & 1) * n2 + (a & 1)];
        }
    }
}

__device__ __forceinline__ int64_t gstride() { return int64_t(gridDim.x) * blockDim.x; }
__device__ __forceinline__ int64_t gtid() { return int64_t(blockIdx.x) * blockDim.x + threadIdx.x; }

// Interior keys: ((b + 1) << 32 | local slot) of the last (block, C-order
// slot) that holds node id strictly inside an eligible block; ids out of
// [0, N) raise the error flag.
__global__ void wire_interior_kernel(Blocks B, int64_t N, unsigned long long* key, int* err)
{
    const int64_t total = B.node_off[B.nb];
    for (int64_t i = gtid(); i < total; i += gstride()) {
        const int64_t id = B.ids[i];
        if (id < 0 || id >= N) {
            atomicExch(err, 1);
            continue;
        }
        if (!key) { continue; }
        const int b = find_block(B.node_off, B.nb, i);
        const int64_t loc = i - B.node_off[b];
        const int64_t n0 = B.n[3 * b], n1 = B.n[3 * b + 1], n2 = B.n[3 * b + 2];
        if (n0 < 3 || n1 < 3 || (B.D == 3 && n2 < 3)) { continue; }
        const int64_t l2 = loc % n2, l1 = (loc / n2) % n1, l0 = loc / (n1 * n2);
        const bool inner = l0 >= 1 && l0 <= n0 - 2 && l1 >= 1 && l1 <= n1 - 2 && (B.D == 2 || (l2 >= 1 && l2 <= n2 - 2));
        if (inner) { atomicMax(&key[id], (static_cast<unsigned long long>(b + 1) << 32) | static_cast<unsigned long long>(loc)); }
    }
}

// Per node: interior block / logical (constrained nodes keep their logical
// but take block -1, as the NumPy builder does), stored-DOF flag, moving flag
// as a count for the DOF compaction.
__global__ void wire_node_kernel(Blocks B, int64_t N, const unsigned long long* key, const uint8_t* moving,
                                 const uint8_t* stored, int32_t* node_block, int32_t* node_logical,
                                 uint8_t* stored_dof, int32_t* moving_cnt)
{
    for (int64_t n = gtid(); n < N; n += gstride()) {
        int32_t blk = -1;
        int32_t l[3] = {0, 0, 0};
        const unsigned long long k = key ? key[n] : 0ull;
        if (k) {
            blk = int32_t(k >> 32) - 1;
            const int64_t loc = int64_t(k & 0xffffffffull);
            const int64_t n1 = B.n[3 * blk + 1], n2 = B.n[3 * blk + 2];
            l[2] = int32_t(loc % n2);
            l[1] = int32_t((loc / n2) % n1);
            l[0] = int32_t(loc / (n1 * n2));
        }
        for (int d = 0; d < B.D; ++d) { node_logical[n * B.D + d] = l[d]; }
        if (stored && stored[n]) { blk = -1; }
        node_block[n] = blk;
        const bool mv = moving[n] != 0;
        stored_dof[n] = (mv && blk < 0) ? 1 : 0;
        moving_cnt[n] = mv ? 1 : 0;
    }
}

// Occurrences (cell, corner a) of stored-DOF nodes.  fill == nullptr: count
// them per node; otherwise place the key 2^D * cell + a in the node's range.
__global__ void wire_occ_kernel(Blocks B, int64_t ncell, const uint8_t* stored_dof, int32_t* cnt, int32_t* fill,
                                const int64_t* off, int64_t* occ)
{
    const int nc = 1 << B.D;
    for (int64_t c = gtid(); c < ncell; c += gstride()) {
        int64_t C[8];
        cell_corners(B, c, C);
        for (int a = 0; a < nc; ++a) {
            const int64_t id = C[a];
            if (!stored_dof[id]) { continue; }
            if (!fill) {
                atomicAdd(&cnt[id], 1);
            } else {
                const int s = atomicAdd(&fill[id], 1);
                occ[off[id] + s] = c * nc + a;
            }
        }
    }
}

// Restore ascending (cell, corner) order inside each node's occurrence range.
__global__ void wire_occ_sort_kernel(int64_t N, const int32_t* cnt, const int64_t* off, int64_t* occ)
{
    for (int64_t n = gtid(); n < N; n += gstride()) {
        const int m = cnt[n];
        if (m < 2) { continue; }
        int64_t* v = occ + off[n];
        for (int i = 1; i < m; ++i) {
            const int64_t x = v[i];
            int j = i - 1;
            while (j >= 0 && v[j] > x) {
                v[j + 1] = v[j];
                --j;
            }
            v[j + 1] = x;
        }
    }
}

// Membership rows of the stored DOFs: occurrence j expands to the 2^D rows
// j * 2^D + b (sample id 2^D * cell + b, role of corner a in it).
__global__ void wire_rows_kernel(Blocks B, int64_t nocc, const int64_t* occ, int32_t* role, int32_t* gc,
                                 int32_t* gn0, int32_t* gn1, int32_t* gn2, double* s0, double* s1, double* s2,
                                 int64_t* sid)
{
    const int D = B.D;
    const int nc = 1 << D;
    int32_t* gn[3] = {gn0, gn1, gn2};
    double* sg[3] = {s0, s1, s2};
    for (int64_t j = gtid(); j < nocc; j += gstride()) {
        const int64_t key = occ[j];
        const int64_t c = key / nc;
        const int a = int(key % nc);
        int64_t C[8];
        cell_corners(B, c, C);
        for (int b = 0; b < nc; ++b) {
            const int64_t r = j * nc + b;
            int rl = -1;
            if (a == b) {
                rl = 0;
            } else {
                for (int k = 0; k < D; ++k) {
                    if ((a ^ b) == (1 << (D - 1 - k))) { rl = 1 + k; }
                }
            }
            role[r] = rl;
            sid[r] = c * nc + b;
            gc[r] = int32_t(C[b]);
            for (int k = 0; k < D; ++k) {
                const int bit = 1 << (D - 1 - k);
                gn[k][r] = int32_t(C[b ^ bit]);
                sg[k][r] = (b & bit) ? -1.0 : 1.0;
            }
        }
    }
}

// DOF arrays: moving nodes in ascending id order.
__global__ void wire_dof_kernel(int64_t N, int D, const uint8_t* moving, const int64_t* dof_pos, const int32_t* cnt,
                                const int32_t* node_block, const int32_t* node_logical, int32_t* dof_idx,
                                int32_t* P_of, int32_t* interior_block, int32_t* interior_logical)
{
    const int nc = 1 << D;
    for (int64_t n = gtid(); n < N; n += gstride()) {
        if (!moving[n]) { continue; }
        const int64_t p = dof_pos[n];
        dof_idx[p] = int32_t(n);
        P_of[p] = nc * cnt[n];
        interior_block[p] = node_block[n];
        for (int d = 0; d < D; ++d) { interior_logical[p * D + d] = node_logical[n * D + d]; }
    }
}

// Energy stencil, one thread per cell: its 2^D samples are consecutive, so
// every array row is written with 16-byte vector stores.
template <int D>
__global__ void wire_stencil_kernel(Blocks B, int64_t ncell, int32_t* gc, int32_t* gn0, int32_t* gn1, int32_t* gn2,
                                    double* s0, double* s1, double* s2)
{
    constexpr int nc = 1 << D;
    int32_t* gn[3] = {gn0, gn1, gn2};
    double* sg[3] = {s0, s1, s2};
    for (int64_t c = gtid(); c < ncell; c += gstride()) {
        int64_t C[8];
        cell_corners(B, c, C);
        int32_t v[nc];
        for (int b = 0; b < nc; ++b) { v[b] = int32_t(C[b]); }
        int4* o = reinterpret_cast<int4*>(gc + c * nc);
        for (int q = 0; q < nc / 4; ++q) { o[q] = make_int4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]); }
        for (int k = 0; k < D; ++k) {
            const int bit = 1 << (D - 1 - k);
            int4* og = reinterpret_cast<int4*>(gn[k] + c * nc);
            for (int q = 0; q < nc / 4; ++q) {
                og[q] = make_int4(v[(4 * q) ^ bit], v[(4 * q + 1) ^ bit], v[(4 * q + 2) ^ bit], v[(4 * q + 3) ^ bit]);
            }
            double2* os = reinterpret_cast<double2*>(sg[k] + c * nc);
            for (int q = 0; q < nc / 2; ++q) {
                os[q] = make_double2(((2 * q) & bit) ? -1.0 : 1.0, ((2 * q + 1) & bit) ? -1.0 : 1.0);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Exclusive scan of n counts (int32 or uint8) into int64 offsets: tile sums,
// one CTA scanning the tile sums, then each tile rescanned with its offset.
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one int64 per thread; *total gets the sum.
__device__ int64_t block_exclusive_scan(int64_t v, int64_t* total)
{
    __shared__ int64_t warp_sum[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) { x += y; }
    }
    if (lane == 31) { warp_sum[w] = x; }
    __syncthreads();
    if (w == 0) {
        int64_t s = lane < nw ? warp_sum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) { s += y; }
        }
        warp_sum[lane] = s;  // inclusive prefix of warp totals
    }
    __syncthreads();
    const int64_t before = (w ? warp_sum[w - 1] : 0) + x - v;
    if (total) { *total = warp_sum[nw - 1]; }
    __syncthreads();
    return before;
}

template <class T> __global__ void __launch_bounds__(kScanThreads) scan_tile_sum_kernel(const T* in, int64_t n, int64_t* tile_sum)
{
    const int64_t base = int64_t(blockIdx.x) * kScanTile;
    int64_t s = 0;
    for (int r = 0; r < kScanItems; ++r) {
        const int64_t i = base + r * kScanThreads + threadIdx.x;
        if (i < n) { s += int64_t(in[i]); }
    }
    int64_t total = 0;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) { tile_sum[blockIdx.x] = total; }
}

// One CTA: tile_sum -> exclusive offsets in place; sum into *total.
__global__ void __launch_bounds__(1024) scan_tile_offsets_kernel(int64_t* tile_sum, int64_t ntiles, int64_t* total)
{
    int64_t carry = 0;
    for (int64_t b = 0; b < ntiles; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        const int64_t v = i < ntiles ? tile_sum[i] : 0;
        int64_t chunk = 0;
        const int64_t ex = block_exclusive_scan(v, &chunk);
        if (i < ntiles) { tile_sum[i] = carry + ex; }
        carry += chunk;
    }
    if (threadIdx.x == 0) { *total = carry; }
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const T* in, int64_t n, const int64_t* tile_off, int64_t* out)
{
    __shared__ int64_t tile[kScanTile];
    const int64_t base = int64_t(blockIdx.x) * kScanTile;
    for (int r = 0; r < kScanItems; ++r) {
        const int t = r * kScanThreads + threadIdx.x;
        const int64_t i = base + t;
        tile[t] = i < n ? int64_t(in[i]) : 0;
    }
    __syncthreads();
    int64_t run[kScanItems];
    int64_t s = 0;
    for (int q = 0; q < kScanItems; ++q) {
        run[q] = s;
        s += tile[threadIdx.x * kScanItems + q];
    }
    const int64_t before = block_exclusive_scan(s, nullptr) + tile_off[blockIdx.x];
    for (int q = 0; q < kScanItems; ++q) { tile[threadIdx.x * kScanItems + q] = before + run[q]; }
    __syncthreads();
    for (int r = 0; r < kScanItems; ++r) {
        const int t = r * kScanThreads + threadIdx.x;
        const int64_t i = base + t;
        if (i < n) { out[i] = tile[t]; }
    }
}

static int grid_for(int64_t n, int threads = 256)
{
    const int64_t want = (n + threads - 1) / threads;
    return int(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(148) * 16)));
}

// out[i] = sum of in[0..i); returns the total (synchronises the stream).
template <class T> static int64_t exclusive_scan(const T* in, int64_t n, int64_t* out, cudaStream_t st)
{
    if (n == 0) { return 0; }
    const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
    Buf<int64_t> part;
    part.alloc(size_t(ntiles) + 1);
    scan_tile_sum_kernel<T><<<unsigned(ntiles), kScanThreads, 0, st>>>(in, n, part.p);
    WIRE_CK(cudaGetLastError());
    scan_tile_offsets_kernel<<<1, 1024, 0, st>>>(part.p, ntiles, part.p + ntiles);
    WIRE_CK(cudaGetLastError());
    scan_apply_kernel<T><<<unsigned(ntiles), kScanThreads, 0, st>>>(in, n, part.p, out);
    WIRE_CK(cudaGetLastError());
    int64_t total = 0;
    WIRE_CK(cudaMemcpyAsync(&total, part.p + ntiles, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    WIRE_CK(cudaStreamSynchronize(st));
    return total;
}

}  // namespace wire
}  // namespace egg_b200

// ===========================================================================
// C-ABI
// ===========================================================================
using namespace egg_b200::wire;

struct egg_b200_wire {
    int device = 0;
    int D = 0;
    int64_t n_dofs = 0, n_rows = 0, n_samples = 0;
    bool stencil = false;
    Buf<int32_t> dof_idx, P_of, interior_block, interior_logical;
    Buf<int32_t> role, gc, gn[3];
    Buf<double> s[3];
    Buf<int64_t> sid;
    Buf<int32_t> es_gc, es_gn[3];
    Buf<double> es_s[3];
};

namespace
{

template <class F> int wire_guarded(F&& f)
{
    try {
        f();
        return EGG_B200_OK;
    } catch (const Fail& e) {
        egg_b200::g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        egg_b200::g_last_error = "egg_b200: host out of memory";
        return EGG_B200_ERUNTIME;
    } catch (const std::exception& e) {
        egg_b200::g_last_error = e.what();
        return EGG_B200_ERUNTIME;
    }
}

[[noreturn]] void wire_invalid(const std::string& m) { throw Fail(EGG_B200_EINVAL, m); }

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { WIRE_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~Stream()
    {
        if (s) { cudaStreamDestroy(s); }
    }
};

void build_wire(const egg_b200_wire_desc& d, egg_b200_wire& W)
{
    const int D = d.dim;
    if (D != 2 && D != 3) { wire_invalid("wire: dimension must be 2 or 3, got " + std::to_string(D)); }
    const int nb = d.num_blocks;
    if (nb < 0) { wire_invalid("wire: negative block count"); }
    const int64_t N = d.num_nodes;
    if (N < 0) { wire_invalid("wire: negative num_nodes"); }
    if (N > std::numeric_limits<int32_t>::max()) {
        throw Fail(EGG_B200_ENOTSUP, "wire: node ids must fit int32 (the wire's index type)");
    }
    if (nb > 0 && !d.shapes) { wire_invalid("wire: shapes is NULL"); }
    if (N > 0 && !d.moving) { wire_invalid("wire: moving mask is NULL"); }
    const int nc = 1 << D;
    std::vector<int32_t> n3(size_t(3) * nb, 1);
    std::vector<int64_t> node_off(nb + 1, 0), cell_off(nb + 1, 0);
    for (int b = 0; b < nb; ++b) {
        int64_t nodes = 1, cells = 1;
        for (int k = 0; k < D; ++k) {
            const int32_t v = d.shapes[b * D + k];
            if (v < 1) { wire_invalid("wire: block shape entries must be >= 1"); }
            n3[3 * b + k] = v;
            nodes *= v;
            cells *= (v - 1);
        }
        node_off[b + 1] = node_off[b] + nodes;
        cell_off[b + 1] = cell_off[b] + cells;
    }
    const int64_t total = node_off[nb], ncell = cell_off[nb];
    if (total > 0 && !d.block_ids) { wire_invalid("wire: block_ids is NULL"); }
    if (total > std::numeric_limits<int32_t>::max()) {
        throw Fail(EGG_B200_ENOTSUP, "wire: the blocks hold more than 2^31 node slots");
    }

    int dev = d.device;
    if (dev < 0) { WIRE_CK(cudaGetDevice(&dev)); }
    WIRE_CK(cudaSetDevice(dev));
    W.device = dev;
    W.D = D;
    Stream stream;
    cudaStream_t st = stream.s;

    Buf<int32_t> n_d;
    Buf<int64_t> noff_d, coff_d, ids_d;
    n_d.upload(n3.data(), n3.size(), st);
    noff_d.upload(node_off.data(), node_off.size(), st);
    coff_d.upload(cell_off.data(), cell_off.size(), st);
    ids_d.upload(d.block_ids, size_t(total), st);
    Buf<uint8_t> moving, stored;
    moving.upload(d.moving, size_t(N), st);
    if (d.stored) { stored.upload(d.stored, size_t(N), st); }
    Blocks B {nb, D, n_d.p, noff_d.p, coff_d.p, ids_d.p};

    Buf<int> err;
    err.alloc(1);
    err.zero(st);
    Buf<unsigned long long> key;
    if (d.synth_interior) {
        key.alloc(size_t(N));
        key.zero(st);
    }
    if (total > 0) {
        wire_interior_kernel<<<grid_for(total), 256, 0, st>>>(B, N, key.p, err.p);
        WIRE_CK(cudaGetLastError());
    }
    int err_h = 0;
    WIRE_CK(cudaMemcpyAsync(&err_h, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    WIRE_CK(cudaStreamSynchronize(st));
    if (err_h) { wire_invalid("wire: a block id is out of range [0, num_nodes)"); }

    Buf<int32_t> node_block, node_logical, moving_cnt, cnt;
    Buf<uint8_t> stored_dof;
    node_block.alloc(size_t(N));
    node_logical.alloc(size_t(N) * D);
    moving_cnt.alloc(size_t(N));
    stored_dof.alloc(size_t(N));
    cnt.alloc(size_t(N));
    cnt.zero(st);
    if (N > 0) {
        wire_node_kernel<<<grid_for(N), 256, 0, st>>>(B, N, key.p, moving.p, stored.p, node_block.p, node_logical.p,
                                                      stored_dof.p, moving_cnt.p);
        WIRE_CK(cudaGetLastError());
    }
    if (ncell > 0) {
        wire_occ_kernel<<<grid_for(ncell), 256, 0, st>>>(B, ncell, stored_dof.p, cnt.p, nullptr, nullptr, nullptr);
        WIRE_CK(cudaGetLastError());
    }
    Buf<int64_t> occ_off, dof_pos;
    occ_off.alloc(size_t(N));
    dof_pos.alloc(size_t(N));
    const int64_t nocc = exclusive_scan(cnt.p, N, occ_off.p, st);
    const int64_t ndof = exclusive_scan(moving_cnt.p, N, dof_pos.p, st);
    Buf<int64_t> occ;
    occ.alloc(size_t(nocc));
    if (nocc > 0) {
        Buf<int32_t> fill;
        fill.alloc(size_t(N));
        fill.zero(st);
        wire_occ_kernel<<<grid_for(ncell), 256, 0, st>>>(B, ncell, stored_dof.p, cnt.p, fill.p, occ_off.p, occ.p);
        WIRE_CK(cudaGetLastError());
        wire_occ_sort_kernel<<<grid_for(N), 256, 0, st>>>(N, cnt.p, occ_off.p, occ.p);
        WIRE_CK(cudaGetLastError());
        WIRE_CK(cudaStreamSynchronize(st));  // fill is freed on return
    }
    const int64_t nrows = nocc * nc;
    W.n_dofs = ndof;
    W.n_rows = nrows;
    W.dof_idx.alloc(size_t(ndof));
    W.P_of.alloc(size_t(ndof));
    W.interior_block.alloc(size_t(ndof));
    W.interior_logical.alloc(size_t(ndof) * D);
    if (ndof > 0) {
        wire_dof_kernel<<<grid_for(N), 256, 0, st>>>(N, D, moving.p, dof_pos.p, cnt.p, node_block.p, node_logical.p,
                                                     W.dof_idx.p, W.P_of.p, W.interior_block.p, W.interior_logical.p);
        WIRE_CK(cudaGetLastError());
    }
    W.role.alloc(size_t(nrows));
    W.sid.alloc(size_t(nrows));
    W.gc.alloc(size_t(nrows));
    for (int k = 0; k < D; ++k) {
        W.gn[k].alloc(size_t(nrows));
        W.s[k].alloc(size_t(nrows));
    }
    if (nocc > 0) {
        wire_rows_kernel<<<grid_for(nocc), 256, 0, st>>>(B, nocc, occ.p, W.role.p, W.gc.p, W.gn[0].p, W.gn[1].p,
                                                         W.gn[2].p, W.s[0].p, W.s[1].p, W.s[2].p, W.sid.p);
        WIRE_CK(cudaGetLastError());
    }
    W.n_samples = ncell * nc;
    W.stencil = d.energy_arrays != 0;
    if (W.stencil) {
        W.es_gc.alloc(size_t(W.n_samples));
        for (int k = 0; k < D; ++k) {
            W.es_gn[k].alloc(size_t(W.n_samples));
            W.es_s[k].alloc(size_t(W.n_samples));
        }
        if (ncell > 0) {
            if (D == 2) {
                wire_stencil_kernel<2><<<grid_for(ncell), 256, 0, st>>>(B, ncell, W.es_gc.p, W.es_gn[0].p, W.es_gn[1].p,
                                                                         nullptr, W.es_s[0].p, W.es_s[1].p, nullptr);
            } else {
                wire_stencil_kernel<3><<<grid_for(ncell), 256, 0, st>>>(B, ncell, W.es_gc.p, W.es_gn[0].p, W.es_gn[1].p,
                                                                         W.es_gn[2].p, W.es_s[0].p, W.es_s[1].p,
                                                                         W.es_s[2].p);
            }
            WIRE_CK(cudaGetLastError());
        }
    }
    WIRE_CK(cudaStreamSynchronize(st));
}

}  // namespace

extern "C" {

int egg_b200_wire_build(const egg_b200_wire_desc* desc, egg_b200_wire** out)
{
    return wire_guarded([&] {
        if (!desc || !out) { wire_invalid("wire: NULL descriptor or output"); }
        *out = nullptr;
        auto W = std::make_unique<egg_b200_wire>();
        build_wire(*desc, *W);
        *out = W.release();
    });
}

int egg_b200_wire_sizes(egg_b200_wire* w, int64_t* sizes)
{
    return wire_guarded([&] {
        if (!w || !sizes) { wire_invalid("wire: NULL handle or output"); }
        sizes[0] = w->n_dofs;
        sizes[1] = w->n_rows;
        sizes[2] = w->n_samples;
    });
}

int egg_b200_wire_download(egg_b200_wire* w, const egg_b200_wire_out* o)
{
    return wire_guarded([&] {
        if (!w || !o) { wire_invalid("wire: NULL handle or output"); }
        WIRE_CK(cudaSetDevice(w->device));
        Stream stream;
        cudaStream_t st = stream.s;
        const size_t nd = size_t(w->n_dofs), nr = size_t(w->n_rows), ns = size_t(w->n_samples);
        w->dof_idx.download(o->dof_idx, nd, st);
        w->P_of.download(o->P_of, nd, st);
        w->interior_block.download(o->interior_block, nd, st);
        w->interior_logical.download(o->interior_logical, nd * w->D, st);
        w->role.download(o->role, nr, st);
        w->sid.download(o->sid, nr, st);
        w->gc.download(o->gc, nr, st);
        for (int k = 0; k < w->D; ++k) {
            w->gn[k].download(o->gn[k], nr, st);
            w->s[k].download(o->s[k], nr, st);
        }
        if (o->es_gc || o->es_gn[0] || o->es_s[0]) {
            if (!w->stencil) { wire_invalid("wire: built without the energy-stencil arrays"); }
            w->es_gc.download(o->es_gc, ns, st);
            for (int k = 0; k < w->D; ++k) {
                w->es_gn[k].download(o->es_gn[k], ns, st);
                w->es_s[k].download(o->es_s[k], ns, st);
            }
        }
        WIRE_CK(cudaStreamSynchronize(st));
    });
}

int egg_b200_wire_destroy(egg_b200_wire* w)
{
    return wire_guarded([&] {
        if (w) {
            cudaSetDevice(w->device);
            delete w;
        }
    });
}

}  // extern "C"
