// egg_b200 session: host-side validation and structured remap, device-resident
// state, the block-Jacobi driver, and the C-ABI declared in include/egg_b200.h.
#include "egg_b200.h"
#include "kernels2d.cuh"
#include "kernels2d_x2.cuh"
#include "kernels3d.cuh"
#include "fas.cuh"
#include "control.cuh"
#include "control_topo.cuh"

#include <algorithm>
#include <array>
#include <map>
#include <set>
#include <unordered_map>
#include <unordered_set>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace egg_b200
{

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

thread_local std::string g_last_error;

#define EGG_CK(call)                                                                        \
    do {                                                                                    \
        cudaError_t e__ = (call);                                                           \
        if (e__ != cudaSuccess) {                                                           \
            throw Error(EGG_B200_ERUNTIME, std::string("CUDA error: ") + cudaGetErrorString(e__) + \
                                             " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
        }                                                                                   \
    } while (0)

[[noreturn]] void invalid(const std::string& m) { throw Error(EGG_B200_EINVAL, m); }

// ---------------------------------------------------------------------------
// Device buffers
// ---------------------------------------------------------------------------
template <class T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { reset(); }
    void reset()
    {
        if (p) { cudaFree(p); }
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count)
    {
        reset();
        if (count) { EGG_CK(cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T))); }
        n = count;
    }
    // A cudaMemcpy from pageable memory may return before its DMA lands, and
    // the sessions' streams do not wait for the legacy stream: the copy is
    // complete when upload() returns, so kernels on any stream see it.
    void upload(const std::vector<T>& h)
    {
        alloc(h.size());
        copy_in(h);
    }
    // upload() that keeps an allocation of the same size; only for buffers
    // that no queued work still reads (the caller has synchronised).
    void put(const std::vector<T>& h)
    {
        if (h.size() != n) { alloc(h.size()); }
        copy_in(h);
    }
    void copy_in(const std::vector<T>& h)
    {
        if (!n) { return; }
        EGG_CK(cudaMemcpy(p, h.data(), n * sizeof(T), cudaMemcpyHostToDevice));
        EGG_CK(cudaStreamSynchronize(cudaStreamLegacy));
    }
};

// Launch variants of the interior kernel: cells per CTA (CI x CJ) and the
// minimum resident CTAs per SM requested from the register allocator.  The
// session's autotuner times each on the session's own data and keeps the
// fastest (egg_b200_session_autotune).
// 2D: (ci, cj) cells per CTA, or with fd = 1 (ci, cj) DOFs per CTA over the
// (ci+1) x (cj+1) cells around them; fd = 2 is the same full-DOF tile on the
// packed two-lane fp32 kernel (interior_x2_kernel, mixed precision only), fd
// = 3 its persistent form with TMA window prefetch (interior_x2p_kernel);
// 3D: (ci, cj, ck) DOFs per CTA.
struct Variant {
    int ci, cj, ck, minb, fd = 0;
};
constexpr int kNumVariants = EGG_B200_NUM_VARIANTS;
// Host threads that copy X between the caller's buffer and pinned staging.
constexpr int kMaxCopyThreads = 16;
constexpr Variant kVar64[kNumVariants] = {{8, 16, 1, 5, 1}, {8, 16, 1, 4}, {8, 16, 1, 5}, {8, 16, 1, 6}, {8, 16, 1, 4, 1}};
constexpr Variant kVar32[kNumVariants] = {{8, 16, 1, 7, 2}, {8, 16, 1, 8, 2}, {8, 16, 1, 6, 2}, {8, 16, 1, 5, 2}, {8, 16, 1, 7, 3}};
constexpr Variant kVar3_64[kNumVariants] = {{4, 8, 8, 1}, {4, 8, 8, 2}, {2, 8, 16, 2}, {2, 8, 16, 3}, {2, 4, 16, 4}};
constexpr Variant kVar3_32[kNumVariants] = {{4, 8, 8, 1}, {4, 8, 8, 2}, {2, 8, 16, 2}, {2, 8, 16, 3}, {2, 4, 16, 4}};

enum KernelId {
    kKInterior = 0,
    kKStored = 1,
    kKBroadcast = 2,
    kKReduce = 3,
    kKFinal = 4,
    kKCopy = 5,
    kKTransfer = 6,
    kKCtl = 7,
    kKCount = 8
};

// Device data of one relaxation level (the fine store or a coarse FAS level):
// block layout, structured-interior DOFs (mask + tiles), stored-patch DOFs and
// the owner -> copy broadcast table.
struct LevelData {
    int64_t nstore = 0;
    std::vector<BlockInfo> blocks_h;
    DevBuf<BlockInfo> blocks_d;
    int64_t n_interior = 0;
    std::vector<uint8_t> active_h;
    // structured-interior DOF slots (the tile kernel's plus those relaxed as
    // stored DOFs for their soft terms): the FAS coarsening's interior set
    std::vector<uint8_t> interior_h;
    DevBuf<uint8_t> active_d;
    DevBuf<Tile2> tiles_d;   // 2D tiles of the current variant's shape
    DevBuf<Tile3> tiles3_d;  // 3D tiles of the current variant's shape
    int64_t ntiles = 0;
    int tile_ci = 0, tile_cj = 0, tile_ck = 0, tile_fd = 0;
    // the coarsest FAS level of a mixed-precision session sweeps its
    // interior with the fp64 kernels (tiles of the first fp64 variant)
    bool fp64_tiles = false;
    // interior-kernel variant of a coarse FAS level, tuned on the level's
    // own data (-1: the session's variant)
    int variant = -1;
    int64_t n_stored = 0;
    DevBuf<int32_t> st_slot, st_gc, st_gn0, st_gn1, st_gn2, st_role;
    DevBuf<int64_t> st_off;
    DevBuf<int8_t> st_s0, st_s1, st_s2;
    DevBuf<double> st_W, st_wt;
    int st_wstride = 0, st_wtstride = 0;
    int64_t n_constrained = 0;  // stored DOFs on a boundary entity
    int64_t n_arc = 0;          // of which on a parametric entity (arc, plane: cold first sweep per run call)
    int64_t n_bspline = 0;      // of which on a B-spline curve (seeded projection)
    int64_t n_composite = 0;    // of which on a composite path
    DevBuf<double> arena;       // entity arena (B-spline knots, control points, weights)
    DevBuf<double> seeds;       // [n_stored] last foot parameter of each B-spline DOF
    DevBuf<int8_t> st_etag;     // [n_stored] entity tag (uploaded when n_constrained > 0)
    DevBuf<double> st_epar;     // [n_stored * EGG_B200_ENTITY_FIELDS] entity records
    int64_t n_soft = 0;          // soft terms over the stored DOFs (0: none)
    DevBuf<int32_t> soft_off;    // [n_stored + 1] term ranges
    DevBuf<SoftTerm> soft_terms;
    double soft_eps = 0.0;
    int64_t nshare = 0;
    DevBuf<int32_t> sh_src, sh_dst;
};

#include "fas_types.inc"
#include "control_types.inc"

struct Session : LevelData {
    int dim = 2;
    int prec = EGG_B200_PREC_FP64;
    int device = 0;
    int num_sms = 148;
    // error flag of kernels with bounded waits (set on device, checked at sync)
    DevBuf<int> kerr;
    bool kerr_armed = false;
    cudaStream_t stream = nullptr;
    // side stream + fork/join events: the stored-patch sweep runs beside the
    // interior tiles (both read the frozen snapshot, write disjoint slots)
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;

    int64_t M = 0;       // global nodes
    std::vector<int32_t> g2s;       // global -> owner slot (-1 if in no block)
    std::vector<int32_t> slot_gid;  // store slot -> global id
    std::vector<int64_t> nb_gid;    // global nodes in no block: get_X returns
    std::vector<double> nb_val;     // their last value set ([nb_gid.size() * dim])
    // X transfers in global node order, allocated on first use: pinned host
    // staging, a device copy in global order, the device remap tables and
    // one event per host copy slice.
    double* pin = nullptr;
    DevBuf<double> Xg;
    DevBuf<int32_t> g2s_d, slot_gid_d;
    cudaEvent_t xfer_ev[kMaxCopyThreads] = {};

    DevBuf<double> Xbuf[2];
    int cur = 0;  // index of the canonical buffer

    // FAS: relaxed-DOF slots of the fine level, the fine halo relation, the
    // lazily built coarse hierarchy and fine scratch.
    std::vector<uint8_t> free_h;
    DevBuf<uint8_t> free_d;
    HaloHost halo;
    bool fas_built = false;
    std::vector<std::unique_ptr<CoarseLevel>> levels;
    DevBuf<double> fine_corr, fine_grad, trial;
    std::vector<double> fas_alphas;

    int variant = 0;
    bool tuned = false;
    bool pinned_variant = false;  // set_variant: every level sweeps with S.variant
    double variant_ms[kNumVariants] = {};
    // energy stencil
    bool es_struct = false;
    int64_t es_ns = 0;
    DevBuf<int64_t> es_cell_off;
    int64_t es_ncell = 0;
    DevBuf<int32_t> es_gc, es_gn0, es_gn1, es_gn2;
    DevBuf<int8_t> es_s0, es_s1, es_s2;
    DevBuf<double> es_W, es_wt;
    int es_wstride = 0, es_wtstride = 0;
    // whole-sample directional table: its total joins every reported energy
    int64_t es_dir_n = 0;
    DevBuf<SoftTerm> es_dir;
    double es_dir_eps = 0.0;
    DevBuf<int64_t> es_dir_seg;  // batch: [n_seg + 1] each mesh's range of es_dir
    // reductions
    int red_grid = 0;
    DevBuf<double> part;      // [3 * red_grid]
    DevBuf<double> red_out;   // [2 * capacity]
    DevBuf<double> red_tmp;   // [2 * n_seg or 2]: report slot written inside a captured chunk
    // batch: several independent meshes packed into one store
    int n_seg = 0;                       // meshes (0: a plain single-mesh session)
    std::vector<int64_t> mesh_node_off;  // [n_seg + 1] global node offsets
    DevBuf<int64_t> seg_d;               // [n_seg + 1] energy-stencil item (cell or sample) offsets
    int seg_gx = 0;                      // reduction CTAs per mesh
    DevBuf<double> seg_part;             // [3 * seg_gx * n_seg]
    // CUDA graphs of report chunks (k sweeps + the report reduction)
    struct ChunkGraph {
        int kind, k;
        bool per_mesh;
        double delta, omega;
        const double* xin;
        const double* xout;
        const void* tiles;
        int variant;
        cudaGraphExec_t exec;
        int64_t launches, updates;
    };
    std::vector<ChunkGraph> graphs;
    // control-net reduced Gauss-Newton (attached on request)
    std::unique_ptr<ControlState> ctl;
    // profiling
    bool profiling = false;
    int64_t launches = 0;  // every kernel launch (copies excluded)
    int64_t updates = 0;   // vertex Newton updates issued (every DOF relaxed once at any level)
    DevBuf<double> ckpt;   // device-side checkpoint of the store
    bool has_ckpt = false;
    double k_ms[kKCount] = {};
    int64_t k_launch[kKCount] = {};
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<cudaEvent_t> event_pool;

    void drop_graphs()
    {
        for (auto& g : graphs) { cudaGraphExecDestroy(g.exec); }
        graphs.clear();
    }

    ~Session()
    {
        if (stream) { cudaStreamSynchronize(stream); }
        drop_graphs();
        for (auto& p : pending) {
            event_pool.push_back(p.second.first);
            event_pool.push_back(p.second.second);
        }
        for (cudaEvent_t e : event_pool) { cudaEventDestroy(e); }
        if (side) { cudaStreamSynchronize(side); }
        if (fork_ev) { cudaEventDestroy(fork_ev); }
        if (join_ev) { cudaEventDestroy(join_ev); }
        if (side) { cudaStreamDestroy(side); }
        if (stream) { cudaStreamDestroy(stream); }
        for (cudaEvent_t e : xfer_ev) {
            if (e) { cudaEventDestroy(e); }
        }
        if (pin) { cudaFreeHost(pin); }
    }

    cudaEvent_t take_event()
    {
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        EGG_CK(cudaEventCreate(&e));
        return e;
    }

    template <class F> void timed(int kid, F&& launch)
    {
        if (kid != kKCopy) { ++launches; }
        if (!profiling) {
            launch();
            EGG_CK(cudaGetLastError());
            return;
        }
        cudaEvent_t a = take_event(), b = take_event();
        EGG_CK(cudaEventRecord(a, stream));
        launch();
        EGG_CK(cudaGetLastError());
        EGG_CK(cudaEventRecord(b, stream));
        pending.push_back({kid, {a, b}});
    }

    void harvest()
    {
        for (auto& p : pending) {
            float ms = 0.f;
            EGG_CK(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
            k_ms[p.first] += ms;
            k_launch[p.first] += 1;
            event_pool.push_back(p.second.first);
            event_pool.push_back(p.second.second);
        }
        pending.clear();
    }

    void sync()
    {
        EGG_CK(cudaStreamSynchronize(stream));
        harvest();
        check_kerr();
    }

    // A kernel whose bounded wait ran out set kerr: report it once as an error.
    void check_kerr()
    {
        if (!kerr_armed || kerr.p == nullptr) { return; }
        kerr_armed = false;
        int e = 0;
        EGG_CK(cudaMemcpy(&e, kerr.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (e != 0) {
            EGG_CK(cudaMemset(kerr.p, 0, sizeof(int)));
            throw Error(EGG_B200_ERUNTIME, "interior sweep: a window copy did not complete within its wait limit");
        }
    }

    double* X(int i) { return Xbuf[i].p; }
};

// ---------------------------------------------------------------------------
// X in global node order <-> the packed store
// ---------------------------------------------------------------------------
// store slot i <- X[slot_gid[i]]: every copy of a node takes its value.
template <int D>
__global__ void gather_global_kernel(const double* __restrict__ Xg, const int32_t* __restrict__ slot_gid, int64_t n,
                                     double* __restrict__ store)
{
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t g = slot_gid[i];
        if constexpr (D == 2) {
            reinterpret_cast<double2*>(store)[i] = reinterpret_cast<const double2*>(Xg)[g];
        } else {
#pragma unroll
            for (int k = 0; k < D; ++k) { store[i * D + k] = Xg[g * D + k]; }
        }
    }
}

// X[g] <- store[g2s[g]] (the owner slot) for every node in a block; nodes in
// no block are left for the host to fill.
template <int D>
__global__ void scatter_global_kernel(const double* __restrict__ store, const int32_t* __restrict__ g2s, int64_t M,
                                      double* __restrict__ Xg)
{
    for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < M; g += int64_t(gridDim.x) * blockDim.x) {
        const int64_t s = g2s[g];
        if (s < 0) { continue; }
        if constexpr (D == 2) {
            reinterpret_cast<double2*>(Xg)[g] = reinterpret_cast<const double2*>(store)[s];
        } else {
#pragma unroll
            for (int k = 0; k < D; ++k) { Xg[g * D + k] = store[s * D + k]; }
        }
    }
}

// Grid of the remap kernels: one thread per item up to 8 CTAs per SM.
static int remap_grid(int64_t n) { return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8))); }

// Host copy threads for a transfer of `bytes`: one per 4 MiB slice, at most
// the hardware threads and kMaxCopyThreads.
static int copy_threads(size_t bytes)
{
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t by_size = bytes >> 22;
    return int(std::max<size_t>(1, std::min({hw, size_t(kMaxCopyThreads), by_size})));
}

// Runs body(t) for t in [0, T): slice 0 on the calling thread, the others on
// new threads (inline when a thread cannot be started).  body must not throw.
template <class F> static void run_slices(int T, F&& body)
{
    std::vector<std::thread> th;
    th.reserve(size_t(std::max(T - 1, 0)));
    int started = 1;
    try {
        for (; started < T; ++started) { th.emplace_back(body, started); }
    } catch (...) {
    }
    for (int t = started; t < T; ++t) { body(t); }
    body(0);
    for (auto& x : th) { x.join(); }
}

// Slice t of T over n doubles.
static inline size_t slice_begin(size_t n, int t, int T) { return n * size_t(t) / size_t(T); }

// ---------------------------------------------------------------------------
// Session construction
// ---------------------------------------------------------------------------
static void check_len(int64_t got, int64_t want, const std::string& what)
{
    if (got != want) {
        invalid("validate_context: " + what + " size " + std::to_string(got) + " != " + std::to_string(want));
    }
}

static void require_ptr(const void* p, int64_t n, const std::string& what)
{
    if (n > 0 && p == nullptr) { invalid("session desc: " + what + " is NULL"); }
}

static std::vector<double> identity_row(int D)
{
    std::vector<double> w(size_t(D) * D, 0.0);
    for (int k = 0; k < D; ++k) { w[size_t(k) * D + k] = 1.0; }
    return w;
}

static bool rows_uniform(const double* W, int64_t rows, int width)
{
    for (int64_t r = 1; r < rows; ++r) {
        if (std::memcmp(W + r * width, W, sizeof(double) * width) != 0) { return false; }
    }
    return true;
}

// Opt the interior kernels into >48 KB of dynamic shared memory.
template <int CI, int CJ, int FD, int KIND, class C> constexpr size_t tile_smem2()
{
    if constexpr (FD == 2) {
        return sizeof(TileSharedX2<CI, CJ>);
    } else if constexpr (FD == 3) {
        return sizeof(TileSharedX2<CI, CJ, 2>);
    } else {
        return sizeof(TileShared2<CI + FD, CJ + FD, C, KIND>);
    }
}

template <int CI, int CJ, int MINB, class C, int FD> static void set_smem_attr()
{
    if constexpr (FD == 3) {
        static_assert(std::is_same_v<C, float>, "the packed kernel is the mixed-precision path");
        constexpr int sz = int(sizeof(TileSharedX2<CI, CJ, 2>));
        EGG_CK(cudaFuncSetAttribute(interior_x2p_kernel<CI, CJ, MINB, kShape>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
        EGG_CK(cudaFuncSetAttribute(interior_x2p_kernel<CI, CJ, MINB, kUntangle>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
        EGG_CK(cudaFuncSetAttribute(interior_x2p_kernel<CI, CJ, MINB, kShapeSize>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, sz));
        return;
    } else if constexpr (FD == 2) {
        static_assert(std::is_same_v<C, float>, "the packed kernel is the mixed-precision path");
        EGG_CK(cudaFuncSetAttribute(interior_x2_kernel<CI, CJ, MINB, kShape>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(TileSharedX2<CI, CJ>))));
        EGG_CK(cudaFuncSetAttribute(interior_x2_kernel<CI, CJ, MINB, kUntangle>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(TileSharedX2<CI, CJ>))));
        EGG_CK(cudaFuncSetAttribute(interior_x2_kernel<CI, CJ, MINB, kShapeSize>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(TileSharedX2<CI, CJ>))));
        return;
    } else {
    EGG_CK(cudaFuncSetAttribute(interior_tile_kernel<CI, CJ, MINB, kShape, C, FD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, int(tile_smem2<CI, CJ, FD, kShape, C>())));
    EGG_CK(cudaFuncSetAttribute(interior_tile_kernel<CI, CJ, MINB, kUntangle, C, FD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(tile_smem2<CI, CJ, FD, kUntangle, C>())));
    EGG_CK(cudaFuncSetAttribute(interior_tile_kernel<CI, CJ, MINB, kShapeSize, C, FD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(tile_smem2<CI, CJ, FD, kShapeSize, C>())));
    }
}

static void configure_kernels(int prec, int dim)
{
    if (dim == 3) { return; }  // 3D kernels use < 48 KB of static shared memory
    if (prec == EGG_B200_PREC_FP64) {
        set_smem_attr<kVar64[0].ci, kVar64[0].cj, kVar64[0].minb, double, kVar64[0].fd>();
        set_smem_attr<kVar64[1].ci, kVar64[1].cj, kVar64[1].minb, double, kVar64[1].fd>();
        set_smem_attr<kVar64[2].ci, kVar64[2].cj, kVar64[2].minb, double, kVar64[2].fd>();
        set_smem_attr<kVar64[3].ci, kVar64[3].cj, kVar64[3].minb, double, kVar64[3].fd>();
        set_smem_attr<kVar64[4].ci, kVar64[4].cj, kVar64[4].minb, double, kVar64[4].fd>();
    } else {
        set_smem_attr<kVar32[0].ci, kVar32[0].cj, kVar32[0].minb, float, kVar32[0].fd>();
        set_smem_attr<kVar32[1].ci, kVar32[1].cj, kVar32[1].minb, float, kVar32[1].fd>();
        set_smem_attr<kVar32[2].ci, kVar32[2].cj, kVar32[2].minb, float, kVar32[2].fd>();
        set_smem_attr<kVar32[3].ci, kVar32[3].cj, kVar32[3].minb, float, kVar32[3].fd>();
        set_smem_attr<kVar32[4].ci, kVar32[4].cj, kVar32[4].minb, float, kVar32[4].fd>();
        // the coarsest FAS level of a mixed session runs the first fp64 variant
        set_smem_attr<kVar64[0].ci, kVar64[0].cj, kVar64[0].minb, double, kVar64[0].fd>();
    }
}

static Variant variant_shape(const Session& S, int v)
{
    if (S.dim == 3) { return S.prec == EGG_B200_PREC_FP64 ? kVar3_64[v] : kVar3_32[v]; }
    return S.prec == EGG_B200_PREC_FP64 ? kVar64[v] : kVar32[v];
}

// Tile list of the interior kernel for variant v over every block's
// structured interior, keeping tiles that hold a moving DOF.  2D: CI x CJ
// cells, (CI-1) x (CJ-1) DOFs per tile (CI x CJ DOFs with fd); 3D: CI x CJ x
// CK DOFs per tile.
static void set_tiles(Session& S, LevelData& L, Variant v)
{
    if (L.tile_ci == v.ci && L.tile_cj == v.cj && L.tile_ck == v.ck && L.tile_fd == v.fd) { return; }
    S.drop_graphs();
    const int shrink = (S.dim == 2 && !v.fd) ? 1 : 0;
    const int di = v.ci - shrink, dj = v.cj - shrink, dk = S.dim == 2 ? 1 : v.ck;
    std::vector<Tile2> tiles2;
    std::vector<Tile3> tiles3;
    for (int b = 0; b < int(L.blocks_h.size()); ++b) {
        const BlockInfo& bi = L.blocks_h[b];
        if (bi.n[0] < 3 || bi.n[1] < 3 || (S.dim == 3 && bi.n[2] < 3)) { continue; }
        const int hk = S.dim == 3 ? bi.n[2] - 2 : 1;
        for (int i0 = 1; i0 <= bi.n[0] - 2; i0 += di) {
            for (int j0 = 1; j0 <= bi.n[1] - 2; j0 += dj) {
                for (int k0 = S.dim == 3 ? 1 : 0; k0 <= (S.dim == 3 ? hk : 0); k0 += dk) {
                    bool any = false;
                    for (int i = i0; i < std::min(i0 + di, bi.n[0] - 1) && !any; ++i) {
                        for (int j = j0; j < std::min(j0 + dj, bi.n[1] - 1) && !any; ++j) {
                            const int kend = S.dim == 3 ? std::min(k0 + dk, bi.n[2] - 1) : 1;
                            for (int k = S.dim == 3 ? k0 : 0; k < kend; ++k) {
                                if (L.active_h[bi.off + (int64_t(i) * bi.n[1] + j) * bi.n[2] + k]) {
                                    any = true;
                                    break;
                                }
                            }
                        }
                    }
                    if (!any) { continue; }
                    if (S.dim == 2) {
                        tiles2.push_back(Tile2 {b, i0, j0, 0});
                    } else {
                        tiles3.push_back(Tile3 {b, i0, j0, k0});
                    }
                }
            }
        }
    }
    if (S.dim == 2) {
        L.tiles_d.upload(tiles2);
        L.ntiles = int64_t(tiles2.size());
    } else {
        L.tiles3_d.upload(tiles3);
        L.ntiles = int64_t(tiles3.size());
    }
    L.tile_ci = v.ci;
    L.tile_cj = v.cj;
    L.tile_ck = v.ck;
    L.tile_fd = v.fd;
}

static Session* create_session(const egg_b200_session_desc& d)
{
    const int D = d.dim;
    if (D != 2 && D != 3) { invalid("egg C++ core: dimension must be 2 or 3, got " + std::to_string(D)); }
    if (d.precision != EGG_B200_PREC_FP64 && d.precision != EGG_B200_PREC_MIXED) {
        invalid("session desc: unknown precision " + std::to_string(d.precision));
    }
    const int64_t M = d.num_nodes;
    if (M < 0) { invalid("session desc: negative num_nodes"); }
    require_ptr(d.X, M, "X");

    auto S = std::make_unique<Session>();
    S->dim = D;
    S->prec = d.precision;
    S->M = M;

    // Host-side validation and remap come first, so malformed input is
    // rejected (ValueError) before any device is touched.

    // ---- blocks ----------------------------------------------------------
    const int nb = d.num_blocks;
    if (nb < 0) { invalid("structured: negative block count"); }
    require_ptr(d.interior_shapes, nb, "interior_shapes");
    S->blocks_h.resize(nb);
    int64_t off = 0;
    for (int b = 0; b < nb; ++b) {
        BlockInfo bi {};
        bi.off = off;
        int64_t cnt = 1;
        for (int k = 0; k < 3; ++k) { bi.n[k] = 1; }
        for (int k = 0; k < D; ++k) {
            const int32_t nk = d.interior_shapes[b * D + k];
            if (nk < 1) { invalid("structured: interior shape entries must be >= 1"); }
            bi.n[k] = nk;
            cnt *= nk;
        }
        S->blocks_h[b] = bi;
        off += cnt;
    }
    if (off > std::numeric_limits<int32_t>::max()) { throw Error(EGG_B200_ENOTSUP, "egg_b200: store exceeds 2^31 nodes"); }
    S->nstore = off;
    require_ptr(d.block_global_dof, off, "block_global_dof");
    S->slot_gid.assign(d.block_global_dof, d.block_global_dof + off);
    for (int64_t i = 0; i < off; ++i) {
        const int32_t g = S->slot_gid[i];
        if (g < 0 || g >= M) { invalid("structured: block_global_dof id " + std::to_string(g) + " out of range"); }
    }

    // Owner (lowest block containing the node) and its slot; singular override.
    std::vector<int32_t> owner_block(M, -1);
    S->g2s.assign(M, -1);
    for (int b = 0; b < nb; ++b) {
        const BlockInfo& bi = S->blocks_h[b];
        const int64_t cnt = int64_t(bi.n[0]) * bi.n[1] * bi.n[2];
        for (int64_t f = 0; f < cnt; ++f) {
            const int32_t g = S->slot_gid[bi.off + f];
            if (owner_block[g] < 0) {
                owner_block[g] = b;
                S->g2s[g] = int32_t(bi.off + f);
            }
        }
    }
    require_ptr(d.sing_block, d.num_sing, "sing_block");
    require_ptr(d.sing_logical, d.num_sing * D, "sing_logical");
    for (int64_t s = 0; s < d.num_sing; ++s) {
        const int32_t b = d.sing_block[s];
        if (b < 0 || b >= nb) { invalid("structured: sing_block out of range"); }
        const BlockInfo& bi = S->blocks_h[b];
        int64_t f = 0;
        for (int k = 0; k < D; ++k) {
            const int32_t l = d.sing_logical[s * D + k];
            if (l < 0 || l >= bi.n[k]) { invalid("structured: sing_logical out of range"); }
            f = f * bi.n[k] + l;
        }
        const int32_t g = S->slot_gid[bi.off + f];
        owner_block[g] = b;
        S->g2s[g] = int32_t(bi.off + f);
    }
    for (int64_t g = 0; g < M; ++g) {
        if (S->g2s[g] >= 0) { continue; }
        S->nb_gid.push_back(g);
        for (int k = 0; k < D; ++k) { S->nb_val.push_back(d.X[g * D + k]); }
    }
    // Halo tables: validated (indices in the padded range); this core reads
    // cross-block neighbours from owner slots and needs no ghost fills.
    for (const auto* p : {d.halo_src_block, d.halo_dst_block}) { require_ptr(p, d.num_halo, "halo block table"); }
    for (const auto* p : {d.halo_src_padded, d.halo_dst_padded}) { require_ptr(p, d.num_halo * D, "halo padded table"); }
    for (int64_t e = 0; e < d.num_halo; ++e) {
        for (int side = 0; side < 2; ++side) {
            const int32_t b = side ? d.halo_dst_block[e] : d.halo_src_block[e];
            const int32_t* pad = side ? d.halo_dst_padded : d.halo_src_padded;
            if (b < 0 || b >= nb) { invalid("structured: halo block index out of range"); }
            for (int k = 0; k < D; ++k) {
                const int32_t v = pad[e * D + k];
                if (v < 0 || v > S->blocks_h[b].n[k] + 1) { invalid("structured: halo padded index out of range"); }
            }
        }
    }
    // Owner -> non-owner copies.
    std::vector<int32_t> sh_src, sh_dst;
    for (int b = 0; b < nb; ++b) {
        const BlockInfo& bi = S->blocks_h[b];
        const int64_t cnt = int64_t(bi.n[0]) * bi.n[1] * bi.n[2];
        for (int64_t f = 0; f < cnt; ++f) {
            const int32_t g = S->slot_gid[bi.off + f];
            if (owner_block[g] == b && S->g2s[g] == int32_t(bi.off + f)) { continue; }
            sh_src.push_back(S->g2s[g]);
            sh_dst.push_back(int32_t(bi.off + f));
        }
    }
    S->nshare = int64_t(sh_src.size());

    // ---- group -----------------------------------------------------------
    const int64_t ndof = d.ndof;
    const int64_t ts = d.total_samples;
    if (ndof < 0 || ts < 0) { invalid("validate_context: negative sizes"); }
    require_ptr(d.dof_idx, ndof, "dof_idx");
    require_ptr(d.P_of, ndof, "P_of");
    require_ptr(d.gc, ts, "gc");
    require_ptr(d.role, ts, "role");
    for (int k = 0; k < D; ++k) {
        require_ptr(d.gn[k], ts, "gn" + std::to_string(k));
        require_ptr(d.s[k], ts, "s" + std::to_string(k));
    }
    const bool w_uniform = d.W_inv_len == D * D;
    if (!w_uniform) { check_len(d.W_inv_len, ts * D * D, "group[0] W_inv"); }
    require_ptr(d.W_inv, d.W_inv_len, "W_inv");
    if (d.weight_len != 0 && d.weight_len != 1) { check_len(d.weight_len, ts, "group[0] weight"); }
    require_ptr(d.weight, d.weight_len, "weight");
    int64_t sumP = 0;
    for (int64_t i = 0; i < ndof; ++i) {
        if (d.P_of[i] < 0) { invalid("validate_context: group[0] negative P_of"); }
        sumP += d.P_of[i];
    }
    if (sumP != ts) {
        invalid("validate_context: group[0] sum(P_of) " + std::to_string(sumP) + " != total_samples " + std::to_string(ts));
    }
    for (int64_t p = 0; p < ts; ++p) {
        const int32_t r = d.role[p];
        if (r < -1 || r > D) {
            invalid("validate_context: group[0] role " + std::to_string(r) + " out of range [-1, " + std::to_string(D) + "]");
        }
        auto chk = [&](int32_t v, const char* nm) {
            if (v < 0 || v >= M) {
                invalid(std::string("validate_context: group[0] ") + nm + " index " + std::to_string(v) +
                        " out of range [0, " + std::to_string(M) + ")");
            }
        };
        chk(d.gc[p], "gc");
        for (int k = 0; k < D; ++k) { chk(d.gn[k][p], ("gn" + std::to_string(k)).c_str()); }
    }

    // ---- soft terms --------------------------------------------------------
    // Per-DOF directional samples (2D, 3D) and curvature windows (2D; the
    // reference reads them in 2D only, src/sweep.hpp:1464).  A structured-
    // interior DOF that carries a term leaves the tile path and relaxes as a
    // stored DOF with the synthesized patch's identity target and unit weight
    // (src/structured_patch.hpp:183-185), so its terms join its Newton system.
    if (d.dir_k < 0 || d.curv_k < 0) { invalid("validate_context: negative dir_k / curv_k"); }
    const int64_t dk = d.dir_k, ck = D == 2 ? d.curv_k : 0;
    if (dk) {
        require_ptr(d.dir_nodes, ndof * dk * 4, "dir_nodes");
        require_ptr(d.dir_slot, ndof * dk, "dir_slot");
        require_ptr(d.dir_kind, ndof * dk, "dir_kind");
        require_ptr(d.dir_ref, ndof * dk * D, "dir_ref");
        require_ptr(d.dir_weight, ndof * dk, "dir_weight");
        if (!std::isfinite(d.dir_eps)) { invalid("validate_context: dir_eps is not finite"); }
    }
    if (ck) {
        require_ptr(d.curv_nodes, ndof * ck * 4, "curv_nodes");
        require_ptr(d.curv_slot, ndof * ck, "curv_slot");
        require_ptr(d.curv_weight, ndof * ck, "curv_weight");
    }
    auto dir_arity = [](int32_t kind) { return (kind >= 0 && kind <= kSoftStem) ? soft_arity(kind) : 0; };
    auto soft_node = [&](int32_t g, const char* what) {
        const int32_t sl = (g >= 0 && g < M) ? S->g2s[g] : -1;
        if (sl < 0) {
            invalid(std::string("structured: a ") + what + " node references a global node absent from every block's interior map");
        }
        return sl;
    };
    std::vector<uint8_t> has_soft(size_t(ndof), 0);
    for (int64_t i = 0; i < ndof; ++i) {
        for (int64_t j = 0; j < ck; ++j) {
            const int32_t sl = d.curv_slot[i * ck + j];
            if (sl < -1 || sl > 3) { invalid("validate_context: curv_slot out of range [-1, 3]"); }
            if (sl >= 0) { has_soft[i] = 1; }
        }
        for (int64_t j = 0; j < dk; ++j) {
            const int32_t sl = d.dir_slot[i * dk + j];
            const int ar = dir_arity(d.dir_kind[i * dk + j]);
            if (sl < -1 || (sl >= 0 && ar > 0 && sl >= ar)) { invalid("validate_context: dir_slot out of range"); }
            if (sl >= 0 && ar > 0) { has_soft[i] = 1; }
        }
    }
    bool any_demote = false;
    for (int64_t i = 0; i < ndof; ++i) {
        if (has_soft[i] && d.interior_block && d.interior_block[i] >= 0) { any_demote = true; }
    }
    auto is_identity = [&](const double* w) {
        for (int a = 0; a < D; ++a) {
            for (int b = 0; b < D; ++b) {
                if (w[a * D + b] != (a == b ? 1.0 : 0.0)) { return false; }
            }
        }
        return true;
    };
    const bool per_row_W = !w_uniform || (any_demote && !is_identity(d.W_inv));
    const bool per_row_wt = d.weight_len > 1 || (any_demote && d.weight_len == 1 && d.weight[0] != 1.0);
    std::vector<SoftTerm> soft_terms;
    std::vector<int32_t> soft_off {0};
    auto soft_terms_of = [&](int64_t i) {
        for (int64_t j = 0; j < ck; ++j) {
            const int32_t sl = d.curv_slot[i * ck + j];
            if (sl < 0) { continue; }
            SoftTerm t {};
            for (int m = 0; m < 4; ++m) { t.node[m] = soft_node(d.curv_nodes[(i * ck + j) * 4 + m], "curvature-window"); }
            t.slot = sl;
            t.kind = kSoftCurv;
            t.w = d.curv_weight[i * ck + j];
            soft_terms.push_back(t);
        }
        for (int64_t j = 0; j < dk; ++j) {
            const int32_t sl = d.dir_slot[i * dk + j], kind = d.dir_kind[i * dk + j];
            const int ar = dir_arity(kind);
            if (sl < 0 || ar == 0) { continue; }
            SoftTerm t {};
            for (int m = 0; m < 4; ++m) {
                t.node[m] = m < ar ? soft_node(d.dir_nodes[(i * dk + j) * 4 + m], "directional-sample") : -1;
            }
            t.slot = sl;
            t.kind = kind;
            for (int k = 0; k < D; ++k) { t.ref[k] = d.dir_ref[(i * dk + j) * D + k]; }
            t.w = d.dir_weight[i * dk + j];
            soft_terms.push_back(t);
        }
        if (soft_terms.size() > size_t(INT32_MAX)) { invalid("validate_context: too many soft terms"); }
        soft_off.push_back(int32_t(soft_terms.size()));
    };

    std::vector<uint8_t> active(off, 0), interior(off, 0);
    std::vector<int32_t> st_slot;
    std::vector<int64_t> st_off {0};
    std::vector<int32_t> st_gc, st_gn0, st_gn1, st_gn2, st_role;
    std::vector<int8_t> st_s0, st_s1, st_s2;
    std::vector<double> st_W, st_wt, st_epar;
    std::vector<int8_t> st_etag;
    std::vector<uint8_t> seen_slot(off, 0);
    int64_t poff = 0;
    for (int64_t i = 0; i < ndof; ++i) {
        const int32_t gid = d.dof_idx[i];
        const int64_t P = d.P_of[i];
        const int64_t p0 = poff;
        poff += P;
        if (gid < 0 || gid >= M) {
            invalid("validate_context: group[0] dof_idx index " + std::to_string(gid) + " out of range [0, " +
                    std::to_string(M) + ")");
        }
        const int32_t etag = d.entity_tag ? d.entity_tag[i] : 0;
        if (etag != 0) {
            if (!entity_supported(D, etag)) {
                throw Error(EGG_B200_ENOTSUP, "egg_b200: constrained entity tag " + std::to_string(etag) +
                                                " is not supported in " + std::to_string(D) +
                                                "D (this core relaxes the 2D LineSeg, Circle, Ellipse, CircleArc, EllipseArc, QuadBezier, CubicBezier, BSpline, "
                                                "LineRail and the 3D Plane, Sphere, Cylinder, Line3, LineRail3, BSplineSurface)");
            }
            if (!d.entity_params) { invalid("validate_context: constrained DOF without entity_params"); }
            for (int f = 0; f < EGG_B200_ENTITY_FIELDS; ++f) {
                if (!std::isfinite(d.entity_params[i * EGG_B200_ENTITY_FIELDS + f])) {
                    invalid("validate_context: entity record of DOF " + std::to_string(i) + " is not finite");
                }
            }
            if (d.interior_block && d.interior_block[i] >= 0) {
                throw Error(EGG_B200_ENOTSUP, "egg_b200: a constrained DOF on the structured-interior path");
            }
            if (etag == EGG_B200_TAG_COMPOSITE) {
                const double* r = d.entity_params + i * EGG_B200_ENTITY_FIELDS;
                const int64_t ns = int64_t(r[0]), ro = int64_t(r[1]), at = int64_t(r[6]);
                if (double(ns) != r[0] || ns < 1 || double(ro) != r[1] || ro < 0 || double(at) != r[6] || at < 0 ||
                    !d.entity_arena || at + ro + ns * kCompositeRec > d.entity_arena_len) {
                    invalid("validate_context: composite segment records outside entity_arena");
                }
                for (int64_t k = 0; k < ns; ++k) {
                    const double* sr = d.entity_arena + at + ro + k * kCompositeRec;
                    const int st = int(sr[0]);
                    if (st != 0 && st != EGG_B200_TAG_COMPOSITE && !composite_segment_ok(st)) {
                        throw Error(EGG_B200_ENOTSUP, "egg_b200: composite segment tag " + std::to_string(st) +
                                                        " is not supported (2D curves are)");
                    }
                    if (st == EGG_B200_TAG_BSPLINE) {  // blob [degree, n_ctrl, knots, ctrl, t0, t1, w, has_w]
                        const double* b = sr + 1;
                        const int64_t deg = int64_t(b[0]), nc = int64_t(b[1]);
                        auto in_slice = [&](double o, int64_t len) {
                            return o >= 0.0 && double(int64_t(o)) == o && at + int64_t(o) + len <= d.entity_arena_len;
                        };
                        if (double(deg) != b[0] || deg < 1 || deg > kBSplineMaxDegree || double(nc) != b[1] ||
                            nc < deg + 1 || !in_slice(b[2], nc + deg + 1) || !in_slice(b[3], 2 * nc) ||
                            (b[7] != 0.0 && !in_slice(b[6], nc))) {
                            invalid("validate_context: a composite B-spline segment's data lies outside entity_arena");
                        }
                    }
                }
            }
            if (etag == EGG_B200_TAG_BSPLINESURF) {
                const double* r = d.entity_params + i * EGG_B200_ENTITY_FIELDS;
                if (!bsurf_record_ok(r, d.entity_arena, d.entity_arena_len)) {
                    invalid("validate_context: B-spline surface degrees (1.." + std::to_string(kBSplineMaxDegree) +
                            "), control net, knots, weights or trim polygon outside entity_arena");
                }
            }
            if (etag == EGG_B200_TAG_BSPLINE) {
                const double* r = d.entity_params + i * EGG_B200_ENTITY_FIELDS;
                const int64_t deg = int64_t(r[0]), nc = int64_t(r[1]);
                if (double(deg) != r[0] || deg < 1 || deg > kBSplineMaxDegree || double(nc) != r[1] || nc < deg + 1) {
                    invalid("validate_context: B-spline degree must be 1.." + std::to_string(kBSplineMaxDegree) +
                            " with n_ctrl > degree");
                }
                auto within = [&](double at, int64_t len) {
                    return at >= 0.0 && double(int64_t(at)) == at && int64_t(at) + len <= d.entity_arena_len;
                };
                if (!d.entity_arena || !within(r[6], nc + deg + 1) || !within(r[7], 2 * nc) ||
                    (r[5] != 0.0 && !within(r[8], nc))) {
                    invalid("validate_context: B-spline knots / control points / weights outside entity_arena");
                }
            }
        }
        const int32_t slot = S->g2s[gid];
        if (slot < 0) {
            invalid("structured: dof_idx references global node " + std::to_string(gid) +
                    " absent from every block's interior map");
        }
        if (seen_slot[slot]) { invalid("validate_context: DOF " + std::to_string(gid) + " listed twice"); }
        seen_slot[slot] = 1;
        const int32_t ib = d.interior_block ? d.interior_block[i] : -1;
        if (ib >= 0) {
            if (ib >= nb) { invalid("structured: interior_block out of range"); }
            const BlockInfo& bi = S->blocks_h[ib];
            int64_t f = 0;
            for (int k = 0; k < D; ++k) {
                const int32_t l = d.interior_logical[i * D + k];
                if (l < 1 || l > bi.n[k] - 2) { invalid("structured: interior_logical not strictly interior"); }
                f = f * bi.n[k] + l;
            }
            if (S->slot_gid[bi.off + f] != gid) {
                invalid("structured: interior_block/interior_logical does not name the DOF's node");
            }
            interior[bi.off + f] = 1;
            if (!has_soft[i]) {
                active[bi.off + f] = 1;
                S->n_interior++;
                continue;
            }
        }
        const bool synth_target = ib >= 0;  // a structured-interior DOF carrying soft terms
        st_slot.push_back(slot);
        st_etag.push_back(int8_t(etag));
        for (int f = 0; f < EGG_B200_ENTITY_FIELDS; ++f) {
            st_epar.push_back(etag != 0 ? d.entity_params[i * EGG_B200_ENTITY_FIELDS + f] : 0.0);
        }
        if (etag != 0) { S->n_constrained++; }
        if ((D == 2 && (is_tcurve(etag) || etag == EGG_B200_TAG_BSPLINE)) || (D == 3 && is_param3(etag))) {
            S->n_arc++;
        }
        if (etag == EGG_B200_TAG_BSPLINE || etag == EGG_B200_TAG_BSPLINESURF) { S->n_bspline++; }
        if (etag == EGG_B200_TAG_COMPOSITE) { S->n_composite++; }
        if (synth_target) {
            // The synthesized interior patch (src/structured_patch.hpp:89-130):
            // every sample of the 2^D cells around the node, identity target,
            // unit weight, node slots in the DOF's block.  Wire rows of such a
            // DOF (none on the reference's wire) are not read.
            const BlockInfo& bi = S->blocks_h[ib];
            const int nz = D == 3 ? bi.n[2] : 1;
            int32_t l[3] = {0, 0, 0};
            for (int k = 0; k < D; ++k) { l[k] = d.interior_logical[i * D + k]; }
            const int nco = 1 << D;
            for (int cell = 0; cell < nco; ++cell) {
                int base[3] = {0, 0, 0};
                for (int k = 0; k < D; ++k) { base[k] = l[k] - 1 + ((cell >> (D - 1 - k)) & 1); }
                auto corner = [&](int a) {
                    int q[3] = {0, 0, 0};
                    for (int k = 0; k < D; ++k) { q[k] = base[k] + ((a >> (D - 1 - k)) & 1); }
                    return int32_t(bi.off + (int64_t(q[0]) * bi.n[1] + q[1]) * nz + q[2]);
                };
                for (int b = 0; b < nco; ++b) {
                    const int32_t c = corner(b);
                    int32_t nbr[3] = {0, 0, 0};
                    int8_t sg[3] = {1, 1, 1};
                    int32_t role = c == slot ? 0 : -1;
                    for (int k = 0; k < D; ++k) {
                        const int bit = 1 << (D - 1 - k);
                        nbr[k] = corner(b ^ bit);
                        sg[k] = (b & bit) ? int8_t(-1) : int8_t(1);
                        if (nbr[k] == slot) { role = k + 1; }
                    }
                    st_gc.push_back(c);
                    st_gn0.push_back(nbr[0]);
                    st_gn1.push_back(nbr[1]);
                    st_s0.push_back(sg[0]);
                    st_s1.push_back(sg[1]);
                    if (D == 3) {
                        st_gn2.push_back(nbr[2]);
                        st_s2.push_back(sg[2]);
                    }
                    st_role.push_back(role);
                    if (per_row_W) {
                        for (int a = 0; a < D; ++a) {
                            for (int e = 0; e < D; ++e) { st_W.push_back(a == e ? 1.0 : 0.0); }
                        }
                    }
                    if (per_row_wt) { st_wt.push_back(1.0); }
                }
            }
        }
        for (int64_t p = p0; p < (synth_target ? p0 : p0 + P); ++p) {
            auto remap = [&](int32_t g) {
                const int32_t s = S->g2s[g];
                if (s < 0) {
                    invalid("structured: a patch sample references global node " + std::to_string(g) +
                            " absent from every block's interior map");
                }
                return s;
            };
            st_gc.push_back(remap(d.gc[p]));
            st_gn0.push_back(remap(d.gn[0][p]));
            st_gn1.push_back(remap(d.gn[1][p]));
            st_s0.push_back(d.s[0][p] < 0 ? int8_t(-1) : int8_t(1));
            st_s1.push_back(d.s[1][p] < 0 ? int8_t(-1) : int8_t(1));
            if (D == 3) {
                st_gn2.push_back(remap(d.gn[2][p]));
                st_s2.push_back(d.s[2][p] < 0 ? int8_t(-1) : int8_t(1));
            }
            st_role.push_back(d.role[p]);
            if (per_row_W) {
                const double* w = w_uniform ? d.W_inv : d.W_inv + p * D * D;
                for (int a = 0; a < D; ++a) {
                    for (int b = 0; b < D; ++b) { st_W.push_back(synth_target ? (a == b ? 1.0 : 0.0) : w[a * D + b]); }
                }
            }
            if (per_row_wt) { st_wt.push_back(synth_target ? 1.0 : d.weight[d.weight_len > 1 ? p : 0]); }
        }
        st_off.push_back(int64_t(st_gc.size()));
        soft_terms_of(i);
    }
    S->n_stored = int64_t(st_slot.size());
    S->free_h.assign(off, 0);
    // FAS masks: Free DOFs only.  Constrained DOFs relax in the fine smoothing
    // but are frozen on the coarse levels and take no coarse correction, so
    // the correction never pushes them off their geometry (src/fas.hpp:120-140
    // masks_from_context, :380-384).
    for (size_t k = 0; k < st_slot.size(); ++k) {
        if (st_etag[k] == 0) { S->free_h[size_t(st_slot[k])] = 1; }
    }
    for (int64_t i = 0; i < off; ++i) {
        if (active[i]) { S->free_h[i] = 1; }
    }
    for (int64_t e = 0; e < d.num_halo; ++e) {
        std::array<int32_t, 3> sp {0, 0, 0}, dp {0, 0, 0};
        for (int k = 0; k < D; ++k) {
            sp[k] = d.halo_src_padded[e * D + k];
            dp[k] = d.halo_dst_padded[e * D + k];
        }
        S->halo.sb.push_back(d.halo_src_block[e]);
        S->halo.db.push_back(d.halo_dst_block[e]);
        S->halo.sp.push_back(sp);
        S->halo.dp.push_back(dp);
    }
    if (!per_row_W || st_W.empty()) {
        st_W.assign(d.W_inv, d.W_inv + (w_uniform ? D * D : 0));
        if (st_W.empty()) { st_W = identity_row(D); }
        S->st_wstride = 0;
    } else if (rows_uniform(st_W.data(), int64_t(st_W.size()) / (D * D), D * D)) {
        st_W.resize(D * D);
        S->st_wstride = 0;
    } else {
        S->st_wstride = D * D;
    }
    if (st_wt.empty()) {
        st_wt = {d.weight_len == 1 ? d.weight[0] : 1.0};
        S->st_wtstride = 0;
    } else {
        S->st_wtstride = 1;
    }

    // ---- energy stencil -------------------------------------------------
    int64_t ncell = 0;
    std::vector<int64_t> cell_off(nb + 1, 0);
    for (int b = 0; b < nb; ++b) {
        const BlockInfo& bi = S->blocks_h[b];
        int64_t c = 1;
        for (int k = 0; k < D; ++k) { c *= std::max(0, bi.n[k] - 1); }
        cell_off[b] = ncell;
        ncell += c;
    }
    cell_off[nb] = ncell;
    const int nc = 1 << D;
    const int64_t ns = d.es_num_samples;
    if (ns < 0) { invalid("validate_context: energy_stencil negative num_samples"); }
    const bool es_w_uniform = d.es_W_inv_len == D * D;
    if (!es_w_uniform) { check_len(d.es_W_inv_len, ns * D * D, "energy_stencil W_inv"); }
    require_ptr(d.es_W_inv, d.es_W_inv_len, "energy_stencil W_inv");
    if (d.es_weight_len > 1) { check_len(d.es_weight_len, ns, "energy_stencil weight"); }
    bool structured = false;
    if (d.es_structured) {
        if (ns != ncell * nc) { invalid("energy_stencil: structured stencil size does not match the blocks"); }
        structured = true;
    } else {
        require_ptr(d.es_gc, ns, "energy_stencil gc");
        for (int k = 0; k < D; ++k) {
            require_ptr(d.es_gn[k], ns, "energy_stencil gn");
            require_ptr(d.es_s[k], ns, "energy_stencil s");
        }
        // Index checks and the canonical-form test run on host threads over
        // slices of the samples (cells); a failure reports the first bad
        // sample in sample order, as a serial scan would.
        const int T = copy_threads(size_t(ns) * 64);
        std::vector<int64_t> bad_at(T, -1);
        std::vector<int32_t> bad_val(T, 0);
        run_slices(T, [&](int t) {
            const int64_t i0 = int64_t(slice_begin(size_t(ns), t, T)), i1 = int64_t(slice_begin(size_t(ns), t + 1, T));
            for (int64_t i = i0; i < i1; ++i) {
                for (int k = -1; k < D; ++k) {
                    const int32_t v = k < 0 ? d.es_gc[i] : d.es_gn[k][i];
                    if (v < 0 || v >= M || S->g2s[v] < 0) {
                        bad_at[t] = i;
                        bad_val[t] = v;
                        return;
                    }
                }
            }
        });
        for (int t = 0; t < T; ++t) {
            if (bad_at[t] < 0) { continue; }
            const int32_t v = bad_val[t];
            if (v < 0 || v >= M) {
                invalid("validate_context: energy_stencil index " + std::to_string(v) + " out of range [0, " +
                        std::to_string(M) + ")");
            }
            invalid("structured: an energy-stencil index references a global node absent from every "
                    "block's interior map");
        }
        // Canonical cell stencil of the blocks?  Sample 2^D * cell + b:
        // corner at cell base + bits(b) (axis 0 most significant), axis-k
        // neighbour at corner ^ bit_k, sign -1 where bit k of b is set.
        if (ns == ncell * nc) {
            std::vector<uint8_t> ok(T, 1);
            run_slices(T, [&](int t) {
                const int64_t c0 = int64_t(slice_begin(size_t(ncell), t, T));
                const int64_t c1 = int64_t(slice_begin(size_t(ncell), t + 1, T));
                int b = 0;
                for (int64_t cell = c0; cell < c1; ++cell) {
                    while (cell >= cell_off[b + 1]) { ++b; }
                    const BlockInfo& bi = S->blocks_h[b];
                    const int64_t c1b = std::max(0, bi.n[1] - 1), c2b = D == 3 ? std::max(0, bi.n[2] - 1) : 1;
                    const int64_t lc = cell - cell_off[b];
                    const int64_t i = lc / (c1b * c2b), j = (lc / c2b) % c1b, k = lc % c2b;
                    int32_t cg[8];
                    for (int a = 0; a < nc; ++a) {
                        int64_t u, v, w;
                        if (D == 2) {
                            u = i + (a >> 1);
                            v = j + (a & 1);
                            w = 0;
                        } else {
                            u = i + (a >> 2);
                            v = j + ((a >> 1) & 1);
                            w = k + (a & 1);
                        }
                        cg[a] = S->slot_gid[bi.off + (u * bi.n[1] + v) * bi.n[2] + w];
                    }
                    for (int bb = 0; bb < nc; ++bb) {
                        const int64_t sid = cell * nc + bb;
                        if (d.es_gc[sid] != cg[bb]) {
                            ok[t] = 0;
                            return;
                        }
                        for (int ax = 0; ax < D; ++ax) {
                            const int bit = 1 << (D - 1 - ax);
                            if (d.es_gn[ax][sid] != cg[bb ^ bit] || d.es_s[ax][sid] != ((bb & bit) ? -1.0 : 1.0)) {
                                ok[t] = 0;
                                return;
                            }
                        }
                    }
                }
            });
            structured = std::all_of(ok.begin(), ok.end(), [](uint8_t x) { return x != 0; });
        }
    }
    S->es_struct = structured;
    S->es_ns = ns;
    S->es_ncell = ncell;
    std::vector<double> es_W_h, es_wt_h;
    std::vector<int32_t> es_a, es_b0, es_b1, es_b2;
    std::vector<int8_t> es_s0h, es_s1h, es_s2h;
    if (es_w_uniform || ns == 0) {
        es_W_h.assign(d.es_W_inv, d.es_W_inv + (es_w_uniform ? D * D : 0));
        if (es_W_h.empty()) { es_W_h = identity_row(D); }
        S->es_wstride = 0;
    } else if (rows_uniform(d.es_W_inv, ns, D * D)) {
        es_W_h.assign(d.es_W_inv, d.es_W_inv + D * D);
        S->es_wstride = 0;
    } else {
        es_W_h.assign(d.es_W_inv, d.es_W_inv + ns * D * D);
        S->es_wstride = D * D;
    }
    if (d.es_weight_len > 1) {
        es_wt_h.assign(d.es_weight, d.es_weight + ns);
        S->es_wtstride = 1;
    } else {
        es_wt_h = {d.es_weight_len == 1 ? d.es_weight[0] : 1.0};
        S->es_wtstride = 0;
    }
    if (!structured) {
        es_a.resize(ns);
        es_b0.resize(ns);
        es_b1.resize(ns);
        es_s0h.resize(ns);
        es_s1h.resize(ns);
        if (D == 3) {
            es_b2.resize(ns);
            es_s2h.resize(ns);
        }
        const int T = copy_threads(size_t(ns) * 64);
        run_slices(T, [&](int t) {
            const int64_t i0 = int64_t(slice_begin(size_t(ns), t, T)), i1 = int64_t(slice_begin(size_t(ns), t + 1, T));
            for (int64_t i = i0; i < i1; ++i) {
                es_a[i] = S->g2s[d.es_gc[i]];
                es_b0[i] = S->g2s[d.es_gn[0][i]];
                es_b1[i] = S->g2s[d.es_gn[1][i]];
                es_s0h[i] = d.es_s[0][i] < 0 ? -1 : 1;
                es_s1h[i] = d.es_s[1][i] < 0 ? -1 : 1;
                if (D == 3) {
                    es_b2[i] = S->g2s[d.es_gn[2][i]];
                    es_s2h[i] = d.es_s[2][i] < 0 ? -1 : 1;
                }
            }
        });
    }

    S->active_h = std::move(active);
    S->interior_h = std::move(interior);

    // ---- device --------------------------------------------------------------
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        throw Error(EGG_B200_ENODEV, "select_queue: no CUDA device available (egg_b200 runs on the GPU only)");
    }
    if (d.device >= 0) {
        if (d.device >= ndev) { invalid("session desc: device ordinal out of range"); }
        EGG_CK(cudaSetDevice(d.device));
    }
    EGG_CK(cudaGetDevice(&S->device));
    EGG_CK(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    EGG_CK(cudaStreamCreateWithFlags(&S->side, cudaStreamNonBlocking));
    EGG_CK(cudaEventCreateWithFlags(&S->fork_ev, cudaEventDisableTiming));
    EGG_CK(cudaEventCreateWithFlags(&S->join_ev, cudaEventDisableTiming));
    configure_kernels(S->prec, S->dim);
    EGG_CK(cudaDeviceGetAttribute(&S->num_sms, cudaDevAttrMultiProcessorCount, S->device));
    S->kerr.upload(std::vector<int> {0});

    // ---- upload -----------------------------------------------------------
    S->es_W.upload(es_W_h);
    S->es_wt.upload(es_wt_h);
    // Whole-sample directional table (src/bindings.cpp:471-480, remapped to
    // owner slots as src/bindings.cpp:1053-1066 does); reserved kinds drop.
    if (d.es_dir_num < 0) { invalid("validate_context: energy_stencil negative dir_num"); }
    if (d.es_dir_num > 0) {
        const int64_t nd = d.es_dir_num;
        require_ptr(d.es_dir_nodes, nd * 4, "energy_stencil dir_nodes");
        require_ptr(d.es_dir_kind, nd, "energy_stencil dir_kind");
        require_ptr(d.es_dir_ref, nd * D, "energy_stencil dir_ref");
        require_ptr(d.es_dir_weight, nd, "energy_stencil dir_weight");
        if (!std::isfinite(d.es_dir_eps)) { invalid("validate_context: energy_stencil dir_eps is not finite"); }
        std::vector<SoftTerm> es_dir;
        for (int64_t q = 0; q < nd; ++q) {
            const int32_t kind = d.es_dir_kind[q];
            const int ar = dir_arity(kind);
            if (ar == 0) { continue; }
            SoftTerm t {};
            for (int m = 0; m < 4; ++m) { t.node[m] = m < ar ? soft_node(d.es_dir_nodes[q * 4 + m], "directional-sample") : -1; }
            t.slot = -1;
            t.kind = kind;
            for (int k = 0; k < D; ++k) { t.ref[k] = d.es_dir_ref[q * D + k]; }
            t.w = d.es_dir_weight[q];
            es_dir.push_back(t);
        }
        S->es_dir_n = int64_t(es_dir.size());
        S->es_dir.upload(es_dir);
        S->es_dir_eps = d.es_dir_eps;
    }
    if (structured) {
        S->es_cell_off.upload(cell_off);
    } else {
        S->es_gc.upload(es_a);
        S->es_gn0.upload(es_b0);
        S->es_gn1.upload(es_b1);
        S->es_s0.upload(es_s0h);
        S->es_s1.upload(es_s1h);
        S->es_gn2.upload(es_b2);
        S->es_s2.upload(es_s2h);
    }
    S->blocks_d.upload(S->blocks_h);
    S->active_d.upload(S->active_h);
    S->free_d.upload(S->free_h);
    S->variant = 0;
    set_tiles(*S, *S, variant_shape(*S, 0));
    S->st_slot.upload(st_slot);
    S->st_off.upload(st_off);
    if (S->n_constrained) {
        S->st_etag.upload(st_etag);
        S->st_epar.upload(st_epar);
    }
    if (S->n_bspline || S->n_composite) {
        S->arena.upload(std::vector<double>(d.entity_arena, d.entity_arena + d.entity_arena_len));
    }
    if (S->n_bspline) {  // D - 1 foot parameters per stored DOF
        S->seeds.alloc(size_t(S->n_stored) * size_t(D - 1));
        EGG_CK(cudaMemset(S->seeds.p, 0xFF, S->seeds.n * sizeof(double)));  // all-ones: NaN
    }
    S->st_gc.upload(st_gc);
    S->st_gn0.upload(st_gn0);
    S->st_gn1.upload(st_gn1);
    S->st_role.upload(st_role);
    S->st_s0.upload(st_s0);
    S->st_s1.upload(st_s1);
    S->st_gn2.upload(st_gn2);
    S->st_s2.upload(st_s2);
    S->st_W.upload(st_W);
    S->st_wt.upload(st_wt);
    S->n_soft = int64_t(soft_terms.size());
    if (S->n_soft) {
        S->soft_off.upload(soft_off);
        S->soft_terms.upload(soft_terms);
        S->soft_eps = d.dir_eps;
    }
    S->sh_src.upload(sh_src);
    S->sh_dst.upload(sh_dst);
    // The packed store is filled on the device: X goes up in global node
    // order and every slot gathers its node, the X remap of the reference's
    // apply_structured_remap (src/bindings.cpp:757-1101) as one kernel.  The
    // global-order buffer and the slot and owner tables stay for later
    // transfers.
    // (The copies go on the session stream, which orders them before the
    // gather; a pageable cudaMemcpy may return before its DMA lands.)
    S->slot_gid_d.alloc(S->slot_gid.size());
    if (off) {
        EGG_CK(cudaMemcpyAsync(S->slot_gid_d.p, S->slot_gid.data(), size_t(off) * sizeof(int32_t),
                               cudaMemcpyHostToDevice, S->stream));
    }
    S->g2s_d.alloc(S->g2s.size());
    if (M) {
        EGG_CK(cudaMemcpyAsync(S->g2s_d.p, S->g2s.data(), size_t(M) * sizeof(int32_t), cudaMemcpyHostToDevice,
                               S->stream));
    }
    S->Xg.alloc(size_t(M) * D);
    if (M) {
        EGG_CK(cudaMemcpyAsync(S->Xg.p, d.X, size_t(M) * D * sizeof(double), cudaMemcpyHostToDevice, S->stream));
    }
    S->Xbuf[0].alloc(size_t(off) * D);
    S->Xbuf[1].alloc(size_t(off) * D);
    if (off) {
        if (D == 2) {
            gather_global_kernel<2><<<remap_grid(off), 256, 0, S->stream>>>(S->Xg.p, S->slot_gid_d.p, off, S->Xbuf[0].p);
        } else {
            gather_global_kernel<3><<<remap_grid(off), 256, 0, S->stream>>>(S->Xg.p, S->slot_gid_d.p, off, S->Xbuf[0].p);
        }
        EGG_CK(cudaGetLastError());
    }
    S->cur = 0;
    S->red_grid = 148 * 4;
    S->part.alloc(3 * size_t(S->red_grid));
    S->red_out.alloc(2);
    EGG_CK(cudaDeviceSynchronize());
    return S.release();
}

// ---------------------------------------------------------------------------
// Sweep driver
// ---------------------------------------------------------------------------
template <int CI, int CJ, int MINB, int KIND, class C, int FD>
static void launch_tile(Session& S, LevelData& L, const double* xin, double* xout, const double* tau, double delta,
                        double omega, double* gout)
{
    const size_t smem = tile_smem2<CI, CJ, FD, KIND, C>();
    const auto* xi = reinterpret_cast<const double2*>(xin);
    auto* xo = reinterpret_cast<double2*>(xout);
    const auto* tv = reinterpret_cast<const double2*>(tau);
    S.timed(kKInterior, [&] {
        if constexpr (FD == 3) {
            // persistent: as many CTAs as fit on the device at once
            static const int per_sm = [] {
                int nb = 0;
                EGG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                  &nb, interior_x2p_kernel<CI, CJ, MINB, KIND>, TileSharedX2<CI, CJ, 2>::NT,
                  sizeof(TileSharedX2<CI, CJ, 2>)));
                return std::max(nb, 1);
            }();
            const int grid = int(std::min<int64_t>(L.ntiles, int64_t(per_sm) * S.num_sms));
            interior_x2p_kernel<CI, CJ, MINB, KIND><<<unsigned(grid), TileSharedX2<CI, CJ, 2>::NT, smem, S.stream>>>(
              xi, xo, L.tiles_d.p, int(L.ntiles), L.blocks_d.p, L.active_d.p, tv, delta, omega,
              reinterpret_cast<double2*>(gout), S.kerr.p);
            S.kerr_armed = true;
        } else if constexpr (FD == 2) {
            interior_x2_kernel<CI, CJ, MINB, KIND><<<unsigned(L.ntiles), TileSharedX2<CI, CJ>::NT, smem, S.stream>>>(
              xi, xo, L.tiles_d.p, L.blocks_d.p, L.active_d.p, tv, delta, omega, reinterpret_cast<double2*>(gout));
        } else {
            interior_tile_kernel<CI, CJ, MINB, KIND, C, FD><<<unsigned(L.ntiles), CI * CJ, smem, S.stream>>>(
              xi, xo, L.tiles_d.p, L.blocks_d.p, L.active_d.p, tv, delta, omega, reinterpret_cast<double2*>(gout));
        }
    });
}

template <int TI, int TJ, int TK, int MINB, int KIND, class C>
static void launch_tile3(Session& S, LevelData& L, const double* xin, double* xout, const double* tau, double delta,
                         double omega, double* gout)
{
    S.timed(kKInterior, [&] {
        interior3_kernel<TI, TJ, TK, MINB, KIND, C><<<unsigned(L.ntiles), TI * TJ * TK, 0, S.stream>>>(
          xin, xout, L.tiles3_d.p, L.blocks_d.p, L.active_d.p, tau, delta, omega, gout);
    });
}

template <int KIND>
static void launch_interior(Session& S, LevelData& L, const double* xin, double* xout, const double* tau, double delta,
                            double omega, double* gout = nullptr)
{
    if (L.ntiles == 0) { return; }
    if (L.fp64_tiles && S.prec != EGG_B200_PREC_FP64) {
        if (S.dim == 3) {
            launch_tile3<kVar3_64[0].ci, kVar3_64[0].cj, kVar3_64[0].ck, kVar3_64[0].minb, KIND, double>(
              S, L, xin, xout, tau, delta, omega, gout);
        } else {
            launch_tile<kVar64[0].ci, kVar64[0].cj, kVar64[0].minb, KIND, double, kVar64[0].fd>(S, L, xin, xout, tau,
                                                                                               delta, omega, gout);
        }
        return;
    }
    const int var = L.variant >= 0 ? L.variant : S.variant;
#define EGG_V3(T, C, i) \
    launch_tile3<T[i].ci, T[i].cj, T[i].ck, T[i].minb, KIND, C>(S, L, xin, xout, tau, delta, omega, gout)
    if (S.dim == 3) {
        if (S.prec == EGG_B200_PREC_FP64) {
            switch (var) {
            case 0: EGG_V3(kVar3_64, double, 0); break;
            case 1: EGG_V3(kVar3_64, double, 1); break;
            case 2: EGG_V3(kVar3_64, double, 2); break;
            case 3: EGG_V3(kVar3_64, double, 3); break;
            default: EGG_V3(kVar3_64, double, 4); break;
            }
        } else {
            switch (var) {
            case 0: EGG_V3(kVar3_32, float, 0); break;
            case 1: EGG_V3(kVar3_32, float, 1); break;
            case 2: EGG_V3(kVar3_32, float, 2); break;
            case 3: EGG_V3(kVar3_32, float, 3); break;
            default: EGG_V3(kVar3_32, float, 4); break;
            }
        }
        return;
    }
#undef EGG_V3
    if (S.prec == EGG_B200_PREC_FP64) {
        switch (var) {
        case 0: launch_tile<kVar64[0].ci, kVar64[0].cj, kVar64[0].minb, KIND, double, kVar64[0].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        case 1: launch_tile<kVar64[1].ci, kVar64[1].cj, kVar64[1].minb, KIND, double, kVar64[1].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        case 2: launch_tile<kVar64[2].ci, kVar64[2].cj, kVar64[2].minb, KIND, double, kVar64[2].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        case 3: launch_tile<kVar64[3].ci, kVar64[3].cj, kVar64[3].minb, KIND, double, kVar64[3].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        default: launch_tile<kVar64[4].ci, kVar64[4].cj, kVar64[4].minb, KIND, double, kVar64[4].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        }
    } else {
        switch (var) {
        case 0: launch_tile<kVar32[0].ci, kVar32[0].cj, kVar32[0].minb, KIND, float, kVar32[0].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        case 1: launch_tile<kVar32[1].ci, kVar32[1].cj, kVar32[1].minb, KIND, float, kVar32[1].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        case 2: launch_tile<kVar32[2].ci, kVar32[2].cj, kVar32[2].minb, KIND, float, kVar32[2].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        case 3: launch_tile<kVar32[3].ci, kVar32[3].cj, kVar32[3].minb, KIND, float, kVar32[3].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        default: launch_tile<kVar32[4].ci, kVar32[4].cj, kVar32[4].minb, KIND, float, kVar32[4].fd>(S, L, xin, xout, tau, delta, omega, gout); break;
        }
    }
}

// Time every interior-kernel variant on the resident data (reads the
// canonical buffer, writes the scratch buffer, so the state is untouched) and
// keep the fastest.
template <int KIND> static void autotune_impl(Session& S, int reps)
{
    if (S.n_interior == 0) {
        S.tuned = true;
        return;
    }
    cudaEvent_t a, b;
    EGG_CK(cudaEventCreate(&a));
    EGG_CK(cudaEventCreate(&b));
    const bool prof = S.profiling;
    S.profiling = false;
    const int64_t launches = S.launches;
    double best = 1e300;
    int best_v = 0;
    for (int v = 0; v < kNumVariants; ++v) {
        S.variant = v;
        set_tiles(S, S, variant_shape(S, v));
        launch_interior<KIND>(S, S, S.X(S.cur), S.X(1 - S.cur), nullptr, 0.0, 1.0);
        EGG_CK(cudaEventRecord(a, S.stream));
        for (int r = 0; r < reps; ++r) {
            launch_interior<KIND>(S, S, S.X(S.cur), S.X(1 - S.cur), nullptr, 0.0, 1.0);
        }
        EGG_CK(cudaEventRecord(b, S.stream));
        EGG_CK(cudaEventSynchronize(b));
        float ms = 0.f;
        EGG_CK(cudaEventElapsedTime(&ms, a, b));
        S.variant_ms[v] = double(ms) / reps;
        if (S.variant_ms[v] < best) {
            best = S.variant_ms[v];
            best_v = v;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    S.variant = best_v;
    set_tiles(S, S, variant_shape(S, best_v));
    S.profiling = prof;
    S.launches = launches;
    S.tuned = true;
}

static bool autotune_enabled()
{
    const char* v = std::getenv("EGG_B200_AUTOTUNE");
    return !(v && std::string(v) == "0");
}

static SoftTable soft_view(LevelData& L)
{
    return SoftTable {L.n_soft ? L.soft_off.p : nullptr, L.n_soft ? L.soft_terms.p : nullptr, L.soft_eps};
}

static StoredPatch2 stored_view(LevelData& S)
{
    StoredPatch2 sp;
    sp.n = S.n_stored;
    sp.slot = S.st_slot.p;
    sp.off = S.st_off.p;
    sp.gc = S.st_gc.p;
    sp.gn0 = S.st_gn0.p;
    sp.gn1 = S.st_gn1.p;
    sp.s0 = S.st_s0.p;
    sp.s1 = S.st_s1.p;
    sp.role = S.st_role.p;
    sp.W = S.st_W.p;
    sp.w_stride = S.st_wstride;
    sp.wt = S.st_wt.p;
    sp.wt_stride = S.st_wtstride;
    sp.etag = S.n_constrained ? S.st_etag.p : nullptr;
    sp.epar = S.n_constrained ? S.st_epar.p : nullptr;
    sp.cold = 0;
    sp.arena = (S.n_bspline || S.n_composite) ? S.arena.p : nullptr;
    sp.seeds = S.n_bspline ? S.seeds.p : nullptr;
    sp.soft = soft_view(S);
    return sp;
}

// Lanes per stored DOF (kStoredFillThreads2/3; EGG_B200_STORED_FILL
// overrides the thread budget).
static int stored_group(int64_t n, int dim)
{
    static const int64_t fill_env = [] {
        const char* e = std::getenv("EGG_B200_STORED_FILL");
        const long long v = e ? std::atoll(e) : 0;
        return int64_t(v > 0 ? v : 0);
    }();
    const int64_t fill = fill_env > 0 ? fill_env : (dim == 3 ? kStoredFillThreads3 : kStoredFillThreads2);
    for (int g : {32, 8, 2}) {
        if (n * g <= fill) { return g; }
    }
    return 1;
}

template <int KIND>
static void launch_stored(Session& S, LevelData& L, const double* xin, double* xout, const double* tau, double delta,
                          double omega, double* gout = nullptr, cudaStream_t on = nullptr, bool cold = false)
{
    if (L.n_stored == 0) { return; }
    const cudaStream_t st = on ? on : S.stream;
    const int G = stored_group(L.n_stored, S.dim);
    const unsigned grid = unsigned(std::min<int64_t>((L.n_stored * G + 127) / 128, 148 * 16));
    if (S.dim == 3) {
        StoredPatch3 sp {L.n_stored, L.st_slot.p, L.st_off.p, L.st_gc.p,  L.st_gn0.p, L.st_gn1.p,
                         L.st_gn2.p, L.st_s0.p,   L.st_s1.p,  L.st_s2.p, L.st_role.p, L.st_W.p,
                         L.st_wstride, L.st_wt.p, L.st_wtstride,
                         L.n_constrained ? L.st_etag.p : nullptr, L.n_constrained ? L.st_epar.p : nullptr,
                         cold ? 1 : 0, soft_view(L), L.n_bspline ? L.arena.p : nullptr,
                         L.n_bspline ? L.seeds.p : nullptr};
        auto go3 = [&](auto con) {
            constexpr bool C = decltype(con)::value;
            switch (G) {
            case 32: stored3_kernel<KIND, 32, C><<<grid, 128, 0, st>>>(sp, xin, xout, tau, delta, omega, gout); break;
            case 8: stored3_kernel<KIND, 8, C><<<grid, 128, 0, st>>>(sp, xin, xout, tau, delta, omega, gout); break;
            case 2: stored3_kernel<KIND, 2, C><<<grid, 128, 0, st>>>(sp, xin, xout, tau, delta, omega, gout); break;
            default: stored3_kernel<KIND, 1, C><<<grid, 128, 0, st>>>(sp, xin, xout, tau, delta, omega, gout); break;
            }
        };
        S.timed(kKStored, [&] {
            if (L.n_constrained) {
                go3(std::true_type {});
            } else {
                go3(std::false_type {});
            }
        });
        return;
    }
    StoredPatch2 sp = stored_view(L);
    sp.cold = cold ? 1 : 0;
    const auto* x2 = reinterpret_cast<const double2*>(xin);
    auto* o2 = reinterpret_cast<double2*>(xout);
    const auto* t2 = reinterpret_cast<const double2*>(tau);
    auto* g2 = reinterpret_cast<double2*>(gout);
    auto go2 = [&](auto con) {
        constexpr bool C = decltype(con)::value;
        switch (G) {
        case 32: stored_patch_kernel<KIND, 32, C><<<grid, 128, 0, st>>>(sp, x2, o2, t2, delta, omega, g2); break;
        case 8: stored_patch_kernel<KIND, 8, C><<<grid, 128, 0, st>>>(sp, x2, o2, t2, delta, omega, g2); break;
        case 2: stored_patch_kernel<KIND, 2, C><<<grid, 128, 0, st>>>(sp, x2, o2, t2, delta, omega, g2); break;
        default: stored_patch_kernel<KIND, 1, C><<<grid, 128, 0, st>>>(sp, x2, o2, t2, delta, omega, g2); break;
        }
    };
    // Levels without constrained DOFs (every coarse FAS level, most meshes)
    // launch the instantiation that carries no entity code.
    S.timed(kKStored, [&] {
        if (L.n_constrained) {
            go2(std::true_type {});
        } else {
            go2(std::false_type {});
        }
    });
}

static void launch_broadcast(Session& S, LevelData& L, double* x)
{
    if (L.nshare == 0) { return; }
    const unsigned grid = unsigned(std::min<int64_t>((L.nshare + 255) / 256, 148 * 8));
    if (S.dim == 3) {
        S.timed(kKBroadcast, [&] { broadcast3_kernel<<<grid, 256, 0, S.stream>>>(x, L.sh_src.p, L.sh_dst.p, L.nshare); });
        return;
    }
    S.timed(kKBroadcast, [&] {
        broadcast2_kernel<<<grid, 256, 0, S.stream>>>(reinterpret_cast<double2*>(x), L.sh_src.p, L.sh_dst.p, L.nshare);
    });
}

// The whole-sample directional total, added onto *out_e (no-op without one).
static void launch_soft_energy(Session& S, const double* x, double* out_e)
{
    if (S.es_dir_n == 0) { return; }
    S.timed(kKFinal, [&] {
        if (S.dim == 3) {
            soft_energy_add_kernel<3><<<1, 256, 0, S.stream>>>(S.es_dir.p, S.es_dir_n, S.es_dir_eps, x, out_e);
        } else {
            soft_energy_add_kernel<2><<<1, 256, 0, S.stream>>>(S.es_dir.p, S.es_dir_n, S.es_dir_eps, x, out_e);
        }
    });
}

template <int KIND> static void launch_reduce(Session& S, const double* x, double delta, double* out_e, double* out_m)
{
    double* ps = S.part.p;
    double* pc = ps + S.red_grid;
    double* pm = pc + S.red_grid;
    const auto* X2 = reinterpret_cast<const double2*>(x);
    if (S.es_struct) {
        EnergyStructured2 es;
        es.nblocks = int32_t(S.blocks_h.size());
        es.blocks = S.blocks_d.p;
        es.cell_off = S.es_cell_off.p;
        es.ncell = S.es_ncell;
        es.W = S.es_W.p;
        es.w_stride = S.es_wstride;
        es.wt = S.es_wt.p;
        es.wt_stride = S.es_wtstride;
        if (S.dim == 3) {
            S.timed(kKReduce, [&] {
                energy_structured3_kernel<KIND><<<S.red_grid, 256, 0, S.stream>>>(es, x, delta, ps, pc, pm);
            });
        } else {
            S.timed(kKReduce, [&] {
                energy_structured2_kernel<KIND><<<S.red_grid, 256, 0, S.stream>>>(es, X2, delta, ps, pc, pm);
            });
        }
    } else if (S.dim == 3) {
        EnergyStored3 es {S.es_ns,  S.es_gc.p, S.es_gn0.p,    S.es_gn1.p, S.es_gn2.p,     S.es_s0.p,
                          S.es_s1.p, S.es_s2.p, S.es_W.p, S.es_wstride, S.es_wt.p, S.es_wtstride};
        S.timed(kKReduce, [&] {
            energy_stored3_kernel<KIND><<<S.red_grid, 256, 0, S.stream>>>(es, x, delta, ps, pc, pm);
        });
    } else {
        EnergyStored2 es;
        es.n = S.es_ns;
        es.gc = S.es_gc.p;
        es.gn0 = S.es_gn0.p;
        es.gn1 = S.es_gn1.p;
        es.s0 = S.es_s0.p;
        es.s1 = S.es_s1.p;
        es.W = S.es_W.p;
        es.w_stride = S.es_wstride;
        es.wt = S.es_wt.p;
        es.wt_stride = S.es_wtstride;
        S.timed(kKReduce, [&] {
            energy_stored2_kernel<KIND><<<S.red_grid, 256, 0, S.stream>>>(es, X2, delta, ps, pc, pm);
        });
    }
    S.timed(kKFinal, [&] { reduce_finalize_kernel<<<1, 1024, 0, S.stream>>>(ps, pc, pm, S.red_grid, out_e, out_m); });
    launch_soft_energy(S, x, out_e);
}

// Per-mesh energy / min det of a batch session: CTA row m reduces mesh m's
// stencil items; out[2m] = energy, out[2m+1] = min det.
template <int KIND> static void launch_reduce_seg(Session& S, const double* x, double delta, double* out)
{
    double* ps = S.seg_part.p;
    const int64_t np = int64_t(S.seg_gx) * S.n_seg;
    double* pc = ps + np;
    double* pm = pc + np;
    const dim3 grid(unsigned(S.seg_gx), unsigned(S.n_seg));
    const auto* X2 = reinterpret_cast<const double2*>(x);
    if (S.es_struct) {
        EnergyStructured2 es;
        es.nblocks = int32_t(S.blocks_h.size());
        es.blocks = S.blocks_d.p;
        es.cell_off = S.es_cell_off.p;
        es.ncell = S.es_ncell;
        es.W = S.es_W.p;
        es.w_stride = S.es_wstride;
        es.wt = S.es_wt.p;
        es.wt_stride = S.es_wtstride;
        es.seg = S.seg_d.p;
        if (S.dim == 3) {
            S.timed(kKReduce, [&] {
                energy_structured3_kernel<KIND><<<grid, 256, 0, S.stream>>>(es, x, delta, ps, pc, pm);
            });
        } else {
            S.timed(kKReduce, [&] {
                energy_structured2_kernel<KIND><<<grid, 256, 0, S.stream>>>(es, X2, delta, ps, pc, pm);
            });
        }
    } else if (S.dim == 3) {
        EnergyStored3 es {S.es_ns,  S.es_gc.p, S.es_gn0.p,    S.es_gn1.p, S.es_gn2.p,     S.es_s0.p,
                          S.es_s1.p, S.es_s2.p, S.es_W.p, S.es_wstride, S.es_wt.p, S.es_wtstride, S.seg_d.p};
        S.timed(kKReduce, [&] {
            energy_stored3_kernel<KIND><<<grid, 256, 0, S.stream>>>(es, x, delta, ps, pc, pm);
        });
    } else {
        EnergyStored2 es;
        es.n = S.es_ns;
        es.gc = S.es_gc.p;
        es.gn0 = S.es_gn0.p;
        es.gn1 = S.es_gn1.p;
        es.s0 = S.es_s0.p;
        es.s1 = S.es_s1.p;
        es.W = S.es_W.p;
        es.w_stride = S.es_wstride;
        es.wt = S.es_wt.p;
        es.wt_stride = S.es_wtstride;
        es.seg = S.seg_d.p;
        S.timed(kKReduce, [&] {
            energy_stored2_kernel<KIND><<<grid, 256, 0, S.stream>>>(es, X2, delta, ps, pc, pm);
        });
    }
    S.timed(kKFinal, [&] {
        reduce_finalize_seg_kernel<<<unsigned(S.n_seg), 256, 0, S.stream>>>(ps, pc, pm, S.seg_gx, out);
    });
    if (S.es_dir_n) {
        S.timed(kKFinal, [&] {
            if (S.dim == 3) {
                soft_energy_add_seg_kernel<3><<<unsigned(S.n_seg), 256, 0, S.stream>>>(S.es_dir.p, S.es_dir_seg.p,
                                                                                       S.es_dir_eps, x, out);
            } else {
                soft_energy_add_seg_kernel<2><<<unsigned(S.n_seg), 256, 0, S.stream>>>(S.es_dir.p, S.es_dir_seg.p,
                                                                                       S.es_dir_eps, x, out);
            }
        });
    }
}

// One report's reduction: the whole store (2 doubles) or every mesh of a
// batch (2 * n_seg doubles, mesh-major).
template <int KIND> static void launch_report(Session& S, const double* x, double delta, bool per_mesh, double* out)
{
    if (per_mesh) {
        launch_reduce_seg<KIND>(S, x, delta, out);
    } else {
        launch_reduce<KIND>(S, x, delta, out, out + 1);
    }
}

// One block-Jacobi sweep xin -> xout (broadcast of the read buffer, then the
// interior tiles and the stored-patch DOFs).
// One relaxation of level L (or its gradient, gout): the interior tiles and
// the stored-patch DOFs read the same snapshot and write disjoint slots, so
// the stored-patch kernel forks onto the side stream beside the tiles.
template <int KIND>
static void relax_level(Session& S, LevelData& L, const double* xin, double* xout, const double* tau, double delta,
                        double omega, double* gout = nullptr, bool cold = false)
{
    if (L.n_stored > 0 && L.ntiles > 0 && !S.profiling) {
        EGG_CK(cudaEventRecord(S.fork_ev, S.stream));
        EGG_CK(cudaStreamWaitEvent(S.side, S.fork_ev, 0));
        launch_stored<KIND>(S, L, xin, xout, tau, delta, omega, gout, S.side, cold);
        EGG_CK(cudaEventRecord(S.join_ev, S.side));
        launch_interior<KIND>(S, L, xin, xout, tau, delta, omega, gout);
        EGG_CK(cudaStreamWaitEvent(S.stream, S.join_ev, 0));
    } else {
        launch_interior<KIND>(S, L, xin, xout, tau, delta, omega, gout);
        launch_stored<KIND>(S, L, xin, xout, tau, delta, omega, gout, nullptr, cold);
    }
}

template <int KIND>
static void sweep_once(Session& S, double* xin, double* xout, double delta, double omega, bool cold = false)
{
    launch_broadcast(S, S, xin);
    relax_level<KIND>(S, S, xin, xout, nullptr, delta, omega, nullptr, cold);
    S.updates += S.n_interior + S.n_stored;
}

static bool graphs_enabled()
{
    const char* e = std::getenv("EGG_B200_GRAPHS");
    return !(e && e[0] == '0');
}

// CUDA graph of one report chunk: k sweeps starting from `xin`, then the
// report reduction into red_tmp.  Captured once per (objective, delta,
// omega, k, start buffer, tile variant) and replayed; kernel arguments are
// baked in, so a change of tiles or buffers selects (or captures) another.
template <int KIND>
static Session::ChunkGraph& chunk_graph(Session& S, int k, bool per_mesh, double delta, double omega, double* xin,
                                        double* xout)
{
    const void* tiles = S.dim == 3 ? static_cast<const void*>(S.tiles3_d.p) : static_cast<const void*>(S.tiles_d.p);
    for (auto& g : S.graphs) {
        if (g.kind == KIND && g.k == k && g.per_mesh == per_mesh && g.delta == delta && g.omega == omega &&
            g.xin == xin && g.xout == xout && g.tiles == tiles && g.variant == S.variant) {
            return g;
        }
    }
    if (S.graphs.size() >= 16) { S.drop_graphs(); }
    const int64_t before = S.launches, upd_before = S.updates;
    EGG_CK(cudaStreamBeginCapture(S.stream, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try {
        double* a = xin;
        double* b = xout;
        for (int s = 0; s < k; ++s) {
            sweep_once<KIND>(S, a, b, delta, omega);
            std::swap(a, b);
        }
        launch_broadcast(S, S, a);
        launch_report<KIND>(S, a, delta, per_mesh, S.red_tmp.p);
    } catch (...) {
        cudaStreamEndCapture(S.stream, &graph);
        if (graph) { cudaGraphDestroy(graph); }
        cudaGetLastError();
        S.launches = before;
        S.updates = upd_before;
        throw;
    }
    EGG_CK(cudaStreamEndCapture(S.stream, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t st = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    EGG_CK(st);
    const int64_t n = S.launches - before, nu = S.updates - upd_before;
    S.launches = before;
    S.updates = upd_before;
    S.graphs.push_back({KIND, k, per_mesh, delta, omega, xin, xout, tiles, S.variant, exec, n, nu});
    return S.graphs.back();
}

template <int KIND> static void run_impl(Session& S, int n_sweeps, double delta, double omega, int report_every,
                                         std::vector<double>& E, std::vector<double>& Md, bool per_mesh = false)
{
    if (!S.tuned && autotune_enabled()) { autotune_impl<KIND>(S, 3); }
    const int k = report_every <= 0 ? n_sweeps : report_every;
    const int64_t nrep = (int64_t(n_sweeps) + k - 1) / k;
    const int64_t width = per_mesh ? S.n_seg : 1;
    if (S.red_out.n < size_t(2 * nrep * width)) { S.red_out.alloc(size_t(2 * nrep * width)); }
    if (S.red_tmp.n < size_t(2 * width)) {
        S.drop_graphs();  // captured chunks write the old red_tmp
        S.red_tmp.alloc(size_t(2 * width));
    }
    const size_t bytes = size_t(S.nstore) * S.dim * sizeof(double);
    double* xin = S.X(S.cur);
    double* xout = S.X(1 - S.cur);
    S.timed(kKCopy, [&] { EGG_CK(cudaMemcpyAsync(xout, xin, bytes, cudaMemcpyDeviceToDevice, S.stream)); });
    // Whole report chunks replay a captured graph (not while profiling, which
    // times every kernel with its own events).
    const bool use_graphs = graphs_enabled() && !S.profiling && k >= 2;
    int64_t ridx = 0;
    int s = 0;
    while (s < n_sweeps) {
        double* slot = S.red_out.p + 2 * width * ridx;
        // With arcs or planes the first sweep of the call is cold, so the first
        // report chunk runs launch by launch; captured chunks are warm.
        if (use_graphs && s % k == 0 && s + k <= n_sweeps && !(S.n_arc > 0 && s == 0)) {
            Session::ChunkGraph& g = chunk_graph<KIND>(S, k, per_mesh, delta, omega, xin, xout);
            EGG_CK(cudaGraphLaunch(g.exec, S.stream));
            S.launches += g.launches;
            S.updates += g.updates;
            EGG_CK(cudaMemcpyAsync(slot, S.red_tmp.p, size_t(2 * width) * sizeof(double), cudaMemcpyDeviceToDevice,
                                   S.stream));
            if (k % 2) {
                std::swap(xin, xout);
                S.cur = 1 - S.cur;
            }
            s += k;
            ++ridx;
            continue;
        }
        sweep_once<KIND>(S, xin, xout, delta, omega, s == 0);
        if ((s + 1) % k == 0 || s == n_sweeps - 1) {
            launch_broadcast(S, S, xout);
            launch_report<KIND>(S, xout, delta, per_mesh, slot);
            ++ridx;
        }
        std::swap(xin, xout);
        S.cur = 1 - S.cur;
        ++s;
        if (s % 64 == 0 && S.profiling) { S.sync(); }
    }
    std::vector<double> buf(size_t(2 * nrep * width));
    if (nrep) {
        EGG_CK(cudaMemcpyAsync(buf.data(), S.red_out.p, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
    }
    S.sync();
    E.resize(size_t(nrep * width));
    Md.resize(size_t(nrep * width));
    for (int64_t i = 0; i < nrep * width; ++i) {
        E[i] = buf[2 * i];
        Md[i] = buf[2 * i + 1];
    }
}

template <int KIND> static void energy_impl(Session& S, double delta, double& e, double& m)
{
    launch_broadcast(S, S, S.X(S.cur));
    launch_reduce<KIND>(S, S.X(S.cur), delta, S.red_out.p, S.red_out.p + 1);
    double buf[2];
    EGG_CK(cudaMemcpyAsync(buf, S.red_out.p, sizeof(buf), cudaMemcpyDeviceToHost, S.stream));
    S.sync();
    e = buf[0];
    m = buf[1];
}

// ---------------------------------------------------------------------------
// Allocation-free energy: the reduction of energy_impl with its scratch in a
// file-scope device array.  Layout (doubles): [0, 2) the results (energy,
// min det), then three runs of n_partials CTA partials (compensated sum,
// its error term, min det).  Each reduction CTA overwrites its own partial
// slot, so only the two result slots are cleared before the launch.
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxPartials = EGG_B200_NOALLOC_MAX_PARTIALS;
constexpr int kNoAllocMaxDevices = 64;
__device__ __align__(256) double g_noalloc_scratch[3 * kNoAllocMaxPartials + 2];

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch, looked up once per device with that
// device current.
static double* noalloc_scratch(int device)
{
    if (device < 0 || device >= kNoAllocMaxDevices) { invalid("energy_noalloc: device ordinal out of range"); }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        EGG_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[device] = static_cast<double*>(p);
    }
    return g_noalloc_ptr[device];
}

template <int KIND>
static void energy_noalloc_impl(Session& S, double delta, int grid, double* scratch, double& e, double& m)
{
    double* out = scratch;
    double* ps = scratch + 2;
    double* pc = ps + grid;
    double* pm = pc + grid;
    double* x = S.X(S.cur);
    const auto* X2 = reinterpret_cast<const double2*>(x);
    if (S.nshare) {
        const unsigned bgrid = unsigned(std::min<int64_t>((S.nshare + 255) / 256, 148 * 8));
        if (S.dim == 3) {
            broadcast3_kernel<<<bgrid, 256, 0, S.stream>>>(x, S.sh_src.p, S.sh_dst.p, S.nshare);
        } else {
            broadcast2_kernel<<<bgrid, 256, 0, S.stream>>>(reinterpret_cast<double2*>(x), S.sh_src.p, S.sh_dst.p,
                                                            S.nshare);
        }
        EGG_CK(cudaGetLastError());
        ++S.launches;
    }
    EGG_CK(cudaMemsetAsync(out, 0, 2 * sizeof(double), S.stream));
    if (S.es_struct) {
        EnergyStructured2 es;
        es.nblocks = int32_t(S.blocks_h.size());
        es.blocks = S.blocks_d.p;
        es.cell_off = S.es_cell_off.p;
        es.ncell = S.es_ncell;
        es.W = S.es_W.p;
        es.w_stride = S.es_wstride;
        es.wt = S.es_wt.p;
        es.wt_stride = S.es_wtstride;
        if (S.dim == 3) {
            energy_structured3_kernel<KIND><<<grid, 256, 0, S.stream>>>(es, x, delta, ps, pc, pm);
        } else {
            energy_structured2_kernel<KIND><<<grid, 256, 0, S.stream>>>(es, X2, delta, ps, pc, pm);
        }
    } else if (S.dim == 3) {
        EnergyStored3 es {S.es_ns,  S.es_gc.p, S.es_gn0.p,    S.es_gn1.p, S.es_gn2.p,     S.es_s0.p,
                          S.es_s1.p, S.es_s2.p, S.es_W.p, S.es_wstride, S.es_wt.p, S.es_wtstride};
        energy_stored3_kernel<KIND><<<grid, 256, 0, S.stream>>>(es, x, delta, ps, pc, pm);
    } else {
        EnergyStored2 es;
        es.n = S.es_ns;
        es.gc = S.es_gc.p;
        es.gn0 = S.es_gn0.p;
        es.gn1 = S.es_gn1.p;
        es.s0 = S.es_s0.p;
        es.s1 = S.es_s1.p;
        es.W = S.es_W.p;
        es.w_stride = S.es_wstride;
        es.wt = S.es_wt.p;
        es.wt_stride = S.es_wtstride;
        energy_stored2_kernel<KIND><<<grid, 256, 0, S.stream>>>(es, X2, delta, ps, pc, pm);
    }
    EGG_CK(cudaGetLastError());
    reduce_finalize_kernel<<<1, 1024, 0, S.stream>>>(ps, pc, pm, grid, out, out + 1);
    EGG_CK(cudaGetLastError());
    S.launches += 2;
    if (S.es_dir_n) {
        if (S.dim == 3) {
            soft_energy_add_kernel<3><<<1, 256, 0, S.stream>>>(S.es_dir.p, S.es_dir_n, S.es_dir_eps, x, out);
        } else {
            soft_energy_add_kernel<2><<<1, 256, 0, S.stream>>>(S.es_dir.p, S.es_dir_n, S.es_dir_eps, x, out);
        }
        EGG_CK(cudaGetLastError());
        ++S.launches;
    }
    double buf[2];
    EGG_CK(cudaMemcpyAsync(buf, out, sizeof(buf), cudaMemcpyDeviceToHost, S.stream));
    EGG_CK(cudaStreamSynchronize(S.stream));
    e = buf[0];
    m = buf[1];
}

#include "fas_host.inc"
#include "batch_host.inc"

template <int KIND> static void batch_energy_impl(Session& S, double delta, std::vector<double>& out)
{
    launch_broadcast(S, S, S.X(S.cur));
    launch_reduce_seg<KIND>(S, S.X(S.cur), delta, S.red_tmp.p);
    out.resize(2 * size_t(S.n_seg));
    EGG_CK(cudaMemcpyAsync(out.data(), S.red_tmp.p, out.size() * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
    S.sync();
}

// ---------------------------------------------------------------------------
// Oracle-primitive kernels
// ---------------------------------------------------------------------------
__global__ void metric_eval_kernel(int kind, double delta, const double* t, int64_t n, double* mu, double* g,
                                   double* H)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    double m, gg[4], hh[16];
    mu_eval<double>(kind, t + 4 * i, delta, m, gg, hh);
    mu[i] = m;
    for (int k = 0; k < 4; ++k) { g[4 * i + k] = gg[k]; }
    for (int k = 0; k < 16; ++k) { H[16 * i + k] = hh[k]; }
}

template <int KIND> __global__ void patch_eval_kernel(StoredPatch2 sp, const double2* X, double delta, double* out)
{
    double g[2], h[4], e0, md;
    stored_patch_eval<KIND>(sp, X, 0, delta, g, h, e0, md);
    double st[2];
    solve2<double>(h, g, st);
    out[0] = g[0];
    out[1] = g[1];
    for (int k = 0; k < 4; ++k) { out[2 + k] = h[k]; }
    out[6] = e0;
    out[7] = md;
    out[8] = st[0];
    out[9] = st[1];
}

__global__ void newton_step_kernel(const double* g, const double* h, double* out) { solve2<double>(h, g, out); }

// in: record[EGG_B200_ENTITY_FIELDS], grad[2], hess[4], pos[2]; out: step[2], foot[2]
__global__ void entity_step_kernel(int tag, const double* in, double* out)
{
    constexpr int R = EGG_B200_ENTITY_FIELDS;
    entity_newton_step(tag, in, in + R + 2, in + R, in[R + 6], in[R + 7], out);
    entity_project(tag, in, in[R + 6], in[R + 7], out[2], out[3]);
}

// Foot and orthonormal tangent basis of n points on one entity: 2D curves
// (the unit tangent at the cold foot, as the sweep's cold path takes it), 3D
// surfaces (two Gram-Schmidt columns of the raw frame at the foot) and lines
// (one column).  basis is packed (point, component, column).
__global__ void entity_frame_kernel(int dim, int tag, const double* __restrict__ e, const double* __restrict__ arena,
                                    const double* __restrict__ q, int64_t n, double* __restrict__ foot,
                                    double* __restrict__ basis)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    if (dim == 2) {
        const double px = q[2 * i], py = q[2 * i + 1];
        double fx, fy, tx, ty;
        if (tag == EGG_B200_TAG_COMPOSITE) {
            const double* slice = arena + int64_t(e[6]);
            composite_frame(slice, slice + int64_t(e[1]), int(e[0]), px, py, fx, fy, tx, ty);
        } else if (tag == EGG_B200_TAG_BSPLINE) {
            const BSplineCurve c = bspline_view(e, arena);
            double t = bspline_foot(c, px, py, NAN);
            if (!bspline_inside(c, t)) { t = bspline_clamp(c, t); }
            bspline_point(c, t, 0, fx, fy);
            double jx, jy;
            bspline_point(c, t, 1, jx, jy);
            unit_or_e0(jx, jy, tx, ty);
        } else {
            entity_project(tag, e, px, py, fx, fy);
            entity_tangent(tag, e, px, py, tx, ty);
        }
        foot[2 * i] = fx;
        foot[2 * i + 1] = fy;
        basis[2 * i] = tx;
        basis[2 * i + 1] = ty;
        return;
    }
    const double* p = q + 3 * i;
    if (tag == EGG_B200_TAG_BSPLINESURF) {
        double io[3] = {p[0], p[1], p[2]}, B[6];
        bsurf_dof(kBsurfFrame, e, arena, nullptr, nullptr, nullptr, 0.0, 0.0, nullptr, nullptr, nullptr, io, B);
        for (int k = 0; k < 3; ++k) {
            foot[3 * i + k] = io[k];
            basis[(3 * i + k) * 2] = B[k];
            basis[(3 * i + k) * 2 + 1] = B[3 + k];
        }
        return;
    }
    entity3_project(tag, e, p, foot + 3 * i);
    double B[2][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}};
    if (is_param3(tag)) {
        double qq[2], J[2][3];
        p3_invert(tag, e, p, qq);
        p3_clamp(tag, e, qq);
        p3_frame(tag, e, qq, J);
        p3_basis(tag, J, B);
    } else {  // rail: its direction
        const double d[3] = {e[3] - e[0], e[4] - e[1], e[5] - e[2]};
        const double norm = sqrt(dot3v(d, d));
        if (!(norm < kGeomZnorm)) {
            for (int k = 0; k < 3; ++k) { B[0][k] = d[k] / norm; }
        }
    }
    const int K = is_surf3(tag) ? 2 : 1;
    for (int k = 0; k < 3; ++k) {
        for (int c = 0; c < K; ++c) { basis[(3 * i + k) * K + c] = B[c][k]; }
    }
}

// Directional soft terms over a sample table: each thread one sample's
// energy and its gradient on each of the sample's nodes (slot order); the
// host sums them in table order.
template <int D>
__global__ void directional_eval_kernel(const double* __restrict__ X, const SoftTerm* __restrict__ terms, int64_t n,
                                        double eps, double* __restrict__ energy, double* __restrict__ grad)
{
    const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    SoftTerm t = terms[i];
    double p[4][3];
    soft_load<D>(t, X, p);
    energy[i] = soft_energy<D>(t, p, eps);
    const int ar = soft_arity(t.kind);
    for (int m = 0; m < ar; ++m) {
        t.slot = m;
        double g[D] = {}, H[D * D] = {}, e0 = 0.0;
        soft_accumulate<D>(t, X, eps, g, H, e0);
        for (int k = 0; k < D; ++k) { grad[(i * 4 + m) * D + k] = g[k]; }
    }
}

template <class F> static int guarded(F&& f)
{
    try {
        f();
        return EGG_B200_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "egg_b200: host out of memory";
        return EGG_B200_ERUNTIME;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return EGG_B200_ERUNTIME;
    }
}

static void check_objective(int obj)
{
    if (obj != EGG_B200_OBJ_SHAPE && obj != EGG_B200_OBJ_UNTANGLE && obj != EGG_B200_OBJ_SHAPE_SIZE) {
        invalid("unknown objective kind " + std::to_string(obj));
    }
}

#include "control_host.inc"
#include "control_topo_host.inc"
#include "control_walls_host.inc"

}  // namespace egg_b200

// ===========================================================================
// C-ABI
// ===========================================================================
using namespace egg_b200;

struct egg_b200_session {
    Session* impl;
};


static void ensure_xfer(Session& S)
{
    const size_t n = size_t(S.M) * S.dim;
    if (!S.pin && n) {
        EGG_CK(cudaHostAlloc(reinterpret_cast<void**>(&S.pin), n * sizeof(double), cudaHostAllocDefault));
    }
    if (S.Xg.n != n) { S.Xg.alloc(n); }
    if (S.g2s_d.n != S.g2s.size()) { S.g2s_d.upload(S.g2s); }
    if (S.slot_gid_d.n != S.slot_gid.size()) { S.slot_gid_d.upload(S.slot_gid); }
    for (cudaEvent_t& e : S.xfer_ev) {
        if (!e) { EGG_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)); }
    }
}

// The B-spline seeds after a position reset: NaN (the next projection seeds
// from its coarse grid), as the reference's upload_X does (src/sweep.hpp:592-597).
static void reset_seeds(Session& S)
{
    if (S.n_bspline) { EGG_CK(cudaMemsetAsync(S.seeds.p, 0xFF, S.seeds.n * sizeof(double), S.stream)); }
}


extern "C" {

int egg_b200_abi_version(void) { return EGG_B200_ABI_VERSION; }

const char* egg_b200_last_error(void) { return g_last_error.c_str(); }

int egg_b200_device_count(int* count)
{
    return guarded([&] {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        *count = n;
    });
}

int egg_b200_session_create(const egg_b200_session_desc* desc, egg_b200_session** out)
{
    return guarded([&] {
        if (!desc || !out) { invalid("egg_b200_session_create: NULL argument"); }
        *out = nullptr;
        Session* s = create_session(*desc);
        *out = new egg_b200_session {s};
    });
}

int egg_b200_batch_create(const egg_b200_session_desc* descs, int32_t n_meshes, egg_b200_session** out)
{
    return guarded([&] {
        if (!descs || !out) { invalid("egg_b200_batch_create: NULL argument"); }
        *out = nullptr;
        Session* s = create_batch(descs, n_meshes);
        *out = new egg_b200_session {s};
    });
}

int egg_b200_batch_size(egg_b200_session* s, int32_t* n_meshes, int64_t* node_offsets)
{
    return guarded([&] {
        if (!s || !n_meshes) { invalid("batch_size: NULL argument"); }
        const Session& S = *s->impl;
        *n_meshes = S.n_seg;
        if (node_offsets) {
            for (size_t i = 0; i < S.mesh_node_off.size(); ++i) { node_offsets[i] = S.mesh_node_off[i]; }
        }
    });
}

int egg_b200_batch_run(egg_b200_session* s, int32_t n_sweeps, int32_t objective, double delta, double omega,
                       int32_t report_every, double* energies, double* mindets, int64_t capacity,
                       int64_t* n_reported)
{
    return guarded([&] {
        if (!s) { invalid("batch_run: NULL session"); }
        check_objective(objective);
        if (n_sweeps < 0) { invalid("batch_run: n_sweeps must be >= 0"); }
        Session& S = *s->impl;
        if (S.n_seg <= 0) { invalid("batch_run: not a batch session"); }
        EGG_CK(cudaSetDevice(S.device));
        std::vector<double> E, Md;
        if (n_sweeps > 0) {
            switch (objective) {
            case EGG_B200_OBJ_SHAPE: run_impl<kShape>(S, n_sweeps, delta, omega, report_every, E, Md, true); break;
            case EGG_B200_OBJ_UNTANGLE:
                run_impl<kUntangle>(S, n_sweeps, delta, omega, report_every, E, Md, true);
                break;
            default: run_impl<kShapeSize>(S, n_sweeps, delta, omega, report_every, E, Md, true); break;
            }
        }
        const int64_t nrep = int64_t(E.size()) / S.n_seg;
        if (n_reported) { *n_reported = nrep; }
        if (nrep > capacity) { invalid("batch_run: report buffer too small"); }
        for (size_t i = 0; i < E.size(); ++i) {
            if (energies) { energies[i] = E[i]; }
            if (mindets) { mindets[i] = Md[i]; }
        }
    });
}

int egg_b200_batch_energy(egg_b200_session* s, int32_t objective, double delta, double* energies, double* mindets)
{
    return guarded([&] {
        if (!s) { invalid("batch_energy: NULL session"); }
        check_objective(objective);
        Session& S = *s->impl;
        if (S.n_seg <= 0) { invalid("batch_energy: not a batch session"); }
        EGG_CK(cudaSetDevice(S.device));
        std::vector<double> out;
        switch (objective) {
        case EGG_B200_OBJ_SHAPE: batch_energy_impl<kShape>(S, delta, out); break;
        case EGG_B200_OBJ_UNTANGLE: batch_energy_impl<kUntangle>(S, delta, out); break;
        default: batch_energy_impl<kShapeSize>(S, delta, out); break;
        }
        for (int m = 0; m < S.n_seg; ++m) {
            if (energies) { energies[m] = out[2 * m]; }
            if (mindets) { mindets[m] = out[2 * m + 1]; }
        }
    });
}

int egg_b200_session_attach_control(egg_b200_session* s, const egg_b200_control_desc* desc)
{
    return guarded([&] {
        if (!s || !desc) { invalid("attach_control: NULL argument"); }
        Session& S = *s->impl;
        if (S.n_seg > 0) { invalid("attach_control: a batch session takes one net per mesh (batch_attach_controls)"); }
        attach_control(S, desc, 1, nullptr, nullptr);
    });
}

int egg_b200_session_attach_control_walls(egg_b200_session* s, const egg_b200_control_desc* desc, const double* X0,
                                          int64_t X0_len, int32_t n_walls, const egg_b200_control_wall* walls)
{
    return guarded([&] {
        if (!s || !desc) { invalid("attach_control_walls: NULL argument"); }
        Session& S = *s->impl;
        if (S.n_seg > 0) { invalid("attach_control_walls: a batch session takes plain nets (batch_attach_controls)"); }
        EGG_CK(cudaSetDevice(S.device));
        attach_control_walls(S, *desc, X0, X0_len, n_walls, walls);
    });
}

int egg_b200_session_attach_control_topo(egg_b200_session* s, const egg_b200_control_topo_desc* desc)
{
    return guarded([&] {
        if (!s || !desc) { invalid("attach_control_topo: NULL argument"); }
        Session& S = *s->impl;
        if (S.n_seg > 0) { invalid("attach_control_topo: a batch session takes one net per mesh"); }
        EGG_CK(cudaSetDevice(S.device));
        attach_control_topo(S, *desc);
    });
}

static Session& topo_session(egg_b200_session* s, const char* what)
{
    if (!s) { invalid(std::string(what) + ": NULL session"); }
    Session& S = *s->impl;
    if (!S.ctl || !S.ctl->topo || S.ctl->walls) {
        invalid(std::string(what) + ": session has no multi-block control wire");
    }
    EGG_CK(cudaSetDevice(S.device));
    return S;
}

int egg_b200_session_set_control_reduction(egg_b200_session* s, int64_t nq, const int32_t* off, int64_t off_len,
                                           const int32_t* col, const double* coef, int64_t nnz)
{
    return guarded([&] {
        Session& S = topo_session(s, "set_control_reduction");
        topo_set_reduction(S, nq, off, off_len, col, coef, nnz);
    });
}

int egg_b200_session_set_control_penalty(egg_b200_session* s, const int32_t* off, int64_t off_len,
                                         const int32_t* col, const double* coef, int64_t nnz, const double* w,
                                         int64_t w_len)
{
    return guarded([&] {
        Session& S = topo_session(s, "set_control_penalty");
        topo_set_penalty(S, off, off_len, col, coef, nnz, w, w_len);
    });
}

int egg_b200_session_set_control_b(egg_b200_session* s, int32_t net_index, const double* b, int64_t len)
{
    return guarded([&] {
        Session& S = topo_session(s, "set_control_b");
        topo_set_b(S, net_index, b, len);
    });
}

int egg_b200_batch_attach_controls(egg_b200_session* s, const egg_b200_control_desc* descs)
{
    return guarded([&] {
        if (!s || !descs) { invalid("batch_attach_controls: NULL argument"); }
        Session& S = *s->impl;
        if (S.n_seg <= 0) { invalid("batch_attach_controls: not a batch session"); }
        // first block of each mesh: blocks are packed mesh by mesh
        std::vector<int32_t> base(size_t(S.n_seg) + 1, 0);
        std::vector<int> mesh(size_t(S.n_seg));
        int32_t b = 0;
        for (int m = 0; m < S.n_seg; ++m) {
            base[size_t(m)] = b;
            mesh[size_t(m)] = m;
            while (b < int32_t(S.blocks_h.size()) && S.slot_gid[size_t(S.blocks_h[size_t(b)].off)] <
                                                         S.mesh_node_off[size_t(m) + 1]) {
                ++b;
            }
        }
        base[size_t(S.n_seg)] = b;
        attach_control(S, descs, S.n_seg, base.data(), mesh.data());
    });
}

int egg_b200_session_run_control(egg_b200_session* s, int32_t n_outer, int32_t objective, double grad_tol,
                                 double alpha_min, double lm0, int32_t pcg_max_iter, double pcg_rtol,
                                 int32_t pcg_forcing, double* energies, double* mindets, double* alphas,
                                 double* pcg_iters, double* pcg_relres, int64_t* counts, int32_t* iters,
                                 int32_t* converged)
{
    return guarded([&] {
        if (!s) { invalid("run_control: NULL session"); }
        run_control_abi(*s->impl, n_outer, objective, grad_tol, alpha_min, lm0, pcg_max_iter, pcg_rtol, pcg_forcing,
                        energies, mindets, alphas, pcg_iters, pcg_relres, counts, iters, converged, false);
    });
}

int egg_b200_session_run_control_ex(egg_b200_session* s, int32_t n_outer, int32_t objective, double grad_tol,
                                    double alpha_min, double lm0, int32_t pcg_max_iter, double pcg_rtol,
                                    int32_t pcg_forcing, int32_t model_db, double* energies, double* mindets,
                                    double* alphas, double* pcg_iters, double* pcg_relres, int64_t* counts,
                                    int32_t* iters, int32_t* converged, double* frame_jumps, int64_t* n_frame_jumps)
{
    return guarded([&] {
        if (!s) { invalid("run_control: NULL session"); }
        run_control_abi(*s->impl, n_outer, objective, grad_tol, alpha_min, lm0, pcg_max_iter, pcg_rtol, pcg_forcing,
                        energies, mindets, alphas, pcg_iters, pcg_relres, counts, iters, converged, false, model_db,
                        frame_jumps, n_frame_jumps);
    });
}

int egg_b200_batch_run_control(egg_b200_session* s, int32_t n_outer, int32_t objective, double grad_tol,
                               double alpha_min, double lm0, int32_t pcg_max_iter, double pcg_rtol,
                               int32_t pcg_forcing, double* energies, double* mindets, double* alphas,
                               double* pcg_iters, double* pcg_relres, int64_t* counts, int32_t* iters,
                               int32_t* converged)
{
    return guarded([&] {
        if (!s) { invalid("batch_run_control: NULL session"); }
        run_control_abi(*s->impl, n_outer, objective, grad_tol, alpha_min, lm0, pcg_max_iter, pcg_rtol, pcg_forcing,
                        energies, mindets, alphas, pcg_iters, pcg_relres, counts, iters, converged, true);
    });
}

int egg_b200_session_control_size(egg_b200_session* s, int64_t* n_reals)
{
    return guarded([&] {
        if (!s || !n_reals) { invalid("control_size: NULL argument"); }
        const Session& S = *s->impl;
        *n_reals = S.ctl ? S.ctl->total_ctrl * S.dim : 0;
    });
}

int egg_b200_session_get_C(egg_b200_session* s, double* C, int64_t len)
{
    return guarded([&] {
        if (!s || !C) { invalid("get_C: NULL argument"); }
        Session& S = *s->impl;
        if (!S.ctl) { invalid("get_C: session has no control wire"); }
        check_len(len, S.ctl->total_ctrl * S.dim, "get_C buffer");
        EGG_CK(cudaSetDevice(S.device));
        EGG_CK(cudaMemcpyAsync(C, S.ctl->C.p, size_t(len) * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
        S.sync();
    });
}

int egg_b200_session_set_C(egg_b200_session* s, const double* C, int64_t len)
{
    return guarded([&] {
        if (!s || !C) { invalid("set_C: NULL argument"); }
        Session& S = *s->impl;
        if (!S.ctl) { invalid("set_C: session has no control wire"); }
        if (len != S.ctl->total_ctrl * S.dim) {
            invalid("set_c: expected " + std::to_string(S.ctl->total_ctrl * S.dim) + " reals, got " +
                    std::to_string(len));
        }
        EGG_CK(cudaSetDevice(S.device));
        EGG_CK(cudaMemcpyAsync(S.ctl->C.p, C, size_t(len) * sizeof(double), cudaMemcpyHostToDevice, S.stream));
        ctl_eval_to_x(S);
        S.sync();
    });
}

int egg_b200_session_destroy(egg_b200_session* s)
{
    return guarded([&] {
        if (!s) { return; }
        delete s->impl;
        delete s;
    });
}

int egg_b200_session_run(egg_b200_session* s, int32_t n_sweeps, int32_t objective, double delta, double omega,
                         int32_t report_every, double* energies, double* mindets, int64_t capacity,
                         int64_t* n_reported)
{
    return guarded([&] {
        if (!s) { invalid("run: NULL session"); }
        check_objective(objective);
        if (n_sweeps < 0) { invalid("run: n_sweeps must be >= 0"); }
        Session& S = *s->impl;
        EGG_CK(cudaSetDevice(S.device));
        std::vector<double> E, Md;
        if (n_sweeps > 0) {
            switch (objective) {
            case EGG_B200_OBJ_SHAPE: run_impl<kShape>(S, n_sweeps, delta, omega, report_every, E, Md); break;
            case EGG_B200_OBJ_UNTANGLE: run_impl<kUntangle>(S, n_sweeps, delta, omega, report_every, E, Md); break;
            default: run_impl<kShapeSize>(S, n_sweeps, delta, omega, report_every, E, Md); break;
            }
        }
        if (n_reported) { *n_reported = int64_t(E.size()); }
        if (int64_t(E.size()) > capacity) { invalid("run: report buffer too small"); }
        for (size_t i = 0; i < E.size(); ++i) {
            if (energies) { energies[i] = E[i]; }
            if (mindets) { mindets[i] = Md[i]; }
        }
    });
}

int egg_b200_session_run_fas(egg_b200_session* s, int32_t n_cycles, int32_t nu_pre, int32_t nu_post,
                             int32_t nu_coarse, double omega, int32_t max_levels, int32_t objective,
                             double* energies, double* mindets, int64_t capacity, int64_t* n_reported)
{
    return guarded([&] {
        if (!s) { invalid("run_fas: NULL session"); }
        check_objective(objective);
        if (objective == EGG_B200_OBJ_UNTANGLE) {
            invalid("run_fas: FAS supports the shape phase only, not \"untangle\"");
        }
        if (n_cycles < 0 || nu_pre < 0 || nu_post < 0 || nu_coarse < 0) { invalid("run_fas: negative counts"); }
        Session& S = *s->impl;
        if (S.n_seg > 0) {
            throw Error(EGG_B200_ENOTSUP, "run_fas: FAS is not available on a batch session (one session per mesh)");
        }
        EGG_CK(cudaSetDevice(S.device));
        std::vector<double> E, Md;
        if (n_cycles > 0) {
            if (objective == EGG_B200_OBJ_SHAPE) {
                run_fas_impl<kShape>(S, n_cycles, nu_pre, nu_post, nu_coarse, omega, max_levels, E, Md);
            } else {
                run_fas_impl<kShapeSize>(S, n_cycles, nu_pre, nu_post, nu_coarse, omega, max_levels, E, Md);
            }
        }
        if (n_reported) { *n_reported = int64_t(E.size()); }
        if (int64_t(E.size()) > capacity) { invalid("run_fas: report buffer too small"); }
        for (size_t i = 0; i < E.size(); ++i) {
            if (energies) { energies[i] = E[i]; }
            if (mindets) { mindets[i] = Md[i]; }
        }
    });
}

int egg_b200_session_mg_levels(egg_b200_session* s, int32_t* n_levels)
{
    return guarded([&] {
        if (!s || !n_levels) { invalid("mg_levels: NULL argument"); }
        Session& S = *s->impl;
        EGG_CK(cudaSetDevice(S.device));
        ensure_hierarchy(S);
        *n_levels = int32_t(S.levels.size());
    });
}

int egg_b200_session_mg_level_shapes(egg_b200_session* s, int32_t level, int32_t* shapes, int64_t len)
{
    return guarded([&] {
        if (!s || !shapes) { invalid("mg_level_shapes: NULL argument"); }
        Session& S = *s->impl;
        ensure_hierarchy(S);
        if (level < 0 || level >= int32_t(S.levels.size())) { invalid("mg_level_shapes: level out of range"); }
        const auto& bl = S.levels[level]->blocks_h;
        if (len != int64_t(bl.size()) * S.dim) { invalid("mg_level_shapes: output length != num_blocks*dim"); }
        for (size_t b = 0; b < bl.size(); ++b) {
            for (int k = 0; k < S.dim; ++k) { shapes[b * S.dim + k] = bl[b].n[k]; }
        }
    });
}

int egg_b200_session_energy(egg_b200_session* s, int32_t objective, double delta, double* energy, double* mindet)
{
    return guarded([&] {
        if (!s) { invalid("energy: NULL session"); }
        check_objective(objective);
        Session& S = *s->impl;
        EGG_CK(cudaSetDevice(S.device));
        double e = 0, m = 0;
        switch (objective) {
        case EGG_B200_OBJ_SHAPE: energy_impl<kShape>(S, delta, e, m); break;
        case EGG_B200_OBJ_UNTANGLE: energy_impl<kUntangle>(S, delta, e, m); break;
        default: energy_impl<kShapeSize>(S, delta, e, m); break;
        }
        if (energy) { *energy = e; }
        if (mindet) { *mindet = m; }
    });
}

int egg_b200_session_energy_noalloc(egg_b200_session* s, int32_t objective, double delta, int32_t n_partials,
                                    double* energy, double* mindet)
{
    return guarded([&] {
        if (!s) { invalid("energy_noalloc: NULL session"); }
        check_objective(objective);
        if (n_partials < 0 || n_partials > kNoAllocMaxPartials) {
            invalid("energy_noalloc: n_partials must lie in [0, " + std::to_string(kNoAllocMaxPartials) +
                    "] (0 = the session's own count); got " + std::to_string(n_partials));
        }
        Session& S = *s->impl;
        const int grid = n_partials ? n_partials : S.red_grid;
        if (grid > kNoAllocMaxPartials) { invalid("energy_noalloc: session partial count exceeds the static array"); }
        EGG_CK(cudaSetDevice(S.device));
        double* scratch = noalloc_scratch(S.device);
        double e = 0, m = 0;
        switch (objective) {
        case EGG_B200_OBJ_SHAPE: energy_noalloc_impl<kShape>(S, delta, grid, scratch, e, m); break;
        case EGG_B200_OBJ_UNTANGLE: energy_noalloc_impl<kUntangle>(S, delta, grid, scratch, e, m); break;
        default: energy_noalloc_impl<kShapeSize>(S, delta, grid, scratch, e, m); break;
        }
        if (energy) { *energy = e; }
        if (mindet) { *mindet = m; }
    });
}

int egg_b200_session_get_X(egg_b200_session* s, double* X, int64_t len)
{
    return guarded([&] {
        if (!s || !X) { invalid("get_X: NULL argument"); }
        Session& S = *s->impl;
        const int D = S.dim;
        if (len != S.M * D) { invalid("get_X: output length " + std::to_string(len) + " != num_nodes*dim"); }
        EGG_CK(cudaSetDevice(S.device));
        ensure_xfer(S);
        const size_t n = size_t(len);
        if (S.M) {
            if (D == 2) {
                scatter_global_kernel<2><<<remap_grid(S.M), 256, 0, S.stream>>>(S.X(S.cur), S.g2s_d.p, S.M, S.Xg.p);
            } else {
                scatter_global_kernel<3><<<remap_grid(S.M), 256, 0, S.stream>>>(S.X(S.cur), S.g2s_d.p, S.M, S.Xg.p);
            }
            EGG_CK(cudaGetLastError());
            ++S.launches;
        }
        // Page-locked output: one DMA straight into it.
        cudaPointerAttributes attr {};
        const bool pinned = cudaPointerGetAttributes(&attr, X) == cudaSuccess && attr.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (pinned && n) {
            EGG_CK(cudaMemcpyAsync(X, S.Xg.p, n * sizeof(double), cudaMemcpyDeviceToHost, S.stream));
            EGG_CK(cudaStreamSynchronize(S.stream));
        }
        // Otherwise D2H slice by slice, each followed by its event; host thread
        // t waits for slice t only, so the copy-out of early slices overlaps
        // the DMA.
        const int T = pinned ? 0 : copy_threads(n * sizeof(double));
        for (int t = 0; t < T; ++t) {
            const size_t a = slice_begin(n, t, T), b = slice_begin(n, t + 1, T);
            if (b > a) {
                EGG_CK(cudaMemcpyAsync(S.pin + a, S.Xg.p + a, (b - a) * sizeof(double), cudaMemcpyDeviceToHost,
                                       S.stream));
            }
            EGG_CK(cudaEventRecord(S.xfer_ev[t], S.stream));
        }
        cudaError_t err[kMaxCopyThreads] = {};
        if (T > 0) {
            run_slices(T, [&](int t) {
                const size_t a = slice_begin(n, t, T), b = slice_begin(n, t + 1, T);
                err[t] = cudaSetDevice(S.device);
                if (err[t] == cudaSuccess) { err[t] = cudaEventSynchronize(S.xfer_ev[t]); }
                if (err[t] == cudaSuccess && b > a) { std::memcpy(X + a, S.pin + a, (b - a) * sizeof(double)); }
            });
        }
        for (int t = 0; t < T; ++t) { EGG_CK(err[t]); }
        for (size_t j = 0; j < S.nb_gid.size(); ++j) {
            for (int k = 0; k < D; ++k) { X[S.nb_gid[j] * D + k] = S.nb_val[j * D + k]; }
        }
        S.sync();
    });
}

int egg_b200_session_set_X(egg_b200_session* s, const double* X, int64_t len)
{
    return guarded([&] {
        if (!s || !X) { invalid("set_X: NULL argument"); }
        Session& S = *s->impl;
        const int D = S.dim;
        if (len != S.M * D) { invalid("set_X: input length != num_nodes*dim"); }
        EGG_CK(cudaSetDevice(S.device));
        ensure_xfer(S);
        const size_t n = size_t(len);
        // Page-locked input: one DMA straight from it.  Otherwise host thread
        // t stages slice t in pinned memory and queues its H2D, so the DMA of
        // early slices overlaps the staging of later ones.
        cudaPointerAttributes attr {};
        const bool pinned = cudaPointerGetAttributes(&attr, X) == cudaSuccess && attr.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (pinned && n) {
            EGG_CK(cudaMemcpyAsync(S.Xg.p, X, n * sizeof(double), cudaMemcpyHostToDevice, S.stream));
        }
        const int T = pinned ? 0 : copy_threads(n * sizeof(double));
        cudaError_t err[kMaxCopyThreads] = {};
        if (T > 0) {
            run_slices(T, [&](int t) {
                const size_t a = slice_begin(n, t, T), b = slice_begin(n, t + 1, T);
                if (b == a) { return; }
                std::memcpy(S.pin + a, X + a, (b - a) * sizeof(double));
                err[t] = cudaSetDevice(S.device);
                if (err[t] == cudaSuccess) {
                    err[t] = cudaMemcpyAsync(S.Xg.p + a, S.pin + a, (b - a) * sizeof(double), cudaMemcpyHostToDevice,
                                             S.stream);
                }
            });
        }
        for (int t = 0; t < T; ++t) { EGG_CK(err[t]); }
        if (S.nstore) {
            if (D == 2) {
                gather_global_kernel<2><<<remap_grid(S.nstore), 256, 0, S.stream>>>(S.Xg.p, S.slot_gid_d.p, S.nstore,
                                                                                 S.X(S.cur));
            } else {
                gather_global_kernel<3><<<remap_grid(S.nstore), 256, 0, S.stream>>>(S.Xg.p, S.slot_gid_d.p, S.nstore,
                                                                                 S.X(S.cur));
            }
            EGG_CK(cudaGetLastError());
            ++S.launches;
        }
        for (size_t j = 0; j < S.nb_gid.size(); ++j) {
            for (int k = 0; k < D; ++k) { S.nb_val[j * D + k] = X[S.nb_gid[j] * D + k]; }
        }
        reset_seeds(S);  // new positions: B-spline projections start cold
        S.sync();
    });
}

int egg_b200_session_info(egg_b200_session* s, int64_t* out, int32_t n)
{
    return guarded([&] {
        if (!s || !out) { invalid("info: NULL argument"); }
        Session& S = *s->impl;
        const int64_t v[11] = {S.dim,    S.M,     S.nstore,           S.n_interior + S.n_stored, S.n_interior, S.n_stored,
                               S.nshare, S.es_ns, S.es_struct ? 1 : 0, S.prec,                    S.updates};
        for (int i = 0; i < n && i < 11; ++i) { out[i] = v[i]; }
    });
}

int egg_b200_session_set_profiling(egg_b200_session* s, int32_t enable)
{
    return guarded([&] {
        if (!s) { invalid("set_profiling: NULL session"); }
        s->impl->sync();
        s->impl->profiling = enable != 0;
    });
}

int egg_b200_session_kernel_stats(egg_b200_session* s, int32_t kernel_id, double* total_ms, int64_t* launches)
{
    return guarded([&] {
        if (!s) { invalid("kernel_stats: NULL session"); }
        if (kernel_id < 0 || kernel_id >= kKCount) { invalid("kernel_stats: unknown kernel id"); }
        s->impl->sync();
        if (total_ms) { *total_ms = s->impl->k_ms[kernel_id]; }
        if (launches) { *launches = s->impl->k_launch[kernel_id]; }
    });
}

int egg_b200_session_checkpoint(egg_b200_session* s)
{
    return guarded([&] {
        if (!s) { invalid("checkpoint: NULL session"); }
        Session& S = *s->impl;
        EGG_CK(cudaSetDevice(S.device));
        const size_t n = size_t(S.nstore) * S.dim;
        if (S.ckpt.n != n) { S.ckpt.alloc(n); }
        if (n) { EGG_CK(cudaMemcpyAsync(S.ckpt.p, S.X(S.cur), n * sizeof(double), cudaMemcpyDeviceToDevice, S.stream)); }
        S.sync();
        S.has_ckpt = true;
    });
}

int egg_b200_session_restore(egg_b200_session* s)
{
    return guarded([&] {
        if (!s) { invalid("restore: NULL session"); }
        Session& S = *s->impl;
        if (!S.has_ckpt) { invalid("restore: no checkpoint taken"); }
        EGG_CK(cudaSetDevice(S.device));
        const size_t n = size_t(S.nstore) * S.dim;
        if (n) { EGG_CK(cudaMemcpyAsync(S.X(S.cur), S.ckpt.p, n * sizeof(double), cudaMemcpyDeviceToDevice, S.stream)); }
        reset_seeds(S);
        S.sync();
    });
}

int egg_b200_session_autotune(egg_b200_session* s, int32_t objective, int32_t reps, int32_t* chosen)
{
    return guarded([&] {
        if (!s) { invalid("autotune: NULL session"); }
        check_objective(objective);
        Session& S = *s->impl;
        EGG_CK(cudaSetDevice(S.device));
        const int r = reps > 0 ? reps : 3;
        switch (objective) {
        case EGG_B200_OBJ_SHAPE: autotune_impl<kShape>(S, r); break;
        case EGG_B200_OBJ_UNTANGLE: autotune_impl<kUntangle>(S, r); break;
        default: autotune_impl<kShapeSize>(S, r); break;
        }
        if (chosen) { *chosen = S.variant; }
    });
}

int egg_b200_session_set_variant(egg_b200_session* s, int32_t variant)
{
    return guarded([&] {
        if (!s) { invalid("set_variant: NULL session"); }
        if (variant < 0 || variant >= kNumVariants) { invalid("set_variant: variant out of range"); }
        Session& S = *s->impl;
        EGG_CK(cudaSetDevice(S.device));
        S.variant = variant;
        set_tiles(S, S, variant_shape(S, variant));
        S.tuned = true;
        S.pinned_variant = true;
        for (auto& L : S.levels) { L->variant = -1; }
    });
}

int egg_b200_session_variant_info(egg_b200_session* s, int32_t* variant, int32_t* shape, double* times_ms,
                                  int32_t n)
{
    return guarded([&] {
        if (!s) { invalid("variant_info: NULL session"); }
        Session& S = *s->impl;
        if (variant) { *variant = S.variant; }
        for (int v = 0; v < n && v < kNumVariants; ++v) {
            const Variant vs = variant_shape(S, v);
            if (shape) {
                shape[5 * v] = vs.ci;
                shape[5 * v + 1] = vs.cj;
                shape[5 * v + 2] = vs.ck;
                shape[5 * v + 3] = vs.minb;
                shape[5 * v + 4] = vs.fd;
            }
            if (times_ms) { times_ms[v] = S.variant_ms[v]; }
        }
    });
}

int egg_b200_session_launch_count(egg_b200_session* s, int64_t* launches)
{
    return guarded([&] {
        if (!s || !launches) { invalid("launch_count: NULL argument"); }
        *launches = s->impl->launches;
    });
}

int egg_b200_session_stream(egg_b200_session* s, void** stream)
{
    return guarded([&] {
        if (!s || !stream) { invalid("stream: NULL argument"); }
        *stream = static_cast<void*>(s->impl->stream);
    });
}

int egg_b200_session_reset_stats(egg_b200_session* s)
{
    return guarded([&] {
        if (!s) { invalid("reset_stats: NULL session"); }
        s->impl->sync();
        s->impl->launches = 0;
        s->impl->updates = 0;
        for (int k = 0; k < kKCount; ++k) {
            s->impl->k_ms[k] = 0;
            s->impl->k_launch[k] = 0;
        }
    });
}

int egg_b200_metric_eval(int32_t objective, double delta, const double* t, int64_t n, double* mu, double* grad,
                         double* hess)
{
    return guarded([&] {
        check_objective(objective);
        if (n < 0) { invalid("metric_eval: negative n"); }
        if (n == 0) { return; }
        if (!t || !mu || !grad || !hess) { invalid("metric_eval: NULL argument"); }
        DevBuf<double> dt, dm, dg, dh;
        dt.upload(std::vector<double>(t, t + 4 * n));
        dm.alloc(n);
        dg.alloc(4 * n);
        dh.alloc(16 * n);
        metric_eval_kernel<<<unsigned((n + 127) / 128), 128>>>(objective, delta, dt.p, n, dm.p, dg.p, dh.p);
        EGG_CK(cudaGetLastError());
        EGG_CK(cudaMemcpy(mu, dm.p, n * sizeof(double), cudaMemcpyDeviceToHost));
        EGG_CK(cudaMemcpy(grad, dg.p, 4 * n * sizeof(double), cudaMemcpyDeviceToHost));
        EGG_CK(cudaMemcpy(hess, dh.p, 16 * n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int egg_b200_patch_eval(int32_t objective, double delta, const double* X, int64_t n_nodes, int32_t P,
                        const int32_t* gc, const int32_t* gn0, const int32_t* gn1, const double* s0, const double* s1,
                        const double* W_inv, const int32_t* role, double* grad, double* hess, double* energy,
                        double* mindet, double* step)
{
    return guarded([&] {
        check_objective(objective);
        if (P < 0 || n_nodes <= 0) { invalid("patch_eval: bad sizes"); }
        for (int p = 0; p < P; ++p) {
            for (int32_t v : {gc[p], gn0[p], gn1[p]}) {
                if (v < 0 || v >= n_nodes) { invalid("patch_eval: node index out of range"); }
            }
            if (role[p] < -1 || role[p] > 2) { invalid("patch_eval: role out of range"); }
        }
        DevBuf<double> dX, dW, dwt, dout;
        DevBuf<int32_t> dgc, dgn0, dgn1, drole, dslot;
        DevBuf<int64_t> doff;
        DevBuf<int8_t> ds0, ds1;
        dX.upload(std::vector<double>(X, X + 2 * n_nodes));
        dW.upload(std::vector<double>(W_inv, W_inv + 4 * P));
        dwt.upload(std::vector<double>{1.0});
        dgc.upload(std::vector<int32_t>(gc, gc + P));
        dgn0.upload(std::vector<int32_t>(gn0, gn0 + P));
        dgn1.upload(std::vector<int32_t>(gn1, gn1 + P));
        drole.upload(std::vector<int32_t>(role, role + P));
        std::vector<int8_t> a(P), b(P);
        for (int p = 0; p < P; ++p) {
            a[p] = s0[p] < 0 ? -1 : 1;
            b[p] = s1[p] < 0 ? -1 : 1;
        }
        ds0.upload(a);
        ds1.upload(b);
        doff.upload(std::vector<int64_t>{0, P});
        dslot.upload(std::vector<int32_t>{0});
        dout.alloc(10);
        StoredPatch2 sp {1, dslot.p, doff.p, dgc.p, dgn0.p, dgn1.p, ds0.p, ds1.p, drole.p, dW.p, 4, dwt.p, 0};
        switch (objective) {
        case EGG_B200_OBJ_SHAPE: patch_eval_kernel<kShape><<<1, 1>>>(sp, reinterpret_cast<const double2*>(dX.p), delta, dout.p); break;
        case EGG_B200_OBJ_UNTANGLE: patch_eval_kernel<kUntangle><<<1, 1>>>(sp, reinterpret_cast<const double2*>(dX.p), delta, dout.p); break;
        default: patch_eval_kernel<kShapeSize><<<1, 1>>>(sp, reinterpret_cast<const double2*>(dX.p), delta, dout.p); break;
        }
        EGG_CK(cudaGetLastError());
        double o[10];
        EGG_CK(cudaMemcpy(o, dout.p, sizeof(o), cudaMemcpyDeviceToHost));
        grad[0] = o[0];
        grad[1] = o[1];
        for (int k = 0; k < 4; ++k) { hess[k] = o[2 + k]; }
        *energy = o[6];
        *mindet = o[7];
        step[0] = o[8];
        step[1] = o[9];
    });
}

int egg_b200_metric3_probe(int32_t objective, double delta, const double* t, const double* v, int64_t n,
                           double* mu, double* grad9, double* hv)
{
    return guarded([&] {
        check_objective(objective);
        if (n < 0) { invalid("metric3_probe: negative n"); }
        if (n == 0) { return; }
        if (!t || !v || !mu || !grad9 || !hv) { invalid("metric3_probe: NULL argument"); }
        DevBuf<double> dt, dv, dm, dg, dh;
        dt.upload(std::vector<double>(t, t + 9 * n));
        dv.upload(std::vector<double>(v, v + 3 * n));
        dm.alloc(n);
        dg.alloc(9 * n);
        dh.alloc(6 * n);
        metric3_probe_kernel<<<unsigned((n + 127) / 128), 128>>>(objective, delta, dt.p, dv.p, n, dm.p, dg.p, dh.p);
        EGG_CK(cudaGetLastError());
        EGG_CK(cudaMemcpy(mu, dm.p, n * sizeof(double), cudaMemcpyDeviceToHost));
        EGG_CK(cudaMemcpy(grad9, dg.p, 9 * n * sizeof(double), cudaMemcpyDeviceToHost));
        EGG_CK(cudaMemcpy(hv, dh.p, 6 * n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int egg_b200_entity_step(int32_t tag, const double* record, const double* grad, const double* hess,
                         const double* pos, double* step, double* foot)
{
    return guarded([&] {
        if (!record || !grad || !hess || !pos || !step || !foot) { invalid("entity_step: NULL argument"); }
        if (!entity_supported(2, tag)) {
            throw Error(EGG_B200_ENOTSUP, "entity_step: entity tag " + std::to_string(tag) +
                                            " is not supported (the 2D curves LineSeg, Circle, Ellipse, CircleArc, EllipseArc, QuadBezier, "
                                            "CubicBezier and LineRail are)");
        }
        constexpr int R = EGG_B200_ENTITY_FIELDS;
        std::vector<double> in(R + 8);
        std::copy(record, record + R, in.begin());
        std::copy(grad, grad + 2, in.begin() + R);
        std::copy(hess, hess + 4, in.begin() + R + 2);
        std::copy(pos, pos + 2, in.begin() + R + 6);
        DevBuf<double> din, dout;
        din.upload(in);
        dout.alloc(4);
        entity_step_kernel<<<1, 1>>>(tag, din.p, dout.p);
        EGG_CK(cudaGetLastError());
        double o[4];
        EGG_CK(cudaMemcpy(o, dout.p, sizeof(o), cudaMemcpyDeviceToHost));
        step[0] = o[0];
        step[1] = o[1];
        foot[0] = o[2];
        foot[1] = o[3];
    });
}

int egg_b200_entity_frame(int32_t dim, int32_t tag, const double* record, const double* arena, int64_t arena_len,
                          const double* q, int64_t n, double* foot, double* basis)
{
    return guarded([&] {
        if (dim != 2 && dim != 3) { invalid("entity_frame: dim must be 2 or 3"); }
        if (!entity_supported(dim, tag) || tag == EGG_B200_TAG_FREE) {
            invalid("entity_frame: tag " + std::to_string(tag) + " is not a projectable curve/surface entity in dimension " +
                    std::to_string(dim));
        }
        if (!record || n < 0 || (n > 0 && (!q || !foot || !basis)) || arena_len < 0 || (arena_len > 0 && !arena)) {
            invalid("entity_frame: bad arguments");
        }
        const bool segd = tag == EGG_B200_TAG_BSPLINE || tag == EGG_B200_TAG_COMPOSITE ||
                          tag == EGG_B200_TAG_BSPLINESURF;
        if (segd && arena_len == 0) { invalid("entity_frame: a B-spline or composite entity needs its arena"); }
        if (tag == EGG_B200_TAG_BSPLINESURF && !bsurf_record_ok(record, arena, arena_len)) {
            invalid("entity_frame: B-spline surface record outside its arena");
        }
        if (n == 0) { return; }
        const int K = (dim == 3 && (tag == EGG_B200_TAG_PLANE || tag == EGG_B200_TAG_SPHERE ||
                                    tag == EGG_B200_TAG_CYLINDER || tag == EGG_B200_TAG_BSPLINESURF)) ? 2 : 1;
        DevBuf<double> de, da, dq, df, db;
        de.upload(std::vector<double>(record, record + EGG_B200_ENTITY_FIELDS));
        da.upload(arena_len ? std::vector<double>(arena, arena + arena_len) : std::vector<double> {0.0});
        dq.upload(std::vector<double>(q, q + n * dim));
        df.alloc(size_t(n * dim));
        db.alloc(size_t(n * dim * K));
        entity_frame_kernel<<<unsigned((n + 127) / 128), 128>>>(dim, tag, de.p, da.p, dq.p, n, df.p, db.p);
        EGG_CK(cudaGetLastError());
        EGG_CK(cudaMemcpy(foot, df.p, size_t(n * dim) * sizeof(double), cudaMemcpyDeviceToHost));
        EGG_CK(cudaMemcpy(basis, db.p, size_t(n * dim * K) * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int egg_b200_directional_eval(int32_t dim, const double* X, int64_t n_nodes, int64_t n, const int32_t* nodes,
                              const int32_t* kind, const double* ref, const double* weight, double eps,
                              double* energy, double* grad)
{
    return guarded([&] {
        if (dim != 2 && dim != 3) { invalid("directional_eval: dim must be 2 or 3"); }
        if (n < 0 || n_nodes < 0 || (n > 0 && (!X || !nodes || !kind || !ref || !weight)) || !energy ||
            (n_nodes > 0 && !grad)) {
            invalid("directional_eval: bad arguments");
        }
        std::vector<SoftTerm> terms(static_cast<size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            SoftTerm& t = terms[size_t(i)];
            t.kind = kind[i];
            const int ar = soft_arity(t.kind);
            if (ar == 0 || t.kind == kSoftCurv) {
                invalid("directional_eval: unsupported sample kind " + std::to_string(kind[i]));
            }
            for (int m = 0; m < 4; ++m) {
                const int32_t v = nodes[i * 4 + m];
                if (m < ar && (v < 0 || v >= n_nodes)) { invalid("directional_eval: node index out of range"); }
                t.node[m] = m < ar ? v : -1;
            }
            t.slot = 0;
            for (int k = 0; k < 3; ++k) { t.ref[k] = k < dim ? ref[i * dim + k] : 0.0; }
            t.w = weight[i];
        }
        std::fill(grad, grad + n_nodes * dim, 0.0);
        *energy = 0.0;
        if (n == 0) { return; }
        DevBuf<double> dX, de, dg;
        DevBuf<SoftTerm> dt;
        dX.upload(std::vector<double>(X, X + n_nodes * dim));
        dt.upload(terms);
        de.alloc(size_t(n));
        dg.alloc(size_t(n) * 4 * dim);
        const unsigned grid = unsigned((n + 127) / 128);
        if (dim == 2) {
            directional_eval_kernel<2><<<grid, 128>>>(dX.p, dt.p, n, eps, de.p, dg.p);
        } else {
            directional_eval_kernel<3><<<grid, 128>>>(dX.p, dt.p, n, eps, de.p, dg.p);
        }
        EGG_CK(cudaGetLastError());
        std::vector<double> e(static_cast<size_t>(n)), g(static_cast<size_t>(n) * 4 * dim);
        EGG_CK(cudaMemcpy(e.data(), de.p, e.size() * sizeof(double), cudaMemcpyDeviceToHost));
        EGG_CK(cudaMemcpy(g.data(), dg.p, g.size() * sizeof(double), cudaMemcpyDeviceToHost));
        // sums in table order, as the reference's host loop adds them
        double et = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            et += e[size_t(i)];
            const int ar = soft_arity(terms[size_t(i)].kind);
            for (int m = 0; m < ar; ++m) {
                for (int k = 0; k < dim; ++k) {
                    grad[int64_t(terms[size_t(i)].node[m]) * dim + k] += g[(size_t(i) * 4 + m) * dim + k];
                }
            }
        }
        *energy = et;
    });
}

int egg_b200_newton_step(const double* grad, const double* hess, double* step)
{
    return guarded([&] {
        if (!grad || !hess || !step) { invalid("newton_step: NULL argument"); }
        DevBuf<double> dg, dh, ds;
        dg.upload(std::vector<double>(grad, grad + 2));
        dh.upload(std::vector<double>(hess, hess + 4));
        ds.alloc(2);
        newton_step_kernel<<<1, 1>>>(dg.p, dh.p, ds.p);
        EGG_CK(cudaGetLastError());
        EGG_CK(cudaMemcpy(step, ds.p, 2 * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

namespace {
// Buffers handed out (pointer -> size) and idle buffers kept for reuse
// (size -> pointer).  Idle bytes are capped; release frees what would exceed
// the cap, and trim frees every idle buffer.
constexpr int64_t kPinnedIdleCap = int64_t(1) << 30;
constexpr size_t kPinnedIdlePerSize = 2;
struct PinnedPool {
    std::mutex m;
    std::unordered_map<void*, int64_t> out;
    std::unordered_multimap<int64_t, void*> idle;
    int64_t idle_bytes = 0;
};
PinnedPool& pinned_pool()
{
    static PinnedPool* p = new PinnedPool;  // outlives every array that holds a buffer
    return *p;
}
}  // namespace

int egg_b200_pinned_acquire(int64_t bytes, void** out)
{
    return guarded([&] {
        if (!out || bytes <= 0) { invalid("pinned_acquire: bad arguments"); }
        *out = nullptr;
        PinnedPool& P = pinned_pool();
        {
            std::lock_guard<std::mutex> lk(P.m);
            const auto it = P.idle.find(bytes);
            if (it != P.idle.end()) {
                *out = it->second;
                P.idle.erase(it);
                P.idle_bytes -= bytes;
                P.out.emplace(*out, bytes);
                return;
            }
        }
        EGG_CK(cudaHostAlloc(out, size_t(bytes), cudaHostAllocPortable));
        std::lock_guard<std::mutex> lk(P.m);
        P.out.emplace(*out, bytes);
    });
}

int egg_b200_pinned_release(void* p)
{
    return guarded([&] {
        if (!p) { return; }
        PinnedPool& P = pinned_pool();
        {
            std::lock_guard<std::mutex> lk(P.m);
            const auto it = P.out.find(p);
            if (it == P.out.end()) { invalid("pinned_release: pointer did not come from pinned_acquire"); }
            const int64_t bytes = it->second;
            P.out.erase(it);
            if (P.idle.count(bytes) < kPinnedIdlePerSize && P.idle_bytes + bytes <= kPinnedIdleCap) {
                P.idle.emplace(bytes, p);
                P.idle_bytes += bytes;
                return;
            }
        }
        EGG_CK(cudaFreeHost(p));
    });
}

int64_t egg_b200_pinned_trim(void)
{
    std::vector<void*> drop;
    int64_t freed = 0;
    {
        PinnedPool& P = pinned_pool();
        std::lock_guard<std::mutex> lk(P.m);
        for (const auto& kv : P.idle) { drop.push_back(kv.second); }
        freed = P.idle_bytes;
        P.idle.clear();
        P.idle_bytes = 0;
    }
    for (void* p : drop) { cudaFreeHost(p); }
    return freed;
}

}  // extern "C"
