// Host-only stand-in for the small subset of the SYCL 2020 API that the egg
// reference core uses, so that its unmodified sources compile with plain g++
// and OpenMP into a CPU oracle.  This is test infrastructure: it exists only to
// build the reference as the parity checker and the timed CPU baseline.
//
// Semantics kept from SYCL:
//   * queue::parallel_for(range<1>, f(id<1>))         -> OpenMP static loop
//     (with EGG_SHIM_SNAPSHOT: serial, last item first -- see parallel_for)
//   * queue::parallel_for(range<1>, red..., f(id, r&...)) -> serial loop with
//     reducers (deterministic order; the reference does not rely on any
//     particular reduction order)
//   * memcpy / memset / fill / wait on host memory (USM device == host here)
//   * reduction(ptr, identity, op, initialize_to_identity) and the accumulating
//     two-argument reduction(ptr, op)
#pragma once

#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <functional>
#include <limits>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>

namespace sycl
{

class exception : public std::runtime_error
{
  public:
    using std::runtime_error::runtime_error;
};

template <int N = 1> struct id {
    std::size_t v[N > 0 ? N : 1] {};
    id() = default;
    id(std::size_t i) { v[0] = i; }  // NOLINT(google-explicit-constructor)
    std::size_t operator[](int k) const { return v[k]; }
    operator std::size_t() const { return v[0]; }  // NOLINT(google-explicit-constructor)
};

template <int N = 1> struct range {
    std::size_t v[N > 0 ? N : 1] {};
    explicit range(std::size_t n) { v[0] = n; }
    std::size_t operator[](int k) const { return v[k]; }
    std::size_t size() const { return v[0]; }
};

struct event {
    void wait() {}
    static void wait(const std::initializer_list<event>&) {}
};

// ---- selectors, properties ---------------------------------------------------
struct cpu_selector_t {};
struct gpu_selector_t {};
inline constexpr cpu_selector_t cpu_selector_v {};
inline constexpr gpu_selector_t gpu_selector_v {};

namespace property
{
namespace queue
{
struct in_order {};
struct AdaptiveCpp_coarse_grained_events {};
}  // namespace queue
namespace reduction
{
struct initialize_to_identity {};
}  // namespace reduction
}  // namespace property

// Accepts (and ignores) any braced list of property tags.
struct property_list {
    property_list() = default;
    template <class... P> property_list(P...) {}  // NOLINT(google-explicit-constructor)
};

struct context {};
struct device {};

// ---- reductions --------------------------------------------------------------
template <class T> struct minimum {
    T operator()(const T& a, const T& b) const { return b < a ? b : a; }
};
template <class T> struct maximum {
    T operator()(const T& a, const T& b) const { return a < b ? b : a; }
};

template <class T, class Op> struct reduction_desc {
    T* out;
    T identity;
    Op op;
    bool init_to_identity;
};

template <class T, class Op>
reduction_desc<T, Op> reduction(T* out, T identity, Op op, property::reduction::initialize_to_identity)
{ return {out, identity, op, true}; }

// Without initialize_to_identity the result is combined with the value *out
// holds when the kernel runs.
template <class T, class Op> reduction_desc<T, Op> reduction(T* out, T identity, Op op)
{ return {out, identity, op, false}; }

template <class T, class Op> reduction_desc<T, Op> reduction(T* out, Op op)
{ return {out, T {}, op, false}; }

template <class T, class Op> struct reducer {
    T acc;
    Op op;
    void combine(const T& x) { acc = op(acc, x); }
    reducer& operator+=(const T& x)
    {
        combine(x);
        return *this;
    }
};

// ---- atomics (host) ----------------------------------------------------------
enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access
{
enum class address_space { global_space, local_space, private_space, generic_space };
}

template <class T, memory_order O = memory_order::relaxed, memory_scope S = memory_scope::device,
          access::address_space A = access::address_space::global_space>
class atomic_ref
{
  public:
    explicit atomic_ref(T& r) : ref_(r) {}
    T fetch_add(T v) const
    {
        T old;
#pragma omp atomic capture
        {
            old = ref_;
            ref_ += v;
        }
        return old;
    }
    T load() const { return ref_; }

  private:
    T& ref_;
};

// ---- queue -------------------------------------------------------------------
class queue
{
  public:
    queue() = default;
    queue(const property_list&) {}  // NOLINT(google-explicit-constructor)
    queue(cpu_selector_t, const property_list& = {}) {}
    queue(gpu_selector_t, const property_list& = {})
    { throw exception("host oracle build: no GPU device"); }
    queue(const context&, const device&, const property_list& = {}) {}

    context get_context() const { return {}; }
    device get_device() const { return {}; }

    event memcpy(void* dst, const void* src, std::size_t bytes)
    {
        if (bytes) { std::memmove(dst, src, bytes); }
        return {};
    }
    event memset(void* dst, int v, std::size_t bytes)
    {
        if (bytes) { std::memset(dst, v, bytes); }
        return {};
    }
    template <class T> event fill(T* dst, const T& v, std::size_t n)
    {
        for (std::size_t i = 0; i < n; ++i) { dst[i] = v; }
        return {};
    }
    void wait() {}

    template <class F> event parallel_for(range<1> r, F&& f)
    {
        const long long n = static_cast<long long>(r[0]);
#ifdef EGG_SHIM_SNAPSHOT
        // Serial, last item first.  The reference's fused ghost-fill +
        // shared-node broadcast launch (src/structured_halo.hpp:215-236) puts
        // the ghost copies first and the owner -> copy refreshes last; when a
        // ghost's source is itself a non-owner copy, a parallel run races and
        // its result depends on the thread count.  Running the refreshes
        // before the ghost fills gives every ghost the refreshed value: the
        // race-free snapshot that the launch's own comment describes.  Every
        // other kernel writes disjoint slots, so its order does not matter.
        for (long long i = n - 1; i >= 0; --i) { f(id<1>(static_cast<std::size_t>(i))); }
#else
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < n; ++i) { f(id<1>(static_cast<std::size_t>(i))); }
#endif
        return {};
    }

    template <class A0, class A1, class... Rest> event parallel_for(range<1> r, A0&& a0, A1&& a1, Rest&&... rest)
    {
        run_reduced(r, std::forward_as_tuple(a0, a1, rest...),
                    std::make_index_sequence<2 + sizeof...(Rest) - 1> {});
        return {};
    }

  private:
    template <class Tup, std::size_t... I>
    void run_reduced(range<1> r, Tup&& args, std::index_sequence<I...>)
    {
        constexpr std::size_t kN = sizeof...(I);
        auto& kernel = std::get<kN>(args);
        auto reducers = std::make_tuple(make_reducer(std::get<I>(args))...);
        for (std::size_t i = 0; i < r[0]; ++i) { kernel(id<1>(i), std::get<I>(reducers)...); }
        (finish(std::get<I>(args), std::get<I>(reducers)), ...);
    }
    template <class T, class Op> static reducer<T, Op> make_reducer(const reduction_desc<T, Op>& d)
    { return {d.init_to_identity ? d.identity : *d.out, d.op}; }
    template <class T, class Op> static void finish(const reduction_desc<T, Op>& d, const reducer<T, Op>& r)
    { *d.out = r.acc; }
};

template <class T> T* malloc_device(std::size_t n, const queue&)
{
    if (n == 0) { return nullptr; }
    void* p = std::aligned_alloc(64, ((n * sizeof(T) + 63) / 64) * 64);
    if (!p) { throw exception("malloc_device: out of host memory"); }
    return static_cast<T*>(p);
}
inline void free(void* p, const queue&) { std::free(p); }

// ---- math --------------------------------------------------------------------
using std::acos;
using std::asin;
using std::atan;
using std::atan2;
using std::cos;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::fmod;
using std::isfinite;
using std::pow;
using std::remainder;
using std::sin;
using std::sqrt;

}  // namespace sycl
