// Host-only stand-in for the subset of SYCL 2020 that FastTree's hot-path headers use
// (src/hlbvh.hpp, src/maxheap.hpp, src/sfc.*.hpp).  Written for this project so the
// unmodified reference headers compile with g++ and run on the CPU as a checker.
//
// TEST INFRASTRUCTURE ONLY (oracle/): never part of the CUDA library.
//
// Execution model
//   * range<1> kernels: OpenMP parallel loop over ids.
//   * reductions: sequential fold into the reduction variable.
//   * nd_range<1> kernels: each work-group runs on one OS thread (groups in parallel via
//     OpenMP); its work-items are fibers switched by a minimal x86-64 context switch.
//     group_barrier, group_broadcast and any_of_group suspend the fiber until every
//     work-item of the group arrives, then all resume with the collective's result.
//     A sub-group is the whole work-group (the reference launches groups of exactly the
//     sub-group width).
//   * USM: malloc_shared / malloc_device are host allocations recorded in a registry so
//     get_pointer_type() tells them apart from plain host memory.
//   * The device reports itself as a GPU (is_cpu() == false) so the grouped self-kNN
//     kernels run with the GPU's group width of 32, and 227 KB of local memory per group.
#pragma once

#include <algorithm>
#include <atomic>
#include <bit>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iomanip>
#include <iostream>
#include <tuple>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

namespace sycl {

// ------------------------------------------------------------------------------------------
// ids and ranges
// ------------------------------------------------------------------------------------------
template <int D = 1> struct id {
    size_t v[D > 0 ? D : 1] = {};
    id() = default;
    id(size_t a) { v[0] = a; }
    size_t  operator[](int i) const { return v[i]; }
    size_t &operator[](int i) { return v[i]; }
    operator size_t() const { return v[0]; }
};
template <int D = 1> struct range {
    size_t v[D > 0 ? D : 1] = {};
    range() = default;
    range(size_t a) { v[0] = a; }
    size_t operator[](int i) const { return v[i]; }
    size_t size() const { return v[0]; }
};
template <int D = 1> struct nd_range {
    range<D> g, l;
    nd_range(range<D> global, range<D> local) : g(global), l(local) {}
    range<D> get_global_range() const { return g; }
    range<D> get_local_range() const { return l; }
};

// ------------------------------------------------------------------------------------------
// work-group runtime (fibers)
// ------------------------------------------------------------------------------------------
namespace detail {

extern "C" void ftshim_switch(void **save_sp, void *load_sp);

struct GroupRT;
inline thread_local GroupRT *tl_group = nullptr;
inline thread_local int      tl_lane  = 0;
inline thread_local std::vector<void *> tl_local_base;

struct Fiber {
    void                 *sp   = nullptr;
    std::vector<uint8_t>  stack;
    int                   state = 0; // 0 runnable, 1 waiting, 2 done
    uint64_t              contrib = 0;
};

struct GroupRT {
    int                  L = 0;
    std::vector<Fiber>   fibers;
    void                *sched_sp = nullptr;
    std::function<void(int)> body;
    uint64_t             result   = 0;
    int                  coll_kind = 0; // 1 barrier, 2 broadcast, 3 any_of
    int                  coll_root = 0;
    int                  running   = 0;
};

[[noreturn]] inline void fiber_entry_impl() {
    GroupRT *g    = tl_group;
    int      lane = tl_lane;
    g->body(lane);
    g->fibers[lane].state = 2;
    ftshim_switch(&g->fibers[lane].sp, g->sched_sp);
    std::abort();
}
extern "C" inline void ftshim_fiber_entry() { fiber_entry_impl(); }

inline void init_fiber(Fiber &f, size_t bytes) {
    if (f.stack.size() < bytes) f.stack.assign(bytes, 0);
    uintptr_t top = reinterpret_cast<uintptr_t>(f.stack.data() + f.stack.size());
    top &= ~uintptr_t(15);
    void **sp = reinterpret_cast<void **>(top);
    *--sp     = nullptr;                                         // fake return slot (alignment)
    *--sp     = reinterpret_cast<void *>(&ftshim_fiber_entry);   // ret target
    for (int i = 0; i < 6; ++i) *--sp = nullptr;                 // rbp rbx r12-r15
    f.sp    = sp;
    f.state = 0;
}

// Suspends the calling work-item at a collective; returns the collective's result.
inline uint64_t arrive(int kind, uint64_t contrib, int root = 0) {
    GroupRT *g            = tl_group;
    int      lane         = tl_lane;
    g->fibers[lane].state = 1;
    g->fibers[lane].contrib = contrib;
    g->coll_kind          = kind;
    g->coll_root          = root;
    ftshim_switch(&g->fibers[lane].sp, g->sched_sp);
    tl_lane = lane;
    return g->result;
}

template <class F> void run_group(GroupRT &g, int L, F &&body_fn) {
    g.L = L;
    if ((int)g.fibers.size() < L) g.fibers.resize(L);
    g.body = std::forward<F>(body_fn);
    for (int i = 0; i < L; ++i) init_fiber(g.fibers[i], 256 * 1024);
    tl_group = &g;
    for (;;) {
        bool any_run = false;
        for (int i = 0; i < L; ++i) {
            if (g.fibers[i].state != 0) continue;
            any_run = true;
            tl_lane = i;
            ftshim_switch(&g.sched_sp, g.fibers[i].sp);
        }
        int waiting = 0, done = 0;
        for (int i = 0; i < L; ++i) {
            waiting += g.fibers[i].state == 1;
            done += g.fibers[i].state == 2;
        }
        if (done == L) break;
        if (waiting + done == L) {
            uint64_t r = 0;
            if (g.coll_kind == 2) r = g.fibers[g.coll_root].contrib;
            if (g.coll_kind == 3)
                for (int i = 0; i < L; ++i)
                    if (g.fibers[i].state == 1) r |= g.fibers[i].contrib;
            g.result = r;
            for (int i = 0; i < L; ++i)
                if (g.fibers[i].state == 1) g.fibers[i].state = 0;
        } else if (!any_run) {
            std::abort();
        }
    }
    tl_group = nullptr;
}

// USM registry
enum class Kind { none, shared, device };
inline std::mutex &reg_mutex() {
    static std::mutex m;
    return m;
}
inline std::unordered_map<const void *, Kind> &registry() {
    static std::unordered_map<const void *, Kind> r;
    return r;
}
inline void *usm_alloc(size_t bytes, Kind k) {
    void *p = std::aligned_alloc(64, ((bytes ? bytes : 1) + 63) / 64 * 64);
    std::lock_guard<std::mutex> lk(reg_mutex());
    registry()[p] = k;
    return p;
}

} // namespace detail

// ------------------------------------------------------------------------------------------
// groups and items
// ------------------------------------------------------------------------------------------
struct group {};
struct sub_group {
    id<1> get_local_id() const { return id<1>((size_t)detail::tl_lane); }
    range<1> get_local_range() const { return range<1>((size_t)detail::tl_group->L); }
};
template <int D = 1> struct nd_item {
    size_t g, l, L;
    size_t get_local_id(int) const { return l; }
    size_t get_group(int) const { return g; }
    size_t get_global_id(int) const { return g * L + l; }
    size_t get_local_range(int) const { return L; }
    group  get_group() const { return group{}; }
    sub_group get_sub_group() const { return sub_group{}; }
};

inline void group_barrier(group) { detail::arrive(1, 0); }
inline void group_barrier(sub_group) { detail::arrive(1, 0); }
template <class T> T group_broadcast(group, T v, size_t root) {
    static_assert(sizeof(T) <= 8, "broadcast of <= 8 bytes");
    uint64_t c = 0;
    std::memcpy(&c, &v, sizeof(T));
    uint64_t r = detail::arrive(2, c, (int)root);
    T        out;
    std::memcpy(&out, &r, sizeof(T));
    return out;
}
inline bool any_of_group(sub_group, bool pred) { return detail::arrive(3, pred ? 1u : 0u) != 0; }
inline bool any_of_group(group, bool pred) { return detail::arrive(3, pred ? 1u : 0u) != 0; }

// ------------------------------------------------------------------------------------------
// math / bit helpers
// ------------------------------------------------------------------------------------------
template <class To, class From> To bit_cast(const From &f) { return std::bit_cast<To>(f); }
inline uint32_t clz(uint32_t x) { return x ? (uint32_t)__builtin_clz(x) : 32u; }
inline uint64_t clz(uint64_t x) { return x ? (uint64_t)__builtin_clzll(x) : 64u; }
inline int      clz(int x) { return x ? __builtin_clz((unsigned)x) : 32; }
inline float    fmin(float a, float b) { return std::fmin(a, b); }
inline double   fmin(double a, double b) { return std::fmin(a, b); }
inline float    fmax(float a, float b) { return std::fmax(a, b); }
inline double   fmax(double a, double b) { return std::fmax(a, b); }
inline float    clamp(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
inline double   clamp(double x, double lo, double hi) { return std::fmin(std::fmax(x, lo), hi); }
template <class T> T min(T a, T b) { return b < a ? b : a; }
template <class T> T max(T a, T b) { return a < b ? b : a; }

template <class T = void> struct minimum {
    T operator()(const T &a, const T &b) const { return (a < b) ? a : b; }
};
template <class T = void> struct maximum {
    T operator()(const T &a, const T &b) const { return (a < b) ? b : a; }
};

// ------------------------------------------------------------------------------------------
// atomics
// ------------------------------------------------------------------------------------------
enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access {
enum class address_space { global_space, local_space, generic_space };
enum class target { device, local };
} // namespace access
template <class T, memory_order O, memory_scope S, access::address_space A = access::address_space::generic_space>
struct atomic_ref {
    std::atomic_ref<T> r;
    explicit atomic_ref(T &x) : r(x) {}
    T fetch_add(T v) { return r.fetch_add(v, std::memory_order_seq_cst); }
    T load() const { return r.load(std::memory_order_seq_cst); }
    void store(T v) { r.store(v, std::memory_order_seq_cst); }
};
inline void atomic_fence(memory_order, memory_scope) { std::atomic_thread_fence(std::memory_order_seq_cst); }

// ------------------------------------------------------------------------------------------
// device / context / queue
// ------------------------------------------------------------------------------------------
namespace info {
namespace device {
struct local_mem_size { using return_type = size_t; };
struct native_vector_width_double { using return_type = uint32_t; };
struct native_vector_width_float { using return_type = uint32_t; };
struct native_vector_width_long { using return_type = uint32_t; };
struct native_vector_width_int { using return_type = uint32_t; };
struct name { using return_type = std::string; };
struct sub_group_sizes { using return_type = std::vector<size_t>; };
struct global_mem_size { using return_type = size_t; };
} // namespace device
} // namespace info

struct device {
    bool is_cpu() const { return false; }
    bool is_gpu() const { return true; }
    template <class P> typename P::return_type get_info() const {
        if constexpr (std::is_same_v<P, info::device::local_mem_size>) return 227 * 1024;
        else if constexpr (std::is_same_v<P, info::device::name>) return std::string("host shim (fibers)");
        else if constexpr (std::is_same_v<P, info::device::sub_group_sizes>) return std::vector<size_t>{32};
        else if constexpr (std::is_same_v<P, info::device::global_mem_size>) return (size_t)64 << 30;
        else return 32;
    }
};
struct context {};
namespace usm {
enum class alloc { host, device, shared, unknown };
}
inline usm::alloc get_pointer_type(const void *p, const context &) {
    std::lock_guard<std::mutex> lk(detail::reg_mutex());
    auto it = detail::registry().find(p);
    if (it == detail::registry().end()) return usm::alloc::unknown;
    return it->second == detail::Kind::device ? usm::alloc::device : usm::alloc::shared;
}

struct event {
    void wait() {}
};

namespace property {
namespace queue {
struct in_order {};
} // namespace queue
} // namespace property
struct property_list {
    template <class... P> property_list(P...) {}
};
struct default_selector_t {};
struct cpu_selector_t {};
inline constexpr default_selector_t default_selector_v{};
inline constexpr cpu_selector_t     cpu_selector_v{};

template <class T, class Op> struct reduction_t {
    T *ptr;
    T  identity;
    Op op;
};
template <class T, class Op> reduction_t<T, Op> reduction(T *p, T identity, Op op) { return {p, identity, op}; }
template <class T, class Op> struct reducer {
    T  v;
    Op op;
    void combine(const T &x) { v = op(v, x); }
};

template <class T, int D = 1> class local_accessor;

class handler {
  public:
    std::vector<std::pair<size_t, size_t>> locals; // (bytes, align)
    int register_local(size_t bytes, size_t align) {
        locals.push_back({bytes, align});
        return (int)locals.size() - 1;
    }

    template <class F> void single_task(F f) { f(); }

    template <class F> void parallel_for(range<1> r, F f) {
        const long long n = (long long)r[0];
#pragma omp parallel for schedule(dynamic, 1024)
        for (long long i = 0; i < n; ++i) f(id<1>((size_t)i));
    }

    // range kernel with reductions: parallel_for(range, red_1, ..., red_m, kernel)
    template <class A, class B, class... Rest> void parallel_for(range<1> r, A a, B b, Rest... rest) {
        auto t = std::make_tuple(a, b, rest...);
        red_dispatch(r, t, std::make_index_sequence<sizeof...(Rest) + 1>{});
    }

    template <class F> void parallel_for(nd_range<1> ndr, F f) {
        const size_t L  = ndr.get_local_range()[0];
        const size_t G  = ndr.get_global_range()[0] / (L ? L : 1);
        auto         locals_copy = locals;
#pragma omp parallel
        {
            detail::GroupRT g;
            std::vector<std::vector<uint8_t>> mem(locals_copy.size());
#pragma omp for schedule(dynamic, 1)
            for (long long gi = 0; gi < (long long)G; ++gi) {
                detail::tl_local_base.assign(locals_copy.size(), nullptr);
                for (size_t a = 0; a < locals_copy.size(); ++a) {
                    mem[a].assign(locals_copy[a].first + 64, 0);
                    uintptr_t b = reinterpret_cast<uintptr_t>(mem[a].data());
                    b           = (b + 63) & ~uintptr_t(63);
                    detail::tl_local_base[a] = reinterpret_cast<void *>(b);
                }
                size_t grp = (size_t)gi;
                detail::run_group(g, (int)L, [&f, grp, L](int lane) {
                    nd_item<1> it{grp, (size_t)lane, L};
                    f(it);
                });
            }
        }
    }

  private:
    template <class Tup, size_t... I> void red_dispatch(range<1> r, Tup &t, std::index_sequence<I...>) {
        auto &kernel = std::get<sizeof...(I)>(t);
        auto  reds   = std::make_tuple(make_reducer(std::get<I>(t))...);
        for (size_t i = 0; i < r[0]; ++i) kernel(id<1>(i), std::get<I>(reds)...);
        (finish(std::get<I>(t), std::get<I>(reds)), ...);
    }
    template <class T, class Op> static reducer<T, Op> make_reducer(reduction_t<T, Op> &rd) {
        return reducer<T, Op>{*rd.ptr, rd.op};
    }
    template <class T, class Op> static void finish(reduction_t<T, Op> &rd, reducer<T, Op> &r) { *rd.ptr = r.v; }
};

template <class T, int D> class local_accessor {
  public:
    int idx = -1;
    local_accessor() = default;
    local_accessor(range<1> r, handler &h) : idx(h.register_local(r[0] * sizeof(T), alignof(T))) {}
    local_accessor(size_t n, handler &h) : idx(h.register_local(n * sizeof(T), alignof(T))) {}
    T &operator[](size_t i) const { return reinterpret_cast<T *>(detail::tl_local_base[idx])[i]; }
};

class queue {
  public:
    queue() = default;
    template <class A> explicit queue(const A &) {}
    template <class A, class B> queue(const A &, const B &) {}
    device  get_device() const { return device{}; }
    context get_context() const { return context{}; }

    template <class F> event submit(F f) {
        handler h;
        f(h);
        return {};
    }
    template <class F> event single_task(F f) {
        f();
        return {};
    }
    template <class F> event parallel_for(range<1> r, F f) {
        handler h;
        h.parallel_for(r, f);
        return {};
    }
    template <class T> event fill(T *p, const T &v, size_t n) {
        for (size_t i = 0; i < n; ++i) p[i] = v;
        return {};
    }
    template <class T, class U> event fill(T *p, const U &v, size_t n) {
        for (size_t i = 0; i < n; ++i) p[i] = (T)v;
        return {};
    }
    template <class T> event copy(const T *src, T *dst, size_t n) {
        if (n) std::memcpy((void *)dst, (const void *)src, n * sizeof(T));
        return {};
    }
    event memcpy(void *dst, const void *src, size_t bytes) {
        if (bytes) std::memcpy(dst, src, bytes);
        return {};
    }
    void wait() {}
};

template <class T> T *malloc_shared(size_t n, const queue &) {
    return static_cast<T *>(detail::usm_alloc(n * sizeof(T), detail::Kind::shared));
}
template <class T> T *malloc_device(size_t n, const queue &) {
    return static_cast<T *>(detail::usm_alloc(n * sizeof(T), detail::Kind::device));
}
inline void free(void *p, const queue &) {
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(detail::reg_mutex());
        detail::registry().erase(p);
    }
    std::free(p);
}

} // namespace sycl
