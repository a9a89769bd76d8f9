// sycl.hpp -- the subset of SYCL 2020 that the reference's two kernel
// sources use, executed on host threads.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle).  It exists so that the
// reference's own C++ -- main.cc's compute_naive / is_correct, the nine
// kernels of tsmttsm.hh and the kernels emitted by sycl_codegen*.py -- can be
// compiled in place by g++ and run in this container, where no SYCL
// implementation (AdaptiveCpp) is installed.  Nothing in the library uses it.
//
// Execution model (what AdaptiveCpp's OpenMP backend also does):
//   * parallel_for(range)     : one OpenMP loop over the work-items; such
//                               kernels cannot contain barriers.
//   * parallel_for(nd_range)  : OpenMP over work-groups; inside a group every
//                               work-item is a ucontext fiber.  A barrier
//                               switches back to the group scheduler, which
//                               resumes the fibers round-robin, so every
//                               work-item reaches barrier i before any passes
//                               it.  local_accessor memory is per group.
//   * sub-groups              : fixed size (TSM_HOST_SG_SIZE, default 32) of
//                               consecutive work-items; reduce_over_group sums
//                               the members in lane order between two group
//                               barriers, so it must be reached by the whole
//                               group (true for every caller in the reference).
//   * atomic_ref              : a compare-and-swap loop on the value's bits.
//   * queue                   : in-order and synchronous; submit() runs the
//                               kernel and returns an event carrying its start
//                               and end time in nanoseconds.
#pragma once

#include <ucontext.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <limits>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef TSM_HOST_SG_SIZE
#define TSM_HOST_SG_SIZE 32
#endif

namespace sycl {

// ---------------------------------------------------------------- enums
enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access {
enum class address_space { global_space, local_space, private_space, generic_space };
enum class fence_space { local_space, global_space, global_and_local };
}  // namespace access

// ------------------------------------------------------- properties / info
namespace property {
namespace queue {
struct in_order {};
struct enable_profiling {};
}  // namespace queue
}  // namespace property

class property_list {
 public:
  template <class... P>
  property_list(P...) {}
};

namespace info {
namespace device {
struct vendor { using return_type = std::string; };
struct name { using return_type = std::string; };
struct max_compute_units { using return_type = unsigned; };
}  // namespace device
namespace event_profiling {
struct command_start {};
struct command_end {};
}  // namespace event_profiling
}  // namespace info

class device {
 public:
  template <class Param>
  typename Param::return_type get_info() const {
    if constexpr (std::is_same_v<Param, info::device::vendor>) {
      return "tsm host SYCL subset";
    } else if constexpr (std::is_same_v<Param, info::device::name>) {
      return "host CPU (OpenMP work-items, ucontext work-groups)";
    } else {
#ifdef _OPENMP
      return static_cast<unsigned>(omp_get_max_threads());
#else
      return 1u;
#endif
    }
  }
};

class event {
 public:
  event() = default;
  event(uint64_t t0, uint64_t t1) : t0_(t0), t1_(t1) {}
  void wait() {}
  template <class P>
  uint64_t get_profiling_info() const {
    if constexpr (std::is_same_v<P, info::event_profiling::command_start>)
      return t0_;
    else
      return t1_;
  }

 private:
  uint64_t t0_ = 0, t1_ = 0;
};

// --------------------------------------------------------- ranges / items
template <int D = 1>
class range {
 public:
  range(size_t r0) : r_{r0, 1} {}
  range(size_t r0, size_t r1) : r_{r0, r1} {}
  size_t operator[](int d) const { return r_[d]; }
  size_t get(int d) const { return r_[d]; }
  size_t size() const { return D == 1 ? r_[0] : r_[0] * r_[1]; }

 private:
  size_t r_[2];
};

template <int D = 1>
class nd_range {
 public:
  nd_range(range<D> g, range<D> l) : g_(g), l_(l) {}
  range<D> get_global_range() const { return g_; }
  range<D> get_local_range() const { return l_; }

 private:
  range<D> g_, l_;
};

template <int D = 1>
class item {
 public:
  item(size_t id, size_t r) : id_(id), r_(r) {}
  size_t operator[](int) const { return id_; }
  operator size_t() const { return id_; }
  size_t get_id(int = 0) const { return id_; }
  size_t get_linear_id() const { return id_; }
  size_t get_range(int = 0) const { return r_; }

 private:
  size_t id_, r_;
};

namespace detail {

// One work-group's fibers.  A thread-local pointer lets barrier() find the
// scheduler context of the group the calling fiber belongs to.
struct group_team {
  int n = 0;
  int cur = 0;
  std::vector<ucontext_t> ctx;
  ucontext_t sched;
  std::vector<char*> stacks;
  std::vector<unsigned char> done;
  std::vector<double> scratch;  // reduce_over_group exchange, one per item
  std::vector<unsigned char> local_mem;
  const std::function<void(int)>* body = nullptr;
  static constexpr size_t kStack = 64 * 1024;

  void ensure(int items, size_t local_bytes) {
    while ((int)stacks.size() < items) stacks.push_back(static_cast<char*>(std::malloc(kStack)));
    ctx.resize(items);
    done.assign(items, 0);
    scratch.assign(items, 0.0);
    if (local_mem.size() < local_bytes + 64) local_mem.resize(local_bytes + 64);
    n = items;
  }
  ~group_team() {
    for (char* s : stacks) std::free(s);
  }
};

inline thread_local group_team* tl_team = nullptr;
inline thread_local unsigned char* tl_local_base = nullptr;

inline void yield_to_scheduler() {
  group_team* t = tl_team;
  swapcontext(&t->ctx[t->cur], &t->sched);
}

inline void fiber_entry(unsigned hi, unsigned lo) {
  auto* t = reinterpret_cast<group_team*>((static_cast<uintptr_t>(hi) << 32) |
                                          static_cast<uintptr_t>(lo));
  const int me = t->cur;
  (*t->body)(me);
  t->done[me] = 1;
}

// Runs body(local_id) for every work-item of one group as fibers.
inline void run_group(group_team& t, int items, size_t local_bytes,
                      const std::function<void(int)>& body) {
  t.ensure(items, local_bytes);
  std::memset(t.local_mem.data(), 0, t.local_mem.size());
  tl_local_base = t.local_mem.data();
  t.body = &body;
  const uintptr_t p = reinterpret_cast<uintptr_t>(&t);
  for (int i = 0; i < items; ++i) {
    getcontext(&t.ctx[i]);
    t.ctx[i].uc_stack.ss_sp = t.stacks[i];
    t.ctx[i].uc_stack.ss_size = group_team::kStack;
    t.ctx[i].uc_link = &t.sched;
    makecontext(&t.ctx[i], reinterpret_cast<void (*)()>(&fiber_entry), 2,
                static_cast<unsigned>(p >> 32), static_cast<unsigned>(p & 0xffffffffu));
  }
  group_team* saved = tl_team;
  tl_team = &t;
  int remaining = items;
  while (remaining > 0) {
    for (int i = 0; i < items; ++i) {
      if (t.done[i]) continue;
      t.cur = i;
      swapcontext(&t.sched, &t.ctx[i]);
      if (t.done[i]) --remaining;
    }
  }
  tl_team = saved;
}

inline uint64_t now_ns() {
  return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(
                                   std::chrono::steady_clock::now().time_since_epoch())
                                   .count());
}

}  // namespace detail

template <int D = 1>
class group {
 public:
  explicit group(size_t id) : id_(id) {}
  size_t get_group_id(int = 0) const { return id_; }

 private:
  size_t id_;
};

class sub_group {
 public:
  sub_group(int lid, int local_size) : lid_(lid), local_size_(local_size) {}
  size_t get_local_linear_id() const { return lid_ % TSM_HOST_SG_SIZE; }
  size_t get_local_linear_range() const { return TSM_HOST_SG_SIZE; }
  size_t get_group_linear_range() const { return local_size_ / TSM_HOST_SG_SIZE; }
  size_t get_group_linear_id() const { return lid_ / TSM_HOST_SG_SIZE; }
  int local_id_in_group() const { return lid_; }

 private:
  int lid_, local_size_;
};

template <int D = 1>
class nd_item {
 public:
  nd_item(size_t group, int lid, int local_size, size_t global_size)
      : group_(group), lid_(lid), local_size_(local_size), global_size_(global_size) {}
  size_t get_local_id(int = 0) const { return lid_; }
  size_t get_local_linear_id() const { return lid_; }
  size_t get_group(int) const { return group_; }
  sycl::group<D> get_group() const { return sycl::group<D>(group_); }
  size_t get_group_linear_id() const { return group_; }
  size_t get_global_id(int = 0) const { return group_ * local_size_ + lid_; }
  size_t get_global_linear_id() const { return group_ * local_size_ + lid_; }
  size_t get_local_range(int = 0) const { return local_size_; }
  size_t get_global_range(int = 0) const { return global_size_; }
  size_t get_group_range(int = 0) const { return global_size_ / local_size_; }
  void barrier(access::fence_space = access::fence_space::global_and_local) const {
    detail::yield_to_scheduler();
  }
  sub_group get_sub_group() const {
    if (local_size_ % TSM_HOST_SG_SIZE != 0)
      throw std::runtime_error("host SYCL subset: local size is not a multiple of the sub-group size");
    return sub_group(lid_, local_size_);
  }

 private:
  size_t group_;
  int lid_, local_size_;
  size_t global_size_;
};

template <int D>
inline void group_barrier(const group<D>&) {
  detail::yield_to_scheduler();
}

template <class T = void>
struct plus {
  T operator()(const T& a, const T& b) const { return a + b; }
};

// Whole-sub-group sum in lane order (see the header comment for the
// uniform-call requirement).
template <class T, class Op>
T reduce_over_group(const sub_group& sg, T x, Op op) {
  detail::group_team* t = detail::tl_team;
  const int lid = sg.local_id_in_group();
  t->scratch[lid] = static_cast<double>(x);
  detail::yield_to_scheduler();
  const int base = lid - lid % TSM_HOST_SG_SIZE;
  T acc = static_cast<T>(t->scratch[base]);
  for (int i = 1; i < TSM_HOST_SG_SIZE; ++i) acc = op(acc, static_cast<T>(t->scratch[base + i]));
  detail::yield_to_scheduler();
  return acc;
}

// ------------------------------------------------------------ atomic_ref
template <class T, memory_order O = memory_order::relaxed,
          memory_scope S = memory_scope::device,
          access::address_space A = access::address_space::generic_space>
class atomic_ref {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte atomics only");
  using bits_t = std::conditional_t<sizeof(T) == 8, uint64_t, uint32_t>;

 public:
  explicit atomic_ref(T& ref) : p_(&ref) {}
  T fetch_add(T v) const {
    bits_t old_bits, new_bits;
    __atomic_load(reinterpret_cast<bits_t*>(p_), &old_bits, __ATOMIC_RELAXED);
    T old_v;
    do {
      std::memcpy(&old_v, &old_bits, sizeof(T));
      T nv = old_v + v;
      std::memcpy(&new_bits, &nv, sizeof(T));
    } while (!__atomic_compare_exchange(reinterpret_cast<bits_t*>(p_), &old_bits, &new_bits,
                                        false, __ATOMIC_RELAXED, __ATOMIC_RELAXED));
    return old_v;
  }
  T operator+=(T v) const { return fetch_add(v) + v; }
  T load() const {
    T v;
    bits_t b;
    __atomic_load(reinterpret_cast<bits_t*>(p_), &b, __ATOMIC_RELAXED);
    std::memcpy(&v, &b, sizeof(T));
    return v;
  }

 private:
  T* p_;
};

// ------------------------------------------------------ command group
class handler;

template <class T, int D = 1>
class local_accessor {
 public:
  local_accessor(range<D> r, handler& h);
  decltype(auto) operator[](size_t i) const {
    T* base = reinterpret_cast<T*>(detail::tl_local_base + offset_);
    if constexpr (D == 1)
      return (base[i]);
    else
      return base + i * cols_;
  }

 private:
  size_t offset_ = 0;
  size_t cols_ = 1;
};

class handler {
 public:
  size_t alloc_local(size_t bytes) {
    size_t off = (local_bytes_ + 63) & ~size_t(63);
    local_bytes_ = off + bytes;
    return off;
  }

  template <class F>
  void parallel_for(range<1> r, F f) {
    t0_ = detail::now_ns();
    const long long n = static_cast<long long>(r[0]);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) {
      if constexpr (std::is_invocable_v<F, item<1>>)
        f(item<1>(static_cast<size_t>(i), static_cast<size_t>(n)));
      else
        f(static_cast<size_t>(i));
    }
    t1_ = detail::now_ns();
  }

  template <class F>
  void parallel_for(nd_range<1> r, F f) {
    t0_ = detail::now_ns();
    const size_t global = r.get_global_range()[0];
    const int local = static_cast<int>(r.get_local_range()[0]);
    if (local <= 0 || global % local != 0)
      throw std::runtime_error("host SYCL subset: global size must be a multiple of the local size");
    const long long groups = static_cast<long long>(global / local);
    const size_t lbytes = local_bytes_;
#pragma omp parallel
    {
      detail::group_team team;
#pragma omp for schedule(dynamic, 1)
      for (long long g = 0; g < groups; ++g) {
        std::function<void(int)> body = [&](int lid) {
          f(nd_item<1>(static_cast<size_t>(g), lid, local, global));
        };
        detail::run_group(team, local, lbytes, body);
      }
    }
    t1_ = detail::now_ns();
  }

  uint64_t t0_ = 0, t1_ = 0;

 private:
  size_t local_bytes_ = 0;
};

template <class T, int D>
local_accessor<T, D>::local_accessor(range<D> r, handler& h) {
  offset_ = h.alloc_local(r.size() * sizeof(T));
  cols_ = (D == 2) ? r[1] : 1;
}

// ------------------------------------------------------------------ queue
class queue {
 public:
  queue() = default;
  queue(const property_list&) {}
  device get_device() const { return device{}; }

  template <class CGF>
  event submit(CGF cgf) {
    handler h;
    cgf(h);
    return event(h.t0_, h.t1_);
  }
  template <class T>
  event fill(T* p, const T& v, size_t count) {
    uint64_t t0 = detail::now_ns();
    std::fill(p, p + count, v);
    return event(t0, detail::now_ns());
  }
  event memcpy(void* dst, const void* src, size_t bytes) {
    uint64_t t0 = detail::now_ns();
    std::memcpy(dst, src, bytes);
    return event(t0, detail::now_ns());
  }
  void wait() {}
  void wait_and_throw() {}
};

template <class T>
T* malloc_shared(size_t count, const queue&) {
  return static_cast<T*>(std::aligned_alloc(64, ((count * sizeof(T) + 63) / 64) * 64 + 64));
}
template <class T>
T* malloc_device(size_t count, const queue& q) {
  return malloc_shared<T>(count, q);
}
template <class T>
T* malloc_host(size_t count, const queue& q) {
  return malloc_shared<T>(count, q);
}
inline void free(void* p, const queue&) { std::free(p); }

}  // namespace sycl
