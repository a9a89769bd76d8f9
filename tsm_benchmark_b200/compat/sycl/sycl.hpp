// sycl/sycl.hpp (compat) -- the host-side SYCL surface that the reference's
// drivers use, implemented on the CUDA runtime so that those drivers build
// and run unmodified against libtsm_b200.so.
//
// Covers exactly what main.cc (main.cc:63-69,88,94,114,120-125,152-160),
// main_codegen.cc:5-10 and the generated run_all_benchmarks
// (sycl_codegen_new.py:420-491) call:
//   queue{in_order, enable_profiling}       one CUDA stream (in order) plus a
//                                           zero-filled library workspace
//   get_device().get_info<vendor|name|max_compute_units>
//   malloc_shared / malloc_device / malloc_host / free
//                                           cudaMallocManaged / cudaMalloc /
//                                           cudaMallocHost / matching frees
//   fill, memcpy, wait, wait_and_throw      stream-ordered CUDA calls
//   event::wait, get_profiling_info<command_start|command_end>
//                                           CUDA events; nanoseconds since the
//                                           queue was created
// Kernels are not submitted through this header: the compat tsmttsm.hh and
// the generated tsmttsm_kernels.hh call the C ABI on the queue's stream.
// Errors surface as sycl::exception at the failing call (the reference's
// kernels report nothing until wait_and_throw).
#pragma once

#include <cuda_runtime_api.h>

// Standard headers a SYCL implementation's sycl.hpp brings in transitively
// and the reference's drivers rely on (main.cc uses <random> and <vector>
// through it).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iostream>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "tsm.h"

namespace sycl {

class exception : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

namespace detail {
inline void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw exception(std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace detail

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
  explicit device(int ordinal = 0) : ordinal_(ordinal) {}
  template <class Param>
  typename Param::return_type get_info() const {
    cudaDeviceProp prop;
    detail::check(cudaGetDeviceProperties(&prop, ordinal_), "cudaGetDeviceProperties");
    if constexpr (std::is_same_v<Param, info::device::vendor>)
      return "NVIDIA";
    else if constexpr (std::is_same_v<Param, info::device::name>)
      return prop.name;
    else
      return static_cast<unsigned>(prop.multiProcessorCount);
  }

 private:
  int ordinal_;
};

namespace detail {
struct queue_impl {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t epoch = nullptr;
  void* workspace = nullptr;
  size_t workspace_bytes = 0;
  queue_impl() {
    check(cudaGetDevice(&device), "cudaGetDevice");
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaEventCreate(&epoch), "cudaEventCreate");
    check(cudaEventRecord(epoch, stream), "cudaEventRecord");
  }
  ~queue_impl() {
    cudaStreamSynchronize(stream);
    if (workspace) cudaFree(workspace);
    cudaEventDestroy(epoch);
    cudaStreamDestroy(stream);
  }
  // Library workspace of at least `bytes`, zero-filled when (re)allocated.
  void* ensure_workspace(size_t bytes) {
    if (bytes > workspace_bytes) {
      check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
      if (workspace) check(cudaFree(workspace), "cudaFree");
      check(cudaMalloc(&workspace, bytes), "cudaMalloc(workspace)");
      check(cudaMemsetAsync(workspace, 0, bytes, stream), "cudaMemsetAsync(workspace)");
      workspace_bytes = bytes;
    }
    return workspace;
  }
};

struct event_impl {
  std::shared_ptr<queue_impl> q;
  cudaEvent_t start = nullptr, end = nullptr;
  explicit event_impl(std::shared_ptr<queue_impl> qi) : q(std::move(qi)) {
    check(cudaEventCreate(&start), "cudaEventCreate");
    check(cudaEventCreate(&end), "cudaEventCreate");
  }
  ~event_impl() {
    cudaEventDestroy(start);
    cudaEventDestroy(end);
  }
};
}  // namespace detail

class event {
 public:
  event() = default;
  explicit event(std::shared_ptr<detail::event_impl> e) : e_(std::move(e)) {}
  void wait() {
    if (e_) detail::check(cudaEventSynchronize(e_->end), "cudaEventSynchronize");
  }
  // Nanoseconds since the queue's creation (CUDA event resolution ~0.5 us).
  template <class P>
  uint64_t get_profiling_info() const {
    if (!e_) return 0;
    wait_const();
    float ms = 0.f;
    cudaEvent_t which = std::is_same_v<P, info::event_profiling::command_start> ? e_->start : e_->end;
    detail::check(cudaEventElapsedTime(&ms, e_->q->epoch, which), "cudaEventElapsedTime");
    return static_cast<uint64_t>(static_cast<double>(ms) * 1e6);
  }
  // Library hooks: bracket work enqueued on the queue's stream.
  void record_start() { detail::check(cudaEventRecord(e_->start, e_->q->stream), "cudaEventRecord"); }
  void record_end() { detail::check(cudaEventRecord(e_->end, e_->q->stream), "cudaEventRecord"); }

 private:
  void wait_const() const { detail::check(cudaEventSynchronize(e_->end), "cudaEventSynchronize"); }
  std::shared_ptr<detail::event_impl> e_;
};

class queue {
 public:
  queue() : q_(std::make_shared<detail::queue_impl>()) {}
  queue(const property_list&) : q_(std::make_shared<detail::queue_impl>()) {}
  device get_device() const { return device(q_->device); }

  template <class T>
  event fill(T* p, const T& v, size_t count) {
    event e = begin();
    bool zero = true;
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
    for (size_t i = 0; i < sizeof(T); ++i) zero = zero && b[i] == 0;
    if (zero) {
      detail::check(cudaMemsetAsync(p, 0, count * sizeof(T), q_->stream), "cudaMemsetAsync");
    } else {
      std::vector<T> host(count, v);
      detail::check(cudaMemcpyAsync(p, host.data(), count * sizeof(T), cudaMemcpyDefault, q_->stream),
                    "cudaMemcpyAsync");
      detail::check(cudaStreamSynchronize(q_->stream), "cudaStreamSynchronize");
    }
    e.record_end();
    return e;
  }
  event memcpy(void* dst, const void* src, size_t bytes) {
    event e = begin();
    detail::check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, q_->stream), "cudaMemcpyAsync");
    e.record_end();
    return e;
  }
  void wait() { detail::check(cudaStreamSynchronize(q_->stream), "cudaStreamSynchronize"); }
  void wait_and_throw() { wait(); }

  // ---- library hooks (not SYCL): the stream, the workspace, event pairs.
  cudaStream_t native_stream() const { return q_->stream; }
  void* workspace(size_t bytes) { return q_->ensure_workspace(bytes); }
  size_t workspace_bytes() const { return q_->workspace_bytes; }
  event begin() {
    event e(std::make_shared<detail::event_impl>(q_));
    e.record_start();
    return e;
  }

 private:
  std::shared_ptr<detail::queue_impl> q_;
};

template <class T>
T* malloc_shared(size_t count, const queue&) {
  void* p = nullptr;
  detail::check(cudaMallocManaged(&p, count * sizeof(T)), "cudaMallocManaged");
  return static_cast<T*>(p);
}
template <class T>
T* malloc_device(size_t count, const queue&) {
  void* p = nullptr;
  detail::check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
  return static_cast<T*>(p);
}
template <class T>
T* malloc_host(size_t count, const queue&) {
  void* p = nullptr;
  detail::check(cudaMallocHost(&p, count * sizeof(T)), "cudaMallocHost");
  return static_cast<T*>(p);
}
inline void free(void* p, const queue&) {
  if (!p) return;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost)
    cudaFreeHost(p);
  else
    cudaFree(p);
}

}  // namespace sycl
