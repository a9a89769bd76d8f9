// tsm_compat_bench.hh -- the benchmark harness behind the generated
// run_all_benchmarks<T>(q, K, warmup, runs) (compat/tsmttsm_kernels.hh),
// the entry main_codegen.cc:10 calls.
//
// Same procedure and table as the reference's generated harness
// (sycl_codegen_new.py:417-521): per width M, allocate device A, B, C, check
// each kernel against an FP64 host product, then `warmup` untimed and `runs`
// timed calls with C zeroed before each, timed by event profiling (kernel
// only).  Three differences, all fixes of the reference's harness:
// the inputs come from the library's seeded generator instead of unseeded
// rand() (sycl_codegen_new.py:436-439); the check covers all K rows, not
// the first 1024 (:443); and the table adds GB/s.
#pragma once

#include <sycl/sycl.hpp>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <iomanip>
#include <iostream>
#include <numeric>
#include <string>
#include <vector>

#include "tsm.h"

namespace tsm_compat {

struct BenchResult {
  std::string name;
  bool correct;
  double avg_ms, min_ms, stddev_ms, gflops, gbs;
};

// Element rule of the reference's generated checks: abs 1e-4 with rel 1e-6
// (sycl_codegen_new.py:402-415) or rel 1e-8 (sycl_codegen.py:305-316).
inline bool check(const std::vector<double>& ref, const double* got, int M, double abs_tol = 1e-4,
                  double rel_tol = 1e-6) {
  for (int i = 0; i < M * M; ++i) {
    const double diff = std::abs(ref[i] - got[i]);
    const double mag = std::max(std::abs(ref[i]), std::abs(got[i]));
    if (!(diff <= abs_tol) && !(diff <= rel_tol * mag)) {
      std::cerr << "Mismatch at " << i << ": ref=" << ref[i] << " got=" << got[i] << " diff=" << diff << "\n";
      return false;
    }
  }
  return true;
}

// One width's inputs, the host-side FP64 product and the timing loop.
template <class T>
struct Problem {
  sycl::queue& q;
  int K, M;
  double rel_tol;
  T *A = nullptr, *B = nullptr, *C = nullptr;
  std::vector<T> ref;
  std::vector<T> host_c;

  Problem(sycl::queue& q_, int K_, int M_, uint64_t seed = 123, double rel_tol_ = 1e-6)
      : q(q_), K(K_), M(M_), rel_tol(rel_tol_), host_c(size_t(M_) * M_) {
    A = sycl::malloc_device<T>(size_t(K) * M, q);
    B = sycl::malloc_device<T>(size_t(K) * M, q);
    C = sycl::malloc_device<T>(size_t(M) * M, q);
    if (tsm_fill_uniform_f64(q.native_stream(), A, int64_t(K) * M, seed, 0) != TSM_SUCCESS ||
        tsm_fill_uniform_f64(q.native_stream(), B, int64_t(K) * M, seed, 1) != TSM_SUCCESS)
      throw sycl::exception("tsm_fill_uniform_f64 failed");
    std::vector<T> ha(size_t(K) * M), hb(size_t(K) * M);
    q.memcpy(ha.data(), A, ha.size() * sizeof(T)).wait();
    q.memcpy(hb.data(), B, hb.size() * sizeof(T)).wait();
    ref.assign(size_t(M) * M, T(0));
    for (int m = 0; m < M; ++m)
      for (int n = 0; n < M; ++n) {
        T acc = 0;
        for (int64_t k = 0; k < K; ++k) acc += ha[k * M + m] * hb[k * M + n];
        ref[size_t(m) * M + n] = acc;
      }
  }
  ~Problem() {
    sycl::free(A, q);
    sycl::free(B, q);
    sycl::free(C, q);
  }

  template <class F>
  BenchResult bench(const std::string& label, F kernel_fn, int warmup, int runs) {
    q.fill(C, T(0), size_t(M) * M).wait();
    kernel_fn(K).wait();
    q.memcpy(host_c.data(), C, host_c.size() * sizeof(T)).wait();
    if (!check(ref, host_c.data(), M, 1e-4, rel_tol)) return {label, false, 0, 0, 0, 0, 0};
    for (int i = 0; i < warmup; ++i) {
      q.fill(C, T(0), size_t(M) * M).wait();
      kernel_fn(K).wait();
    }
    std::vector<double> times(runs);
    for (int i = 0; i < runs; ++i) {
      q.fill(C, T(0), size_t(M) * M).wait();
      auto ev = kernel_fn(K);
      ev.wait();
      auto t0 = ev.template get_profiling_info<sycl::info::event_profiling::command_start>();
      auto t1 = ev.template get_profiling_info<sycl::info::event_profiling::command_end>();
      times[i] = (t1 - t0) * 1e-6;
    }
    const double avg = std::accumulate(times.begin(), times.end(), 0.0) / runs;
    const double mn = *std::min_element(times.begin(), times.end());
    const double sq = std::inner_product(times.begin(), times.end(), times.begin(), 0.0);
    const double sd = std::sqrt(std::max(0.0, sq / runs - avg * avg));
    const double flops = 2.0 * K * double(M) * M;
    const double bytes = double(sizeof(T)) * (2.0 * K * M + double(M) * M);
    return {label, true, avg, mn, sd, flops / (avg * 1e-3) / 1e9, bytes / (avg * 1e-3) / 1e9};
  }
};

inline void print_results(const std::vector<BenchResult>& results) {
  const int W = 122;
  std::cout << "\n" << std::string(W, '=') << "\n";
  std::cout << "BENCHMARK RESULTS\n";
  std::cout << std::string(W, '=') << "\n\n";
  std::cout << std::setw(22) << "Kernel" << std::setw(10) << "Correct" << std::setw(12) << "Avg (ms)" << std::setw(12)
            << "Min (ms)" << std::setw(12) << "Stddev" << std::setw(12) << "GFLOP/s" << std::setw(12) << "GB/s"
            << "\n";
  std::cout << std::string(W, '-') << "\n";
  for (const auto& r : results) {
    std::cout << std::setw(22) << r.name << std::setw(10) << (r.correct ? "PASS" : "FAIL") << std::fixed
              << std::setprecision(4);
    if (r.correct)
      std::cout << std::setw(12) << r.avg_ms << std::setw(12) << r.min_ms << std::setw(12) << r.stddev_ms
                << std::setprecision(2) << std::setw(12) << r.gflops << std::setw(12) << r.gbs;
    std::cout << "\n";
  }
  std::cout << std::string(W, '=') << "\n";
}

}  // namespace tsm_compat
