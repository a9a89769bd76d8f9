// ref_harness.cc -- runs the reference's own C++ on the host, for pinning the
// oracle.  TEST INFRASTRUCTURE ONLY.
//
// The reference sources are compiled IN PLACE (their path is passed on the
// command line by oracle/Makefile; nothing is copied into this repository):
//   * main.cc            -- compute_naive (main.cc:14-27), is_correct
//                           (main.cc:29-41) and, through its #include,
//                           the nine kernels of tsmttsm.hh:15-586;
//   * the output of sycl_codegen_new.py / sycl_codegen.py, generated into
//     oracle/_ref/ by the same recipe.
// <sycl/sycl.hpp> resolves to oracle/sycl_host/, a host-thread subset of
// SYCL 2020.  main.cc's own main() is renamed and never called.
//
// Everything is exported as extern "C" for ctypes (tests/ and the CPU
// baseline of bench.py).  Widths and launch shapes are template parameters
// in the reference, so each callable configuration is instantiated below.
#include <sycl/sycl.hpp>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <numeric>
#include <random>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define main tsm_reference_main_not_called
#include REF_MAIN_CC
#undef main

#ifdef REF_GEN_V2
#include REF_GEN_V2
#endif
#ifdef REF_GEN_V1
#include REF_GEN_V1
#endif

namespace {

// Work decompositions the reference cannot run (a zero row stride would loop
// forever, a non-divisible stride double-counts rows) are refused here, the
// way the reference's own drivers only ever instantiate safe shapes.
template <int V, int M, int S, int L, int T>
constexpr bool valid_config() {
  constexpr int tile = T < M ? T : M;
  if ((M * M) % (tile * tile) != 0) return false;
  constexpr int tiles = (M * M) / (tile * tile);
  if constexpr (V == 1 || V == 8) return true;
  if constexpr (V == 6 || V == 9) {
    if (S % L != 0) return false;
    constexpr int groups = S / L;
    return groups % tiles == 0 && groups >= tiles;
  }
  return S % tiles == 0 && S >= tiles;
}

using variant_fn = int (*)(int, double*, double*, double*, uint64_t*);

template <int V, int M, int S, int L, int T>
int run_variant(int K, double* A, double* B, double* C, uint64_t* ns) {
  if constexpr (!valid_config<V, M, S, L, T>()) {
    return -2;
  } else {
    sycl::queue q{{sycl::property::queue::in_order{}, sycl::property::queue::enable_profiling{}}};
    sycl::event e;
    if constexpr (V == 1) e = tsmttsm<double, M, S>(q, K, A, B, C);
    if constexpr (V == 2) e = tsmttsm2<double, M, S, T>(q, K, A, B, C);
    if constexpr (V == 3) e = tsmttsm3<double, M, S, T>(q, K, A, B, C);
    if constexpr (V == 4) e = tsmttsm4<double, M, S, T>(q, K, A, B, C);
    if constexpr (V == 5) e = tsmttsm5<double, M, S, T>(q, K, A, B, C);
    if constexpr (V == 6) e = tsmttsm6<double, M, S, L, T>(q, K, A, B, C);
    if constexpr (V == 7) e = tsmttsm7<double, M, S, T>(q, K, A, B, C);
    if constexpr (V == 8) e = tsmttsm8<double, M>(q, K, A, B, C);
    if constexpr (V == 9) e = tsmttsm9<double, M, S, L, T>(q, K, A, B, C);
    e.wait();
    if (ns)
      *ns = e.get_profiling_info<sycl::info::event_profiling::command_end>() -
            e.get_profiling_info<sycl::info::event_profiling::command_start>();
    return 0;
  }
}

struct variant_entry {
  int v, m, s, l, t;
  variant_fn fn;
};

#define TSM_E(V, M, S, T) {V, M, S, 32, T, &run_variant<V, M, S, 32, T>}
#define TSM_TILES(V, M, S) TSM_E(V, M, S, 2), TSM_E(V, M, S, 4)
#define TSM_STRIDES(V, M) \
  TSM_TILES(V, M, 4096), TSM_TILES(V, M, 8192), TSM_TILES(V, M, 16384), TSM_TILES(V, M, 32768)
#define TSM_WIDTHS(V) \
  TSM_STRIDES(V, 1), TSM_STRIDES(V, 2), TSM_STRIDES(V, 4), TSM_STRIDES(V, 8), TSM_STRIDES(V, 16), TSM_STRIDES(V, 32)

const variant_entry kVariants[] = {
    TSM_WIDTHS(1), TSM_WIDTHS(2), TSM_WIDTHS(3), TSM_WIDTHS(4), TSM_WIDTHS(5),
    TSM_WIDTHS(6), TSM_WIDTHS(7), TSM_WIDTHS(8), TSM_WIDTHS(9),
};

using gen_fn = sycl::event (*)(sycl::queue&, int, const double*, const double*, double*);
using gen_fn_v1 = sycl::event (*)(sycl::queue&, int, double*, double*, double*);

struct gen_entry {
  const char* name;
  gen_fn fn;
};
struct gen_entry_v1 {
  const char* name;
  gen_fn_v1 fn;
};

const gen_entry kGenV2[] = {
#ifdef REF_GEN_V2_TABLE
#include REF_GEN_V2_TABLE
#endif
    {nullptr, nullptr}};

const gen_entry_v1 kGenV1[] = {
#ifdef REF_GEN_V1_TABLE
#include REF_GEN_V1_TABLE
#endif
    {nullptr, nullptr}};

}  // namespace

extern "C" {

// compute_naive<double>(K, M, A, B) of main.cc:14-27; C receives M*M values.
__attribute__((visibility("default"))) int ref_compute_naive_f64(int K, int M, const double* A,
                                                                 const double* B, double* C) {
  std::vector<double> c = compute_naive<double>(K, M, const_cast<double*>(A), const_cast<double*>(B));
  std::memcpy(C, c.data(), sizeof(double) * c.size());
  return 0;
}

// is_correct<double>(C_correct, C, M, rel_tol, abs_tol) of main.cc:29-41.
__attribute__((visibility("default"))) int ref_is_correct_f64(const double* C_correct, const double* C,
                                                              int M, double rel_tol, double abs_tol) {
  std::vector<double> ref(C_correct, C_correct + static_cast<size_t>(M) * M);
  return is_correct<double>(ref, const_cast<double*>(C), M, rel_tol, abs_tol) ? 1 : 0;
}

// tsmttsm{,2..9}<double, M, stride[, local_size=32], tile> of tsmttsm.hh, run
// on host threads.  Accumulates into C.  Returns 0, -1 (not instantiated) or
// -2 (a launch shape the reference cannot run).  *ns = kernel time.
__attribute__((visibility("default"))) int ref_tsmttsm_f64(int variant, int M, int stride, int tile, int K,
                                                           const double* A, const double* B, double* C,
                                                           uint64_t* ns) {
  for (const auto& e : kVariants)
    if (e.v == variant && e.m == M && e.s == stride && e.t == tile)
      return e.fn(K, const_cast<double*>(A), const_cast<double*>(B), C, ns);
  return -1;
}

// One kernel emitted by sycl_codegen_new.py (v2) or sycl_codegen.py (v1), by
// its generated name.  Accumulates into C.  Returns 0 or -1 (unknown name).
__attribute__((visibility("default"))) int ref_generated_f64(const char* name, int K, const double* A,
                                                             const double* B, double* C, uint64_t* ns) {
  sycl::queue q{{sycl::property::queue::in_order{}, sycl::property::queue::enable_profiling{}}};
  for (const gen_entry* e = kGenV2; e->name; ++e)
    if (std::strcmp(e->name, name) == 0) {
      sycl::event ev = e->fn(q, K, A, B, C);
      if (ns)
        *ns = ev.get_profiling_info<sycl::info::event_profiling::command_end>() -
              ev.get_profiling_info<sycl::info::event_profiling::command_start>();
      return 0;
    }
  for (const gen_entry_v1* e = kGenV1; e->name; ++e)
    if (std::strcmp(e->name, name) == 0) {
      sycl::event ev = e->fn(q, K, const_cast<double*>(A), const_cast<double*>(B), C);
      if (ns)
        *ns = ev.get_profiling_info<sycl::info::event_profiling::command_end>() -
              ev.get_profiling_info<sycl::info::event_profiling::command_start>();
      return 0;
    }
  return -1;
}

// Inputs exactly as main.cc:71-86 draws them in a build without OpenMP: one
// std::minstd_rand0 seeded with `seed`, std::uniform_real_distribution on
// [-1, 1), A[i] and B[i] drawn alternately.  Produced with the C++ standard
// library itself, to pin the C restatement in tsm_oracle.c.
__attribute__((visibility("default"))) void ref_fill_main_cc_f64(double* A, double* B, long count,
                                                                 unsigned seed) {
  std::minstd_rand0 engine(seed);
  std::uniform_real_distribution<double> dist(-1, 1);
  for (long i = 0; i < count; ++i) {
    A[i] = dist(engine);
    B[i] = dist(engine);
  }
}

// Number of host threads the work-item loops use.
__attribute__((visibility("default"))) int ref_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
