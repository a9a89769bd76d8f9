// tsmttsm.hh (compat) -- the reference's kernel entry points, same names and
// template parameters, running on libtsm_b200.so.
//
// The reference header (tsmttsm.hh:15-586) defines nine variants
//   tsmttsm  <T, M, stride>                                   (V1, :15)
//   tsmttsm2 <T, M, stride, max_tile_size>                    (V2, :40)
//   tsmttsm3 <T, M, stride, max_tile_size>                    (V3, :80)
//   tsmttsm4 <T, M, stride, max_tile_size>                    (V4, :125)
//   tsmttsm5 <T, M, stride, max_tile_size>                    (V5, :170)
//   tsmttsm6 <T, M, global_size, local_size, max_tile_size>   (V6, :230)
//   tsmttsm7 <T, M, stride, max_tile_size>                    (V7, :303)
//   tsmttsm9 <T, M, global_size, local_size, max_tile_size>   (V9, :368)
//   tsmttsm8 <T, M, worker_mult = 64>                         (V8, :445)
// each `sycl::event f(sycl::queue& q, int K, T* A, T* B, T* C)` adding
// A^T * B (A, B: K x M row-major; C: M x M) into C.  Here every one of them
// submits tsm_gemm_tn_f64 with accumulate = 1 on the queue's stream and
// returns an event bracketing it.  The launch-shape parameters (stride,
// local_size, max_tile_size, worker_mult) are accepted and ignored: the
// library picks its own tuned variant.  The reference's compile-time shape
// checks are kept, so code that compiled against it compiles here.  T must be
// double, as in every reference driver (main.cc:162, main_codegen.cc:10).
#pragma once

#include <sycl/sycl.hpp>

#include <algorithm>
#include <string>

#include "tsm.h"

namespace tsm_compat {

// C += A^T B on the queue's stream with the given variant (-1: the tuned
// default) on at most max_ctas CTAs (0: the variant's own grid).
template <class T>
sycl::event accumulate_tn(sycl::queue& q, long long K, int M, int N, const T* A, const T* B, T* C,
                          int variant = -1, long long max_ctas = 0) {
  static_assert(std::is_same_v<T, double>, "the plain path is FP64 (T = double)");
  const size_t ws_bytes = tsm_gemm_tn_workspace_size(K, M, N);
  if (ws_bytes == 0) throw sycl::exception("tsmttsm: unsupported width or no CUDA device");
  void* ws = q.workspace(ws_bytes);
  sycl::event e = q.begin();
  const tsm_status st = tsm_gemm_tn_f64_launch(q.native_stream(), K, M, N, A, M, B, N, C, N, /*accumulate=*/1, ws,
                                               q.workspace_bytes(), variant, max_ctas);
  if (st != TSM_SUCCESS)
    throw sycl::exception(std::string("tsm_gemm_tn_f64: ") + tsm_status_string(st) + " " + tsm_last_cuda_error());
  e.record_end();
  return e;
}

// Index of the compiled variant called `name`, or -1 (use the default).
inline int variant_by_name(const char* name) {
  const int n = tsm_variant_count();
  for (int i = 0; i < n; ++i) {
    tsm_variant_info info;
    if (tsm_variant_get_info(i, &info) == TSM_SUCCESS && std::string(info.name) == name) return i;
  }
  return -1;
}

template <int M, int max_tile_size>
constexpr bool tiles_fit() {
  constexpr int tile = std::min(max_tile_size, M);
  return (M * M) % (tile * tile) == 0;
}

}  // namespace tsm_compat

template <typename T, int M_, int stride>
sycl::event tsmttsm(sycl::queue& q, int K, T* A, T* B, T* C) {
  return tsm_compat::accumulate_tn<T>(q, K, M_, M_, A, B, C);
}

template <typename T, int M, int stride, int max_tile_size>
sycl::event tsmttsm2(sycl::queue& q, int K, T* A, T* B, T* C) {
  static_assert(tsm_compat::tiles_fit<M, max_tile_size>(), "Currently it is assumed that the tiles fit perfectly");
  return tsm_compat::accumulate_tn<T>(q, K, M, M, A, B, C);
}

template <typename T, int M, int stride, int max_tile_size>
sycl::event tsmttsm3(sycl::queue& q, int K, T* A, T* B, T* C) {
  static_assert(tsm_compat::tiles_fit<M, max_tile_size>(), "Currently it is assumed that the tiles fit perfectly");
  return tsm_compat::accumulate_tn<T>(q, K, M, M, A, B, C);
}

template <typename T, int M, int stride, int max_tile_size>
sycl::event tsmttsm4(sycl::queue& q, int K, T* A, T* B, T* C) {
  static_assert(tsm_compat::tiles_fit<M, max_tile_size>(), "Currently it is assumed that the tiles fit perfectly");
  return tsm_compat::accumulate_tn<T>(q, K, M, M, A, B, C);
}

template <typename T, int M, int stride, int max_tile_size>
sycl::event tsmttsm5(sycl::queue& q, int K, T* A, T* B, T* C) {
  static_assert(tsm_compat::tiles_fit<M, max_tile_size>(), "Currently it is assumed that the tiles fit perfectly");
  return tsm_compat::accumulate_tn<T>(q, K, M, M, A, B, C);
}

template <typename T, int M, int global_size, int local_size, int max_tile_size>
sycl::event tsmttsm6(sycl::queue& q, int K, T* A, T* B, T* C) {
  static_assert(tsm_compat::tiles_fit<M, max_tile_size>(), "tiles must divide M x M");
  return tsm_compat::accumulate_tn<T>(q, K, M, M, A, B, C);
}

template <typename T, int M, int stride, int max_tile_size>
sycl::event tsmttsm7(sycl::queue& q, int K, T* A, T* B, T* C) {
  static_assert(tsm_compat::tiles_fit<M, max_tile_size>(), "Currently it is assumed that the tiles fit perfectly");
  return tsm_compat::accumulate_tn<T>(q, K, M, M, A, B, C);
}

template <typename T, int M, int worker_mult = 64>
sycl::event tsmttsm8(sycl::queue& q, int K, T* A, T* B, T* C) {
  return tsm_compat::accumulate_tn<T>(q, K, M, M, A, B, C);
}

template <typename T, int M, int global_size, int local_size, int max_tile_size>
sycl::event tsmttsm9(sycl::queue& q, int K, T* A, T* B, T* C) {
  static_assert(tsm_compat::tiles_fit<M, max_tile_size>(), "tiles must divide M x M");
  return tsm_compat::accumulate_tn<T>(q, K, M, M, A, B, C);
}
