// tsm_tsmm.cuh -- tall-skinny times small: Y (n x q) = X (n x p) * W (p x q),
// the backward products of C = A^T * B:
//     dA = B * dC^T      (X = B, W = dC^T: p = k, q = m)
//     dB = A * dC        (X = A, W = dC:   p = m, q = k)
// The reference has no backward; this is the differentiation form.  One
// launch can carry both products (the fused backward): its chunks are split
// between the two problems.
//
// Kernels: dense, 16-byte aligned X streams through a TMA ring into the FP64
// tensor cores (tsm_tsmm_dmma.cuh); any other X (a column slice, an odd
// row stride) takes the SIMT kernel below, which loads rows directly:
//   * each lane owns ONE output column o of Y and keeps column o of W in
//     registers (C = capacity of p and q, a power of two <= 64);
//   * for C < 32 a warp covers 32 / C rows at a time, for C >= 32 each row's
//     outputs span C / 32 warps;
//   * Y is stored straight from registers, coalesced.
// There is no reduction across rows, hence no workspace beyond the error
// word; results are deterministic (each output is one fixed-order sum).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"
#include "tsm_plain.cuh"  // Vec16

namespace tsm {

template <typename T>
struct TsmmProblem {
  const T* X;
  int64_t ldx;
  const T* W;  // W[a][b] = W[a * w_row + b * w_col]
  int64_t w_row, w_col;
  T* Y;
  int64_t ldy;
  int64_t n;
  int p, q;
  int beta;            // 0: Y = X W, 1: Y += X W
  int negate;          // 1: W is read as -W (exact), so beta = 1 gives Y -= X W
  int64_t rows_main;   // rows the TMA ring streams; the rest are read directly
  int64_t num_chunks;  // ceil(rows_main / RS)
};

template <typename T>
struct TsmmArgs {
  TsmmProblem<T> prob[2];
  int nprob;
  int64_t split;  // chunks [0, split) belong to prob[0], the rest to prob[1]
  int64_t total_chunks;
  unsigned* error;
};

namespace detail {

template <typename T, int C>
__device__ __forceinline__ void load_w_column(const TsmmProblem<T>& pr, int o, T (&w)[C]) {
#pragma unroll
  for (int a = 0; a < C; ++a) {
    const T x = (a < pr.p && o < pr.q) ? pr.W[static_cast<int64_t>(a) * pr.w_row + static_cast<int64_t>(o) * pr.w_col]
                                       : T(0);
    w[a] = pr.negate ? -x : x;
  }
}

// y = x_row . w for one row held in memory at `x` (p valid elements).
template <typename T, int C, bool VEC>
__device__ __forceinline__ T row_dot(const T* x, int p, const T (&w)[C]) {
  T acc = T(0);
  if constexpr (VEC) {
    using V = Vec16<T>;
#pragma unroll
    for (int c = 0; c < C / V::N; ++c) {
      T v[V::N];
      V::split(reinterpret_cast<const typename V::type*>(x)[c], v);
#pragma unroll
      for (int e = 0; e < V::N; ++e) acc = fma(v[e], w[V::N * c + e], acc);
    }
  } else {
#pragma unroll
    for (int a = 0; a < C; ++a)
      if (a < p) acc = fma(x[a], w[a], acc);
  }
  return acc;
}

template <typename T>
__device__ __forceinline__ void store_y(const TsmmProblem<T>& pr, int64_t row, int o, T y) {
  T* dst = pr.Y + row * pr.ldy + o;
  *dst = pr.beta ? *dst + y : y;
}

}  // namespace detail

// Direct loads: any ldx / alignment.  Same lane mapping; every CTA walks its
// row groups of both problems from global memory.
template <typename T, int C, int THREADS>
__global__ void __launch_bounds__(THREADS) tsm_tsmm_direct_kernel(const TsmmArgs<T> args) {
  constexpr int NW = THREADS / 32;
  constexpr int WPR = C >= 32 ? C / 32 : 1;
  constexpr int RW = C >= 32 ? 1 : 32 / C;
  static_assert(NW % WPR == 0, "warps must cover whole rows");
  constexpr int RGN = (NW / WPR) * RW;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int o, rgp;
  if constexpr (C >= 32) {
    o = (warp % WPR) * 32 + lane;
    rgp = warp / WPR;
  } else {
    o = lane % C;
    rgp = warp * RW + lane / C;
  }
  T w[C];
  for (int pi = 0; pi < args.nprob; ++pi) {
    const TsmmProblem<T>& pr = args.prob[pi];
    detail::load_w_column<T, C>(pr, o, w);
    const int64_t step = static_cast<int64_t>(gridDim.x) * RGN;
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * RGN + rgp; r < pr.n; r += step) {
      const T y = detail::row_dot<T, C, false>(pr.X + r * pr.ldx, pr.p, w);
      if (o < pr.q) detail::store_y(pr, r, o, y);
    }
  }
}

}  // namespace tsm
