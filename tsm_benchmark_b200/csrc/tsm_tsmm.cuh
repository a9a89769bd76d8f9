// tsm_tsmm.cuh -- tall-skinny times small: Y (n x q) = X (n x p) * W (p x q),
// the backward products of C = A^T * B:
//     dA = B * dC^T      (X = B, W = dC^T: p = k, q = m)
//     dB = A * dC        (X = A, W = dC:   p = m, q = k)
// The reference has no backward; this is the differentiation form.  One
// launch can carry both products (the fused backward): its chunks are split
// between the two problems.
//
// Mapping (C = capacity of p and q, a power of two <= 64):
//   * each consumer lane owns ONE output column o of Y and keeps column o of
//     W in registers (C values) for the whole launch (reloaded once if the
//     launch switches problems);
//   * the rows of X are streamed into a shared-memory ring by 1-D TMA bulk
//     copies (producer warp, mbarriers, as in tsm_plain.cuh) and every lane
//     of a row group reads the same row -- broadcast loads, no bank
//     conflicts;
//   * for C < 32 a warp covers 32 / C rows at a time, for C >= 32 each row's
//     outputs span C / 32 warps;
//   * Y is stored straight from registers, coalesced (the lanes of a row
//     group write consecutive columns).
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

template <typename T, int C, int CW, int STAGES, int RS>
struct TsmmKernel {
  static_assert(C >= 1 && C <= 64 && (C & (C - 1)) == 0, "capacity must be a power of two <= 64");
  static constexpr int EPC = 16 / int(sizeof(T));
  static constexpr int CT = CW * 32;
  static constexpr int THREADS = CT + 32;
  static constexpr int WPR = C >= 32 ? C / 32 : 1;  // warps per row (C >= 32)
  static constexpr int RW = C >= 32 ? 1 : 32 / C;   // rows per warp (C < 32)
  static_assert(CW % WPR == 0, "warps must cover whole rows");
  static constexpr int RGN = (CW / WPR) * RW;       // rows in flight per CTA
  static_assert(RS % RGN == 0 && RS % EPC == 0, "chunk rows must be whole passes and 16-byte copies");
  static constexpr int STAGE = RS * C;              // elements per stage (capacity)
  static constexpr size_t RING_BYTES = size_t(STAGES) * STAGE * sizeof(T);
  static constexpr size_t BAR_OFFSET = (RING_BYTES + 127) / 128 * 128;
  static constexpr size_t SMEM_BYTES = BAR_OFFSET + 2 * STAGES * sizeof(uint64_t) + 16;
};

namespace detail {

template <typename T, int C>
__device__ __forceinline__ void load_w_column(const TsmmProblem<T>& pr, int o, T (&w)[C]) {
#pragma unroll
  for (int a = 0; a < C; ++a)
    w[a] = (a < pr.p && o < pr.q) ? pr.W[static_cast<int64_t>(a) * pr.w_row + static_cast<int64_t>(o) * pr.w_col]
                                  : T(0);
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

template <typename T, int C, int CW, int STAGES, int RS>
__global__ void __launch_bounds__(TsmmKernel<T, C, CW, STAGES, RS>::THREADS, 1)
    tsm_tsmm_bulk_kernel(const TsmmArgs<T> args) {
  using K = TsmmKernel<T, C, CW, STAGES, RS>;
  extern __shared__ __align__(128) unsigned char smem[];
  T* ring = reinterpret_cast<T*>(smem);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + K::BAR_OFFSET);
  uint64_t* empty = full + STAGES;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + STAGES);

  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  if (t == 0) {
    for (int s = 0; s < STAGES; ++s) {
      dev::mbar_init(&full[s], 1);
      dev::mbar_init(&empty[s], CW);
    }
    *abort = 0;
    dev::fence_mbar_init();
  }
  __syncthreads();
  const int64_t G = gridDim.x;

  if (warp == CW) {
    // ---------------- producer warp
    int64_t issued = 0;
    const uint64_t policy = dev::policy_evict_first();
    for (int64_t c = blockIdx.x; c < args.total_chunks; c += G, ++issued) {
      const int s = static_cast<int>(issued % STAGES);
      const int64_t round = issued / STAGES;
      bool ok = true;
      if (lane == 0) {
        if (round > 0) ok = dev::mbar_wait(&empty[s], static_cast<uint32_t>((round - 1) & 1), abort);
        if (ok) {
          const int pi = c < args.split ? 0 : 1;
          const TsmmProblem<T>& pr = args.prob[pi];
          const int64_t r0 = (c - (pi ? args.split : 0)) * RS;
          const int64_t rows = (pr.rows_main - r0) < RS ? (pr.rows_main - r0) : RS;
          const uint32_t bytes = static_cast<uint32_t>(rows * pr.p * sizeof(T));
          dev::mbar_arrive_expect_tx(&full[s], bytes);
          dev::bulk_g2s_evict_first(ring + s * K::STAGE, pr.X + r0 * pr.p, bytes, &full[s], policy);
        } else {
          *abort = 1;
          atomicOr(args.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else {
    // ---------------- consumer warps
    int o, rgp;
    if constexpr (C >= 32) {
      o = (warp % K::WPR) * 32 + lane;
      rgp = warp / K::WPR;
    } else {
      o = lane % C;
      rgp = warp * K::RW + lane / C;
    }
    int cur = -1;
    T w[C];
    int64_t it = 0;
    for (int64_t c = blockIdx.x; c < args.total_chunks; c += G, ++it) {
      const int s = static_cast<int>(it % STAGES);
      const int pi = c < args.split ? 0 : 1;
      const TsmmProblem<T>& pr = args.prob[pi];
      if (pi != cur) {
        detail::load_w_column<T, C>(pr, o, w);
        cur = pi;
      }
      if (!dev::mbar_wait(&full[s], static_cast<uint32_t>((it / STAGES) & 1), abort)) {
        *abort = 1;
        atomicOr(args.error, dev::kErrTimeout);
        break;
      }
      const int64_t r0 = (c - (pi ? args.split : 0)) * RS;
      const int rows = static_cast<int>((pr.rows_main - r0) < RS ? (pr.rows_main - r0) : RS);
      const T* stage = ring + s * K::STAGE;
      const bool vec = (pr.p == C) && (C % K::EPC == 0);
      if (vec) {
        for (int r = rgp; r < rows; r += K::RGN) {
          const T y = detail::row_dot<T, C, (C % K::EPC == 0)>(stage + r * pr.p, pr.p, w);
          if (o < pr.q) detail::store_y(pr, r0 + r, o, y);
        }
      } else {
        for (int r = rgp; r < rows; r += K::RGN) {
          const T y = detail::row_dot<T, C, false>(stage + r * pr.p, pr.p, w);
          if (o < pr.q) detail::store_y(pr, r0 + r, o, y);
        }
      }
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&empty[s]);
    }
    // Rows the ring did not stream (at most three per problem): CTA 0 reads
    // them from global memory.
    if (blockIdx.x == 0) {
      for (int pi = 0; pi < args.nprob; ++pi) {
        const TsmmProblem<T>& pr = args.prob[pi];
        if (pr.rows_main >= pr.n) continue;
        detail::load_w_column<T, C>(pr, o, w);
        for (int64_t r = pr.rows_main + rgp; r < pr.n; r += K::RGN) {
          const T y = detail::row_dot<T, C, false>(pr.X + r * pr.ldx, pr.p, w);
          if (o < pr.q) detail::store_y(pr, r, o, y);
        }
      }
    }
  }

  __syncthreads();
  if (*abort && warp == CW && lane == 0) {
    int64_t issued = 0;
    for (int64_t c = blockIdx.x; c < args.total_chunks; c += G) ++issued;
    volatile int no_abort = 0;
    for (int64_t q = issued > STAGES ? issued - STAGES : 0; q < issued; ++q)
      if (!dev::mbar_wait(&full[q % STAGES], static_cast<uint32_t>((q / STAGES) & 1), &no_abort)) break;
  }
}

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
