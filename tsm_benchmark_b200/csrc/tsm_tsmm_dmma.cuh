// tsm_tsmm_dmma.cuh -- Y (n x q) = X (n x p) * W (p x q) on the FP64 tensor
// cores (mma.sync m8n8k4 f64, "DMMA"; tcgen05 has no FP64 kind, so this is
// the FP64 tensor path of sm_100a).  Used for the fused backward of
// C = A^T B (dA = B dC^T, dB = A dC) when X is dense and 16-byte aligned.
// FP32 storage (TX = float) converts X and W to FP64 in registers, so each
// Y element is an FP64 sum rounded once to FP32.
//
// One DMMA multiplies an 8 x 4 block of X (8 rows, 4 of the p columns) by a
// 4 x 8 block of W into an 8 x 8 block of Y: 256 FMAs in one warp
// instruction, where the SIMT form needs 8 DFMA warp instructions and their
// shared-memory loads -- the SIMT form is issue-bound at these widths.
//
// Fragments (PTX ISA, mma.m8n8k4 .f64; lane = 4 g + t):
//   A (8 x 4, row):  lane holds A[g][t]
//   B (4 x 8, col):  lane holds B[t][g]
//   D (8 x 8):       lane holds D[g][2t], D[g][2t + 1]
// The contraction index may be permuted freely (the same way in A and B):
// k-step s = 2 kb + e uses column kappa = 8 kb + 2 t + e for lane t, so one
// 16-byte shared load gives a lane its A values of two k-steps (P >= 8; at
// P = 4 the single k-step uses kappa = t).  At Q = 4 a tile's columns 4..7
// are zero and not stored.
//
// Mapping (P = capacity of p, Q = capacity of q, powers of two in 4..64):
//   * a warp owns NO of the Q output columns (NT = NO / 8 tiles) and keeps
//     the matching W fragments in registers (KS x NT doubles, <= 32);
//   * a warp computes RG row groups of 8 rows at once (RG x NT independent
//     accumulator chains);
//   * rows of X stream through the TMA ring exactly as in tsm_tsmm.cuh;
//   * Y is stored from the D fragments: column pairs, streaming (evict-first)
//     stores -- Y is not read again by this launch.
//   * Y += X W (beta = 1) with YS = true: the producer streams each chunk's
//     old Y rows into the same stage after its X rows (one more bulk copy,
//     dense Y: ldy = q, q * sizeof(TX) a multiple of 16), and the consumers
//     add them from shared memory.  Without YS, beta = 1 reads each old Y
//     pair from global memory just before its store, one dependent load per
//     pair, which leaves the read stream latency-bound.
// Each Y element is one FP64 sum in a fixed order: deterministic (with beta,
// the product's sum plus the old Y value, staged or not).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"
#include "tsm_tsmm.cuh"

namespace tsm {

template <typename TX, int P, int Q, int CW, int STAGES, int RS, bool YS = false>
struct TsmmDmmaKernel {
  static_assert(P >= 4 && P <= 64 && (P & (P - 1)) == 0, "P: power of two in 4..64");
  static_assert(Q >= 4 && Q <= 64 && (Q & (Q - 1)) == 0, "Q: power of two in 4..64");
  static constexpr int NO_LIM = 1024 / P < 64 ? 1024 / P : 64;
  static constexpr int NO = Q < NO_LIM ? Q : NO_LIM;  // output columns per warp
  static constexpr int NT = NO >= 8 ? NO / 8 : 1;     // 8-column tiles per warp
  static constexpr int WPR = Q / NO;                  // warps sharing one row block
  static_assert(CW % WPR == 0, "warps must cover whole row blocks");
  static constexpr int NRS = CW / WPR;                // row-block slots per CTA
  static constexpr int KS = P / 4;                    // k-steps
  static constexpr int KPL = P >= 8 ? 2 : 1;          // k-steps per shared load
  static constexpr int KB = KS / KPL;                 // shared loads per row group
  // Row groups per warp (a power of two): up to 4, accumulators RG x NT x 2
  // <= 32 doubles, W fragments + accumulators + A values <= 68 doubles (no
  // spills under the 168-register cap of 9 warps), and no more than one
  // CTA pass per chunk fills.
  static constexpr int RG_ACC = 16 / NT < 4 ? 16 / NT : 4;
  static constexpr int RG_REG = KS * NT + 4 * (2 * NT + 2) <= 68 ? 4 : (KS * NT + 2 * (2 * NT + 2) <= 68 ? 2 : 1);
  static constexpr int RG_FIT = RS / (8 * NRS) < 1 ? 1 : RS / (8 * NRS);
  static constexpr int RG_A = RG_ACC < RG_REG ? RG_ACC : RG_REG;
  static constexpr int RG = RG_A < RG_FIT ? RG_A : RG_FIT;
  static constexpr int BLK = 8 * RG;                  // rows per warp block
  static constexpr int PASS = BLK * NRS;              // rows per CTA pass
  static_assert(RS % PASS == 0 && RS % 2 == 0, "chunk rows must be whole passes");
  static constexpr int THREADS = CW * 32 + 32;
  static constexpr int STAGE = RS * P;                // X elements per stage (capacity)
  static constexpr int STAGE_ALL = STAGE + (YS ? RS * Q : 0);  // + old Y rows (YS)
  static_assert((size_t(STAGE) * sizeof(TX)) % 16 == 0, "staged Y must start 16-byte aligned");
  static constexpr size_t RING_BYTES = size_t(STAGES) * STAGE_ALL * sizeof(TX);
  static constexpr size_t BAR_OFFSET = (RING_BYTES + 127) / 128 * 128;
  static constexpr size_t SMEM_BYTES = BAR_OFFSET + 2 * STAGES * sizeof(uint64_t) + 16;
};

namespace detail {

// W fragments of output columns [o0, o0 + 8 NT): b[s][j] = W[kappa(s)][o0 + 8 j + g].
template <typename TX, int KS, int NT>
__device__ __forceinline__ void load_w_frags(const TsmmProblem<TX>& pr, int o0, int g, int t,
                                             double (&b)[KS][NT]) {
#pragma unroll
  for (int s = 0; s < KS; ++s) {
    const int kappa = KS >= 2 ? 8 * (s >> 1) + 2 * t + (s & 1) : t;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const int o = o0 + 8 * j + g;
      const double w = (kappa < pr.p && o < pr.q)
                           ? static_cast<double>(
                                 pr.W[static_cast<int64_t>(kappa) * pr.w_row + static_cast<int64_t>(o) * pr.w_col])
                           : 0.0;
      b[s][j] = pr.negate ? -w : w;
    }
  }
}

// Two consecutive X elements (a lane's A values of two k-steps), as FP64.
__device__ __forceinline__ void load_pair(const double* x, double& a0, double& a1) {
  const double2 v = *reinterpret_cast<const double2*>(x);
  a0 = v.x;
  a1 = v.y;
}
__device__ __forceinline__ void load_pair(const float* x, double& a0, double& a1) {
  const float2 v = *reinterpret_cast<const float2*>(x);
  a0 = static_cast<double>(v.x);
  a1 = static_cast<double>(v.y);
}

// Two consecutive Y elements (aligned), streaming store; beta: Y += value.
__device__ __forceinline__ void store_pair(double* y, double v0, double v1, int beta) {
  double2 v = make_double2(v0, v1);
  if (beta) {
    const double2 old = *reinterpret_cast<const double2*>(y);
    v.x += old.x;
    v.y += old.y;
  }
  __stcs(reinterpret_cast<double2*>(y), v);
}
__device__ __forceinline__ void store_pair(float* y, double v0, double v1, int beta) {
  if (beta) {
    const float2 old = *reinterpret_cast<const float2*>(y);
    v0 += static_cast<double>(old.x);
    v1 += static_cast<double>(old.y);
  }
  __stcs(reinterpret_cast<float2*>(y), make_float2(static_cast<float>(v0), static_cast<float>(v1)));
}

// Y += value with the old pair read from the staged rows in shared memory
// (same sum as store_pair with beta: value + old, rounded once to TX).
__device__ __forceinline__ void store_pair_staged(double* y, const double* old, double v0, double v1) {
  const double2 o = *reinterpret_cast<const double2*>(old);
  store_pair(y, v0 + o.x, v1 + o.y, 0);
}
__device__ __forceinline__ void store_pair_staged(float* y, const float* old, double v0, double v1) {
  const float2 o = *reinterpret_cast<const float2*>(old);
  store_pair(y, v0 + static_cast<double>(o.x), v1 + static_cast<double>(o.y), 0);
}

}  // namespace detail

template <typename TX, int P, int Q, int CW, int STAGES, int RS, bool YS = false>
__global__ void __launch_bounds__(TsmmDmmaKernel<TX, P, Q, CW, STAGES, RS, YS>::THREADS, 1)
    tsm_tsmm_dmma_kernel(const TsmmArgs<TX> args) {
  using K = TsmmDmmaKernel<TX, P, Q, CW, STAGES, RS, YS>;
  extern __shared__ __align__(128) unsigned char smem[];
  TX* ring = reinterpret_cast<TX*>(smem);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + K::BAR_OFFSET);
  uint64_t* empty = full + STAGES;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + STAGES);

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
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
    // ---------------- producer warp: X rows into the ring (1-D bulk copies)
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
          const TsmmProblem<TX>& pr = args.prob[pi];
          const int64_t r0 = (c - (pi ? args.split : 0)) * RS;
          const int64_t rows = (pr.rows_main - r0) < RS ? (pr.rows_main - r0) : RS;
          const uint32_t bytes = static_cast<uint32_t>(rows * pr.p * sizeof(TX));
          const uint32_t ybytes = YS ? static_cast<uint32_t>(rows * pr.q * sizeof(TX)) : 0u;
          dev::mbar_arrive_expect_tx(&full[s], bytes + ybytes);
          dev::bulk_g2s_evict_first(ring + s * K::STAGE_ALL, pr.X + r0 * pr.p, bytes, &full[s], policy);
          if constexpr (YS)  // the old Y rows of the chunk (dense: pitch q)
            dev::bulk_g2s_evict_first(ring + s * K::STAGE_ALL + K::STAGE, pr.Y + r0 * pr.q, ybytes, &full[s],
                                      policy);
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
    const int g = lane >> 2, t = lane & 3;
    const int ot = warp % K::WPR;   // output-column group of this warp
    const int slot = warp / K::WPR; // row-block slot
    const int o0 = ot * K::NO;
    int cur = -1;
    double b[K::KS][K::NT];
    int64_t it = 0;
    for (int64_t c = blockIdx.x; c < args.total_chunks; c += G, ++it) {
      const int s = static_cast<int>(it % STAGES);
      const int pi = c < args.split ? 0 : 1;
      const TsmmProblem<TX>& pr = args.prob[pi];
      if (pi != cur) {
        detail::load_w_frags<TX, K::KS, K::NT>(pr, o0, g, t, b);
        cur = pi;
      }
      if (!dev::mbar_wait(&full[s], static_cast<uint32_t>((it / STAGES) & 1), abort)) {
        *abort = 1;
        atomicOr(args.error, dev::kErrTimeout);
        break;
      }
      const int64_t r0 = (c - (pi ? args.split : 0)) * RS;
      const int rows = static_cast<int>((pr.rows_main - r0) < RS ? (pr.rows_main - r0) : RS);
      const TX* stage = ring + s * K::STAGE_ALL;
      const TX* ystage = stage + K::STAGE;  // old Y rows, pitch q (YS only)
      const int p = pr.p;
      const bool exact_p = p == P;
      const bool vec_y =
          pr.q == Q && (pr.ldy & 1) == 0 && (reinterpret_cast<uintptr_t>(pr.Y) & (2 * sizeof(TX) - 1)) == 0;
      if (rows == RS && exact_p && vec_y && pr.ldy == Q && (YS || pr.beta == 0)) {
        // Fast path: a full chunk, p = P, q = Q = ldy, Y = X W (or, with YS,
        // Y += X W from the staged rows).  Every stride is a compile-time
        // constant and no row needs a guard.
        TX* const ybase = pr.Y + (r0 + g) * Q + o0 + 2 * t;
        const TX* const xbase = stage + g * P + (K::KPL == 2 ? 2 * t : t);
#pragma unroll 1
        for (int rb = slot * K::BLK; rb < RS; rb += K::PASS) {
          double d[K::RG][K::NT][2];
#pragma unroll
          for (int kb = 0; kb < K::KB; ++kb) {
            double a[K::RG][2];
#pragma unroll
            for (int i = 0; i < K::RG; ++i) {
              if constexpr (K::KPL == 2)
                detail::load_pair(xbase + (rb + 8 * i) * P + 8 * kb, a[i][0], a[i][1]);
              else
                a[i][0] = static_cast<double>(xbase[(rb + 8 * i) * P]);  // P = 4: column t
            }
#pragma unroll
            for (int e = 0; e < K::KPL; ++e)
#pragma unroll
              for (int j = 0; j < K::NT; ++j)
#pragma unroll
                for (int i = 0; i < K::RG; ++i) {
                  if (kb == 0 && e == 0)
                    dev::dmma_m8n8k4_first(d[i][j][0], d[i][j][1], a[i][e], b[K::KPL * kb + e][j]);
                  else
                    dev::dmma_m8n8k4(d[i][j][0], d[i][j][1], a[i][e], b[K::KPL * kb + e][j]);
                }
          }
          if (Q >= 8 || 2 * t < Q) {
#pragma unroll
            for (int i = 0; i < K::RG; ++i)
#pragma unroll
              for (int j = 0; j < K::NT; ++j) {
                const int off = (rb + 8 * i + g) * Q + o0 + 8 * j + 2 * t;
                if constexpr (YS)
                  detail::store_pair_staged(ybase + (rb + 8 * i) * Q + 8 * j, ystage + off, d[i][j][0], d[i][j][1]);
                else
                  detail::store_pair(ybase + (rb + 8 * i) * Q + 8 * j, d[i][j][0], d[i][j][1], 0);
              }
          }
        }
      } else
      for (int rb = slot * K::BLK; rb < rows; rb += K::PASS) {
        double d[K::RG][K::NT][2];
#pragma unroll
        for (int i = 0; i < K::RG; ++i)
#pragma unroll
          for (int j = 0; j < K::NT; ++j) d[i][j][0] = d[i][j][1] = 0.0;
        // Row of this lane in each group (clamped to the last valid row: a
        // clamped row's results are not stored).
        const TX* xr[K::RG];
#pragma unroll
        for (int i = 0; i < K::RG; ++i) {
          const int r = rb + 8 * i + g;
          xr[i] = stage + static_cast<int64_t>(r < rows ? r : rows - 1) * p;
        }
#pragma unroll
        for (int kb = 0; kb < K::KB; ++kb) {
          double a[K::RG][2];
          const int kappa = K::KPL == 2 ? 8 * kb + 2 * t : t;
          if (exact_p && K::KPL == 2) {
#pragma unroll
            for (int i = 0; i < K::RG; ++i) detail::load_pair(xr[i] + kappa, a[i][0], a[i][1]);
          } else {
#pragma unroll
            for (int i = 0; i < K::RG; ++i) {
              a[i][0] = kappa < p ? static_cast<double>(xr[i][kappa]) : 0.0;
              a[i][1] = K::KPL == 2 && kappa + 1 < p ? static_cast<double>(xr[i][kappa + 1]) : 0.0;
            }
          }
#pragma unroll
          for (int e = 0; e < K::KPL; ++e)
#pragma unroll
            for (int j = 0; j < K::NT; ++j)
#pragma unroll
              for (int i = 0; i < K::RG; ++i)
                dev::dmma_m8n8k4(d[i][j][0], d[i][j][1], a[i][e], b[K::KPL * kb + e][j]);
        }
        // D[g][2t + {0,1}] of tile j -> Y[r][o0 + 8 j + 2 t + {0,1}]
#pragma unroll
        for (int i = 0; i < K::RG; ++i) {
          const int r = rb + 8 * i + g;
          if (r >= rows) continue;
          TX* yrow = pr.Y + (r0 + r) * pr.ldy;
#pragma unroll
          for (int j = 0; j < K::NT; ++j) {
            const int o = o0 + 8 * j + 2 * t;
            if constexpr (YS) {
              // Dense Y (ldy = q): old values at r * q + o of the staged rows.
              const TX* old = ystage + r * pr.q + o;
              if (vec_y) {
                if (Q >= 8 || o < Q) detail::store_pair_staged(yrow + o, old, d[i][j][0], d[i][j][1]);
              } else {
                if (o < pr.q) yrow[o] = static_cast<TX>(static_cast<double>(old[0]) + d[i][j][0]);
                if (o + 1 < pr.q) yrow[o + 1] = static_cast<TX>(static_cast<double>(old[1]) + d[i][j][1]);
              }
            } else if (vec_y) {
              if (Q >= 8 || o < Q) detail::store_pair(yrow + o, d[i][j][0], d[i][j][1], pr.beta);
            } else {
              if (o < pr.q) detail::store_y(pr, r0 + r, o, static_cast<TX>(d[i][j][0]));
              if (o + 1 < pr.q) detail::store_y(pr, r0 + r, o + 1, static_cast<TX>(d[i][j][1]));
            }
          }
        }
      }
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&empty[s]);
    }
    // Rows the ring did not stream (fewer than 16 bytes' worth per problem):
    // CTA 0 computes them from global memory, one output per thread.
    if (blockIdx.x == 0) {
      for (int pi = 0; pi < args.nprob; ++pi) {
        const TsmmProblem<TX>& pr = args.prob[pi];
        const int64_t tail = pr.n - pr.rows_main;
        for (int64_t e = tid; e < tail * pr.q; e += CW * 32) {
          const int64_t r = pr.rows_main + e / pr.q;
          const int o = static_cast<int>(e % pr.q);
          double y = 0.0;
          for (int a = 0; a < pr.p; ++a)
            y = fma(static_cast<double>(pr.X[r * pr.ldx + a]),
                    static_cast<double>(pr.W[static_cast<int64_t>(a) * pr.w_row + static_cast<int64_t>(o) * pr.w_col]),
                    y);
          if (pr.negate) y = -y;
          detail::store_y(pr, r, o, static_cast<TX>(y));
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

}  // namespace tsm
