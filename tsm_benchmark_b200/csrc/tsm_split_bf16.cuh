// tsm_split_bf16.cuh -- the precision form with BF16 parts: C (m x k, FP64)
// = A^T B for FP32-stored A (n x m) and B (n x k), m, k <= 32 and multiples
// of 4, on the tcgen05 tensor cores (kind::f16, BF16 inputs, FP32
// accumulation in tensor memory).
//
// Every FP32 value x is split into PARTS BF16 values (8 significant bits
// each), h = rn(x), then rn of what is left:
//   PARTS = 2 (hi/lo):      |x - h - l|     <= 2^-16 |x|
//   PARTS = 3 (hi/mid/lo):  |x - h - m - l| <= 2^-24 |x|
// (each remainder is exact in FP32).  One MMA per 16 rows computes all
// PARTS x PARTS part products at once, accumulated in FP32 over 256 rows:
//   D (M = 128, N = 32 PARTS) = [A_0; A_1; ...]  x  [B_0 | B_1 | ...]^T
// over K = 16 rows: D row 32 p + i is A's part p of column i, D column
// 32 q + j is B's part q of column j.  The sum over (p, q) of those blocks is
// C's contribution from the rows.  Rows 32 PARTS .. 127 of the A operand are
// not A data (the descriptor runs on into the B tiles of the same stage):
// their D rows are never read.
//
// Operand layout: K-major with the 128-byte swizzle (the canonical tcgen05
// layout for 16-bit types): a stage holds 64 rows of the input (K = 64, one
// swizzle atom wide); operand row y (a part of one column) is 128 bytes of
// 64 BF16 values, 16-byte chunk q of it at chunk q ^ (y mod 8), 8-row atoms
// 1024 bytes apart (SBO).  The k-step s of 16 values starts 32 s bytes into
// the atom rows.
//
// Pipeline, one persistent CTA per SM (16 warps):
//   warp 0       TMA producer: 64-row boxes of raw FP32 A and B (tensor maps,
//                32 columns, zero fill past m, k and n) into a raw ring
//   warps 2-9    converters: lane c takes column c of 8 rows of A or B, splits
//                the 8 values into PARTS BF16 parts and writes each part as
//                one 16-byte chunk (8 consecutive K values) of operand row
//                32 p + c -- a warp's 8 chunks per 8-lane phase land in 8
//                different bank groups (chunk rg ^ (c mod 8))
//   warps 1, 14, 15  MMA issuers: chunk it goes to issuer it mod 3, which
//                owns operand stages it mod 6 and TMEM accumulator it mod 3
//                (issuing from one thread was the bottleneck of the TF32 form)
//                and accumulates kFlush = 4 of its chunks before a drain
//   warps 10-13  epilogue: warp w reads TMEM lanes 32 w .. +31, i.e. A's part
//                w (w < PARTS): all PARTS column blocks of 16 columns, one
//                wait, their FP32 sum (smallest part first) into FP64.  A
//                timing copy without the drains ran in 63-66 % of the time
//                with one TMEM wait per block and a drain per 64 rows.
// All waits are bounded (dev::mbar_wait); on a timeout the CTA records the
// error, drains its copies and MMAs (bounded) and frees its TMEM.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"
#include "tsm_split.cuh"
#include "tsm_split_tma.cuh"

namespace tsm {

namespace split16 {

constexpr int kRows = 64;                      // rows per chunk: 4 MMAs of K = 16
constexpr int kIssuers = 3;
constexpr int kOpStages = 2 * kIssuers;        // two operand stages per issuer: converters run a round ahead
static_assert(kOpStages % kIssuers == 0, "an operand stage belongs to one issuer");
// An issuer's chunks per accumulator drain (256 rows).  Against drains every
// 2 chunks, on one B200 at n = 2^25, 32 x 32 (300-call loops): hi/mid/lo
// 2.01 vs 2.06 ms (normwise error 1.8e-7 vs 9.7e-8), hi/lo 1.75 vs 1.80 ms
// (3.0e-6 either way, the split's own error); every 8 chunks gains ~1 % more.
constexpr int kFlushDefault = 4;
constexpr int kRawTile = kRows * 32 * 4;       // one operand: 64 rows x 32 floats (8 KB)
constexpr int kRawStageBytes = 2 * kRawTile;   // A, B
constexpr int kConvWarps = 8;
constexpr int kEpiWarp0 = 10;
constexpr int kWarps = 16;                     // 0 producer, 1/14/15 issuers, 2-9 converters, 10-13 epilogue
constexpr int kThreads = kWarps * 32;
constexpr int kAccCols = 128;                  // TMEM columns per accumulator

template <int PARTS>
struct Shape {
  static_assert(PARTS == 2 || PARTS == 3, "two or three BF16 parts");
  static constexpr int OP_ROWS = 32 * PARTS;            // operand rows of A (and of B)
  static constexpr int OP_TILE = OP_ROWS * 128;         // bytes of one operand (K = 64)
  static constexpr int OP_STAGE = 2 * OP_TILE;          // A, then B (A's M = 128 reads on into B)
  static_assert(OP_STAGE >= 128 * 128, "M = 128 rows of A must stay inside the stage");
  static constexpr int N = 32 * PARTS;
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
                                    (static_cast<uint32_t>(128 >> 4) << 24);  // F32 D, BF16 A/B, K-major
  // Raw ring depth: what shared memory leaves (the pipeline is not bound by
  // HBM: a timing copy with no copies at all ran within 2 %).
  static constexpr int RAW_STAGES = PARTS == 2 ? 8 : 4;
  static constexpr size_t OP_OFFSET = 0;
  static constexpr size_t RAW_OFFSET = OP_OFFSET + size_t(kOpStages) * OP_STAGE;
  static constexpr size_t BAR_OFFSET = RAW_OFFSET + size_t(RAW_STAGES) * kRawStageBytes;
  static constexpr int NUM_BARS = 2 * RAW_STAGES + 2 * kOpStages + 2 * kIssuers;
  static constexpr size_t SMEM_BYTES = BAR_OFFSET + NUM_BARS * 8 + 32 + 1024;  // + alignment slack
  static_assert(SMEM_BYTES <= 232448, "dynamic shared memory limit of sm_100a");
  static_assert(OP_STAGE % 1024 == 0 && RAW_OFFSET % 1024 == 0, "1024-byte aligned swizzle atoms");
  static constexpr uint32_t TMEM_COLS = kIssuers * kAccCols <= 256 ? 256 : 512;
};

// BF16 x2 (round to nearest even) of two floats, and back.
__device__ __forceinline__ uint32_t pack_bf16x2(float lo_elem, float hi_elem) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo_elem, hi_elem);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float bf16_lo_f32(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi_f32(uint32_t v) { return __uint_as_float(v & 0xFFFF0000u); }

}  // namespace split16

// FLUSH: an issuer's chunks accumulated in its TMEM accumulator before a
// drain (FP32 accumulation over FLUSH * 64 rows).
template <int PARTS, int FLUSH>
__global__ void __launch_bounds__(split16::kThreads, 1)
    tsm_tn_split_bf16_kernel(const __grid_constant__ SplitTmaArgs args) {
  using namespace split16;
  using S = Shape<PARTS>;
  constexpr int kFlush = FLUSH;
  const SplitArgs& p = args.p;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024u - (dev::smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::BAR_OFFSET);
  uint64_t* raw_full = bars;                      // raw stage landed (TMA transaction count)
  uint64_t* raw_empty = raw_full + S::RAW_STAGES;    // raw stage read (converter warps)
  uint64_t* op_full = raw_empty + S::RAW_STAGES;     // operand stage written (converter warps)
  uint64_t* op_empty = op_full + kOpStages;       // operand stage's MMAs completed (commit)
  uint64_t* d_full = op_empty + kOpStages;        // accumulator b complete (commit)
  uint64_t* d_empty = d_full + kIssuers;          // accumulator b drained (epilogue warps)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + S::NUM_BARS);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  unsigned* s_is_last = reinterpret_cast<unsigned*>(tmem_slot + 2);

  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  const int64_t G = gridDim.x;

  if (t == 0) {
    for (int s = 0; s < S::RAW_STAGES; ++s) {
      dev::mbar_init(&raw_full[s], 1);
      dev::mbar_init(&raw_empty[s], kConvWarps);
    }
    for (int o = 0; o < kOpStages; ++o) {
      dev::mbar_init(&op_full[o], kConvWarps);
      dev::mbar_init(&op_empty[o], 1);
    }
    for (int b = 0; b < kIssuers; ++b) {
      dev::mbar_init(&d_full[b], 1);
      dev::mbar_init(&d_empty[b], 4);
    }
    *abort = 0;
    dev::fence_mbar_init();
  }
  if (warp == 1) {
    dev::tmem_alloc(tmem_slot, S::TMEM_COLS);
    dev::tmem_relinquish();
  }
  dev::tc_fence_before();
  __syncthreads();
  dev::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  int64_t nchunks_mine = 0;
  for (int64_t c = blockIdx.x; c < p.num_chunks; c += G) ++nchunks_mine;

  double acc[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) acc[j] = 0.0;

  if (warp == 0) {
    // ---------------- TMA producer (lane 0)
    if (lane == 0 && nchunks_mine > 0) {
      dev::prefetch_tensormap(&args.ta);
      dev::prefetch_tensormap(&args.tb);
    }
    const uint64_t policy = dev::policy_evict_first();
    for (int64_t it = 0; it < nchunks_mine; ++it) {
      const int s = static_cast<int>(it % S::RAW_STAGES);
      bool ok = true;
      if (lane == 0) {
        if (it >= S::RAW_STAGES)
          ok = dev::mbar_wait(&raw_empty[s], static_cast<uint32_t>(((it / S::RAW_STAGES) - 1) & 1), abort);
        if (ok) {
          unsigned char* st = smem + S::RAW_OFFSET + s * kRawStageBytes;
          const int y = static_cast<int>((blockIdx.x + it * G) * kRows);
          dev::mbar_arrive_expect_tx(&raw_full[s], kRawStageBytes);
          dev::tma_load_2d(st, &args.ta, 0, y, &raw_full[s], policy);
          dev::tma_load_2d(st + kRawTile, &args.tb, 0, y, &raw_full[s], policy);
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else if (warp == 1 || warp >= 14) {
    // ---------------- MMA issuers (lane 0): issuer r (warp 1, then 14, 15)
    // takes the chunks it = r mod 3; the warp stays converged.
    const uint32_t base = dev::smem_u32(smem + S::OP_OFFSET);
    const int64_t first = warp == 1 ? 0 : warp - 13;
    for (int64_t it = first; it < nchunks_mine; it += kIssuers) {
      const int o = static_cast<int>(it % kOpStages);
      const int b = static_cast<int>(it % kIssuers);
      const int64_t j = it / kIssuers;  // this issuer's j-th chunk; group j / kFlush
      const bool group_first = j % kFlush == 0;
      const bool group_last = j % kFlush == kFlush - 1 || it + kIssuers >= nchunks_mine;
      bool ok = true;
      if (lane == 0) {
        ok = dev::mbar_wait(&op_full[o], static_cast<uint32_t>((it / kOpStages) & 1), abort);
        if (ok && group_first && j >= kFlush)
          ok = dev::mbar_wait(&d_empty[b], static_cast<uint32_t>(((j / kFlush) - 1) & 1), abort);
        if (ok) {
          dev::tc_fence_after();
          const uint32_t a_base = base + o * S::OP_STAGE;
          const uint32_t b_base = a_base + S::OP_TILE;
#pragma unroll
          for (int ks = 0; ks < kRows / 16; ++ks) {
            const uint64_t ad = dev::umma_smem_desc(a_base + 32 * ks, 16, 1024, 2);
            const uint64_t bd = dev::umma_smem_desc(b_base + 32 * ks, 16, 1024, 2);
            dev::umma_bf16(tmem + b * kAccCols, ad, bd, S::IDESC, (ks > 0 || !group_first) ? 1u : 0u);
          }
          dev::umma_commit(&op_empty[o]);  // the operand stage may be rewritten once these MMAs are done
          if (group_last) dev::umma_commit(&d_full[b]);
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else if (warp < kEpiWarp0) {
    // ---------------- converters: warp cw splits 8 rows (row group cw) of
    // A and of B; lane = column.
    const int cw = warp - 2;
    for (int64_t it = 0; it < nchunks_mine; ++it) {
      const int s = static_cast<int>(it % S::RAW_STAGES);
      const int o = static_cast<int>(it % kOpStages);
      bool ok = dev::mbar_wait(&raw_full[s], static_cast<uint32_t>((it / S::RAW_STAGES) & 1), abort);
      if (ok && it >= kOpStages)
        ok = dev::mbar_wait(&op_empty[o], static_cast<uint32_t>(((it / kOpStages) - 1) & 1), abort);
      if (!ok) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      const float* raw = reinterpret_cast<const float*>(smem + S::RAW_OFFSET + s * kRawStageBytes);
      unsigned char* op = smem + S::OP_OFFSET + o * S::OP_STAGE;
#pragma unroll
      for (int which = 0; which < 2; ++which) {
        const float* src = raw + which * (kRows * 32) + (8 * cw) * 32 + lane;
        float x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = src[32 * i];
        unsigned char* dst = op + which * S::OP_TILE;
        const uint32_t chunk = static_cast<uint32_t>((cw ^ (lane & 7)) << 4);
#pragma unroll
        for (int part = 0; part < PARTS; ++part) {
          uint32_t w[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            w[i] = pack_bf16x2(x[2 * i], x[2 * i + 1]);
            if (part + 1 < PARTS) {  // what is left (exact in FP32)
              x[2 * i] -= bf16_lo_f32(w[i]);
              x[2 * i + 1] -= bf16_hi_f32(w[i]);
            }
          }
          *reinterpret_cast<uint4*>(dst + (32 * part + lane) * 128 + chunk) = make_uint4(w[0], w[1], w[2], w[3]);
        }
      }
      dev::fence_proxy_async_smem();  // make the operand tiles visible to the tensor core
      __syncwarp();
      if (lane == 0) {
        dev::mbar_arrive(&op_full[o]);
        dev::mbar_arrive(&raw_empty[s]);
      }
    }
  } else {
    // ---------------- epilogue: warp w reads TMEM lanes 32 w .. +31 = A's part w
    // Drains in (group, issuer) order: issuer b's g-th group of kFlush
    // chunks is complete at phase g of d_full[b].
    const int q = warp & 3;
    const uint32_t lane_base = static_cast<uint32_t>(32 * q) << 16;
    int64_t groups[kIssuers];
    int64_t max_groups = 0;
    for (int b = 0; b < kIssuers; ++b) {
      const int64_t nb = nchunks_mine > b ? (nchunks_mine - b + kIssuers - 1) / kIssuers : 0;
      groups[b] = (nb + kFlush - 1) / kFlush;
      max_groups = groups[b] > max_groups ? groups[b] : max_groups;
    }
    bool ok = true;
    for (int64_t g = 0; g < max_groups && ok; ++g) {
      for (int b = 0; b < kIssuers; ++b) {
        if (g >= groups[b]) continue;
        if (!dev::mbar_wait(&d_full[b], static_cast<uint32_t>(g & 1), abort)) {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
          ok = false;
          break;
        }
        dev::tc_fence_after();
        if (q < PARTS) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            uint32_t v[PARTS][16];
#pragma unroll
            for (int pb = 0; pb < PARTS; ++pb) dev::tmem_ld16(tmem + lane_base + b * kAccCols + 32 * pb + 16 * h, v[pb]);
            dev::tmem_ld_wait();
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              float sum = __uint_as_float(v[PARTS - 1][j]);  // B's smallest part first
#pragma unroll
              for (int pb = PARTS - 2; pb >= 0; --pb) sum += __uint_as_float(v[pb][j]);
              acc[16 * h + j] += static_cast<double>(sum);
            }
          }
        }
        dev::tc_fence_before();
        __syncwarp();
        if (lane == 0) dev::mbar_arrive(&d_empty[b]);
      }
    }
  }

  __syncthreads();
  if (*abort && lane == 0) {
    // Bounded drains: tensor loads still landing (producer), MMAs still
    // running (issuer warp 1 waits for every accumulator).  A second timeout
    // is only recorded.
    volatile int no_abort = 0;
    if (warp == 0) {
      for (int64_t it = nchunks_mine > S::RAW_STAGES ? nchunks_mine - S::RAW_STAGES : 0; it < nchunks_mine; ++it)
        if (!dev::mbar_wait(&raw_full[it % S::RAW_STAGES], static_cast<uint32_t>((it / S::RAW_STAGES) & 1), &no_abort))
          break;
    } else if (warp == 1) {
      for (int b = 0; b < kIssuers; ++b) {
        const int64_t nb = nchunks_mine > b ? (nchunks_mine - b + kIssuers - 1) / kIssuers : 0;
        const int64_t gb = (nb + kFlush - 1) / kFlush;
        if (gb > 0 && !dev::mbar_wait(&d_full[b], static_cast<uint32_t>((gb - 1) & 1), &no_abort)) break;
      }
    }
  }
  dev::tc_fence_before();
  __syncthreads();
  dev::tc_fence_after();
  if (warp == 1) dev::tmem_dealloc(tmem, S::TMEM_COLS);

  // CTA partial: epilogue warp w (A's part w) -> red slot w; then C[i][j] =
  // sum over parts, smallest first.
  double* red = reinterpret_cast<double*>(smem);
  if (warp >= kEpiWarp0 && warp < kEpiWarp0 + 4 && (warp & 3) < PARTS) {
#pragma unroll
    for (int j = 0; j < 32; ++j) red[((warp & 3) * 32 + lane) * 32 + j] = acc[j];
  }
  __syncthreads();
  const int m = p.m, k = p.k, mk = m * k;
  double* mine = p.partials + static_cast<int64_t>(blockIdx.x) * mk;
  for (int e = t; e < mk; e += kThreads) {
    const int i = e / k, j = e - (e / k) * k;
    double v = 0.0;
#pragma unroll
    for (int w = PARTS - 1; w >= 0; --w) v += red[(w * 32 + i) * 32 + j];
    mine[e] = v;
  }
  split_finish_ctas(p, t, kThreads, s_is_last);
}

}  // namespace tsm
