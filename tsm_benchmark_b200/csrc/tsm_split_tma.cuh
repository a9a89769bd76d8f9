// tsm_split_tma.cuh -- the precision form (FP32 storage, C = A^T B in FP64,
// m, k <= 32) for widths and row pitches that are multiples of 4 floats.
//
// Same arithmetic as tsm_split.cuh -- x = hi + lo with two TF32 parts, one
// tcgen05.mma (kind::tf32, M = 64 = [A_hi ; A_lo], N = 64 = [B_hi | B_lo],
// K = 8 rows) per 8 rows, FP32 accumulation in tensor memory for DRAIN
// chunks of one issuer, FP64 beyond -- with a leaner data path:
//   * the producer loads 128-row chunks of A and B with 2-D tiled TMA
//     (tensor maps with CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, box 32 columns x
//     128 rows): the raw FP32 tile lands directly in the MN-major layout that
//     tcgen05.mma reads for 32-bit operands (4-row x 128-byte atoms, 32-byte
//     chunks swizzled by row), columns beyond m and rows beyond n zero-filled;
//   * the tensor core reads that raw tile as the hi part -- a TF32 operand is
//     the FP32 bit pattern with its 13 low mantissa bits ignored, so
//     hi = trunc_tf32(x) costs nothing;
//   * converter warps write only lo = rna_tf32(x - trunc_tf32(x)) (x - hi is
//     exact), elementwise at the same offset of a parallel tile: no address
//     arithmetic, 16-byte loads and stores, integer rounding (no conversion
//     instructions).  |x - hi - lo| <= 2^-21 |x|.
// Shared memory: a ring of hi stages (A_hi | B_hi, 16 KB each) that the TMA
// unit fills -- a stage stays busy until its MMAs complete, so its depth is
// what keeps bytes in flight -- and, after it, a shallower ring of lo stages
// (A_lo | B_lo).  Each chunk's descriptors carry the distance from its hi
// stage to its lo stage as the leading byte offset (LBO) between the hi and
// lo atoms of an operand.
//
// Warp roles (16 warps): 0 producer, 1-3 MMA issuers of chunks 0, 3, 6 ..,
// 1, 4 .. and 2, 5 .. (warp 1 also owns TMEM; issuing tcgen05.mma from one
// thread was a measured bottleneck: 2^25 x 32 x 32 took 1.79 ms with one
// issuer, 1.56 with two, 1.53 with three; each issuer owns one lo stage and
// one TMEM accumulator, so they share no barrier phase), 4-11 converters,
// 12-15 epilogue (TMEM -> FP64 sums).  A fourth issuer does not pay: with 17
// warps the register cap (96) spills the epilogue sums, and with the
// converters halved to make room (13 warps) the form ran 1.91 ms,
// converter-bound.  All waits are bounded (dev::mbar_wait); on a timeout the
// CTA records the error, drains its copies and MMAs (bounded) and frees its
// TMEM.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"
#include "tsm_split.cuh"

namespace tsm {

struct SplitTmaArgs {
  SplitArgs p;
  CUtensorMap ta;  // A: {m, n} FP32, box {32, 128}, 128-byte swizzle with 32-byte atoms
  CUtensorMap tb;  // B: {k, n} FP32, same boxes
};

namespace split2 {

// Constants of the kernel for chunks of ROWS rows (ROWS / 8 MMAs of K = 8)
// and ISSUERS MMA-issuing warps.
template <int ROWS, int ISSUERS = 3>
struct Cfg {
  static constexpr int kRows = ROWS;
  // kIssuers warps issue the MMAs (chunk it goes to issuer it % kIssuers);
  // each owns one lo stage and one TMEM accumulator.
  static constexpr int kIssuers = ISSUERS;
  static constexpr int kTileBytes = kRows * 128;      // one operand part: 32 floats x kRows rows
  static constexpr int kStageBytes = 2 * kTileBytes;  // A part, B part
  static constexpr int kLoStages = kIssuers;
  // hi and lo stages share 224 KB: 4 hi stages of 128 rows, 11 of 64 rows
  static constexpr int kHiStages = (7 * 32768) / kStageBytes - kLoStages;
  static constexpr int kLoRing = kHiStages * kStageBytes;  // offset of the lo ring
  static constexpr int kConvWarps = 8;
  static constexpr int kConvWarp0 = 1 + kIssuers;           // warps: 0 producer, 1 .. kIssuers issuers,
  static constexpr int kEpiWarp0 = kConvWarp0 + kConvWarps;  // then converters, then 4 epilogue warps
  static constexpr int kWarps = kEpiWarp0 + 4;
  static constexpr int kConvJobs = 2 * kTileBytes / 16 / (32 * kConvWarps);  // 16-byte vectors per converter thread
  static constexpr int kThreads = kWarps * 32;
  static constexpr int kTmemCols = kIssuers * 64 <= 128 ? 128 : 256;  // one 64-column accumulator per issuer
  static constexpr size_t kBarOffset = size_t(kLoRing) + size_t(kLoStages) * kStageBytes;
  static constexpr int kNumBars = 2 * kHiStages + 2 * kLoStages + 2 * kIssuers;
  static constexpr size_t kSmemBytes = kBarOffset + kNumBars * 8 + 32 + 1024;  // + alignment slack
  static_assert(kHiStages >= 2, "at least a double-buffered hi ring");
  static_assert(kConvJobs * 32 * kConvWarps * 16 == 2 * kTileBytes, "converters cover the stage exactly");
  static_assert(kTileBytes % 1024 == 0, "tiles keep the 1024-byte alignment of the swizzle atoms");
  static_assert((kLoRing + (kLoStages - 1) * kStageBytes) / 16 < (1 << 14), "LBO must fit the descriptor field");
  static_assert(kSmemBytes <= 232448, "dynamic shared memory limit of sm_100a");
  static_assert(kWarps <= 16, "17 warps cap registers at 96 a thread and spill the epilogue sums");
};

constexpr uint32_t kIdesc = dev::umma_idesc_tf32(64, 64, true, true);

// lo part of x: x - trunc_tf32(x) (exact) rounded to nearest TF32, ties away
// from zero (add half a TF32 unit to the magnitude bits, clear 13 bits).
__device__ __forceinline__ uint32_t lo_part(uint32_t xb) {
  const float x = __uint_as_float(xb);
  const float hi = __uint_as_float(xb & 0xFFFFE000u);
  const uint32_t rb = __float_as_uint(x - hi);
  return (rb + 0x1000u) & 0xFFFFE000u;
}

}  // namespace split2

// DRAIN: chunks of one issuer accumulated in its TMEM accumulator before the
// epilogue drains it (FP32 accumulation over DRAIN * ROWS rows).
template <int ROWS, int DRAIN, int ISSUERS = 3>
__global__ void __launch_bounds__(split2::Cfg<ROWS, ISSUERS>::kThreads, 1)
    tsm_tn_split_tf32_tma_kernel(const __grid_constant__ SplitTmaArgs args) {
  using S = split2::Cfg<ROWS, ISSUERS>;
  static_assert(DRAIN >= 1, "at least one chunk per drain");
  using split2::kIdesc;
  using split2::lo_part;
  constexpr int kRows = S::kRows, kIssuers = S::kIssuers, kTileBytes = S::kTileBytes;
  constexpr int kStageBytes = S::kStageBytes, kLoStages = S::kLoStages, kHiStages = S::kHiStages;
  constexpr int kLoRing = S::kLoRing, kConvWarps = S::kConvWarps, kConvWarp0 = S::kConvWarp0;
  constexpr int kEpiWarp0 = S::kEpiWarp0, kConvJobs = S::kConvJobs, kThreads = S::kThreads;
  constexpr int kTmemCols = S::kTmemCols, kNumBars = S::kNumBars;
  constexpr size_t kBarOffset = S::kBarOffset;
  const SplitArgs& p = args.p;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024u - (dev::smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kBarOffset);
  uint64_t* full = bars;                     // hi stage landed (TMA transaction count)
  uint64_t* empty = full + kHiStages;        // hi stage's MMAs completed (commit)
  uint64_t* lo_full = empty + kHiStages;     // lo stage written (converter warps)
  uint64_t* lo_empty = lo_full + kLoStages;  // lo stage's MMAs completed (commit)
  uint64_t* d_full = lo_empty + kLoStages;   // accumulator b complete (commit)
  uint64_t* d_empty = d_full + kIssuers;     // accumulator b drained (epilogue warps)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kNumBars);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  unsigned* s_is_last = reinterpret_cast<unsigned*>(tmem_slot + 2);

  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  const int64_t G = gridDim.x;

  if (t == 0) {
    for (int s = 0; s < kHiStages; ++s) {
      dev::mbar_init(&full[s], 1);
      dev::mbar_init(&empty[s], 1);
    }
    for (int o = 0; o < kLoStages; ++o) {
      dev::mbar_init(&lo_full[o], kConvWarps);
      dev::mbar_init(&lo_empty[o], 1);
    }
    for (int b = 0; b < kIssuers; ++b) {
      dev::mbar_init(&d_full[b], 1);
      dev::mbar_init(&d_empty[b], 4);
    }
    *abort = 0;
    dev::fence_mbar_init();
  }
  if (warp == 1) {
    dev::tmem_alloc(tmem_slot, kTmemCols);
    dev::tmem_relinquish();
  }
  dev::tc_fence_before();
  __syncthreads();
  dev::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  int64_t nchunks_mine = 0;
  for (int64_t c = blockIdx.x; c < p.num_chunks; c += G) ++nchunks_mine;
  // Chunk it belongs to issuer (and accumulator) it % kIssuers, as that
  // issuer's chunk j = it / kIssuers, in drain group j / DRAIN; the group's
  // last chunk (or the issuer's last) hands the accumulator to the epilogue.
  auto ends_group = [&](int64_t it) {
    return (it / kIssuers) % DRAIN == DRAIN - 1 || it + kIssuers >= nchunks_mine;
  };

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
      const int s = static_cast<int>(it % kHiStages);
      bool ok = true;
      if (lane == 0) {
        if (it >= kHiStages)
          ok = dev::mbar_wait(&empty[s], static_cast<uint32_t>(((it / kHiStages) - 1) & 1), abort);
        if (ok) {
          unsigned char* st = smem + s * kStageBytes;
          const int y = static_cast<int>((blockIdx.x + it * G) * kRows);
          dev::mbar_arrive_expect_tx(&full[s], 2 * kTileBytes);
          dev::tma_load_2d(st, &args.ta, 0, y, &full[s], policy);
          dev::tma_load_2d(st + kTileBytes, &args.tb, 0, y, &full[s], policy);
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else if (warp <= kIssuers) {
    // ---------------- MMA issuers (lane 0): issuer r (warp 1, then 14 ..)
    // takes the chunks it = r mod kIssuers; the warp stays converged.
    const uint32_t base = dev::smem_u32(smem);
    const int64_t first = warp - 1;
    for (int64_t it = first; it < nchunks_mine; it += kIssuers) {
      const int s = static_cast<int>(it % kHiStages);
      const int o = static_cast<int>(it % kLoStages);
      const int b = static_cast<int>(it % kIssuers);
      const int64_t j = it / kIssuers, grp = j / DRAIN;
      const bool group_first = j % DRAIN == 0;
      bool ok = true;
      if (lane == 0) {
        ok = dev::mbar_wait(&lo_full[o], static_cast<uint32_t>((it / kLoStages) & 1), abort);
        if (ok && group_first && grp > 0)
          ok = dev::mbar_wait(&d_empty[b], static_cast<uint32_t>((grp - 1) & 1), abort);
        if (ok) {
          dev::tc_fence_after();
          const uint32_t a_base = base + s * kStageBytes;
          const uint32_t b_base = a_base + kTileBytes;
          const uint32_t lbo = static_cast<uint32_t>(kLoRing + o * kStageBytes - s * kStageBytes);  // hi -> lo
#pragma unroll
          for (int g = 0; g < kRows / 8; ++g) {
            const uint64_t ad = dev::umma_smem_desc(a_base + g * 1024, lbo, split::kSbo, split::kLayout);
            const uint64_t bd = dev::umma_smem_desc(b_base + g * 1024, lbo, split::kSbo, split::kLayout);
            dev::umma_tf32(tmem + b * 64, ad, bd, kIdesc, (g > 0 || !group_first) ? 1u : 0u);
          }
          dev::umma_commit(&empty[s]);     // the hi stage may be refilled once these MMAs are done
          dev::umma_commit(&lo_empty[o]);  // and the lo stage rewritten
          if (ends_group(it)) dev::umma_commit(&d_full[b]);
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else if (warp < kEpiWarp0) {
    // ---------------- converters: lo parts, elementwise at the hi offsets
    const int ct = t - 32 * kConvWarp0;
    for (int64_t it = 0; it < nchunks_mine; ++it) {
      const int s = static_cast<int>(it % kHiStages);
      const int o = static_cast<int>(it % kLoStages);
      bool ok = dev::mbar_wait(&full[s], static_cast<uint32_t>((it / kHiStages) & 1), abort);
      if (ok && it >= kLoStages)
        ok = dev::mbar_wait(&lo_empty[o], static_cast<uint32_t>(((it / kLoStages) - 1) & 1), abort);
      if (!ok) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      const uint4* hi = reinterpret_cast<const uint4*>(smem + s * kStageBytes);
      uint4* lo = reinterpret_cast<uint4*>(smem + kLoRing + o * kStageBytes);
      // A_hi and B_hi: 2 x 16 KB = 2048 16-byte vectors over 256 threads.
#pragma unroll
      for (int q = 0; q < kConvJobs; ++q) {
        const uint4 v = hi[ct + q * 32 * kConvWarps];
        uint4 w;
        w.x = lo_part(v.x);
        w.y = lo_part(v.y);
        w.z = lo_part(v.z);
        w.w = lo_part(v.w);
        lo[ct + q * 32 * kConvWarps] = w;
      }
      dev::fence_proxy_async_smem();  // make the lo tiles visible to the tensor core
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&lo_full[o]);
    }
  } else {
    // ---------------- epilogue: TMEM -> FP64 sums (lanes 0-15 of each warp)
    const int q = warp & 3;
    const uint32_t lane_base = static_cast<uint32_t>(32 * q) << 16;
    for (int64_t it = 0; it < nchunks_mine; ++it) {
      if (!ends_group(it)) continue;
      const int b = static_cast<int>(it % kIssuers);
      if (!dev::mbar_wait(&d_full[b], static_cast<uint32_t>(((it / kIssuers) / DRAIN) & 1), abort)) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      dev::tc_fence_after();
      // Columns 0..31 hold x B_hi, 32..63 x B_lo (below 2^-10 of the former):
      // one FP32 addition, then one conversion to FP64.
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint32_t v[16], u[16];
        dev::tmem_ld16(tmem + lane_base + b * 64 + 16 * h, v);
        dev::tmem_ld16(tmem + lane_base + b * 64 + 32 + 16 * h, u);
        dev::tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j)
          acc[16 * h + j] += static_cast<double>(__uint_as_float(v[j]) + __uint_as_float(u[j]));
      }
      dev::tc_fence_before();
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&d_empty[b]);
    }
  }

  __syncthreads();
  if (*abort && lane == 0) {
    // Bounded drains: tensor loads still landing (producer), MMAs still
    // running (issuer).  A second timeout is only recorded.
    volatile int no_abort = 0;
    if (warp == 0) {
      for (int64_t it = nchunks_mine > kHiStages ? nchunks_mine - kHiStages : 0; it < nchunks_mine; ++it)
        if (!dev::mbar_wait(&full[it % kHiStages], static_cast<uint32_t>((it / kHiStages) & 1), &no_abort)) break;
    } else if (warp == 1) {
      const int64_t span = int64_t(kIssuers) * DRAIN;
      for (int64_t it = nchunks_mine > span ? nchunks_mine - span : 0; it < nchunks_mine; ++it)
        if (ends_group(it) && !dev::mbar_wait(&d_full[it % kIssuers],
                                              static_cast<uint32_t>(((it / kIssuers) / DRAIN) & 1), &no_abort))
          break;
    }
  }
  dev::tc_fence_before();
  __syncthreads();
  dev::tc_fence_after();
  if (warp == 1) dev::tmem_dealloc(tmem, kTmemCols);

  split_finish(p, acc, reinterpret_cast<double*>(smem), t, kThreads, kEpiWarp0, s_is_last);
}

}  // namespace tsm
