// tsm_split.cuh -- the precision form: C (m x k, FP64) = A^T B for FP32-stored
// A (n x m) and B (n x k), m, k <= 32, on the 5th-generation tensor cores.
//
// Every FP32 value x is split into two TF32 parts, hi = rna_tf32(x) and
// lo = rna_tf32(x - hi) (x - hi is exact; |x - hi - lo| <= 2^-23 |x|).  One
// tcgen05.mma (kind::tf32, M = 64, N = 64, K = 8 rows) per 8 rows computes
//     D = [A_hi ; A_lo]^T-stacked  x  [B_hi | B_lo]
// so the four 32 x 32 quadrants of D are hi.hi, hi.lo, lo.hi and lo.lo; their
// sum is C's contribution from those rows, with exact products and FP32
// accumulation inside the tensor core.  Every 128 rows (kFlush chunks) the
// FP32 accumulator is drained from tensor memory into FP64 registers, which
// bounds the FP32 rounding to 128-row partial sums; all later sums (across
// drains, warps and CTAs) are FP64, in a fixed order (deterministic).
//
// Warp roles in one persistent CTA per SM (14 warps):
//   warp 0      TMA producer: raw FP32 row chunks -> raw ring (1-D bulk copies)
//   warp 1      TMEM owner and MMA issuer (one elected thread)
//   warps 2-9   converters: raw chunk -> TF32 hi/lo operand tiles, written in
//               the canonical MN-major layout tcgen05 reads for 32-bit types
//               (128-byte swizzle, 32-byte atomicity: 4 data rows x 128 bytes
//               per 512-byte atom, 32-byte chunks XOR-permuted by row; hi
//               atoms then lo atoms LBO bytes later)
//   warps 10-13 epilogue: tcgen05.ld of the accumulator (double-buffered in
//               TMEM) into FP64 sums; warp w reads TMEM sub-partition w % 4,
//               whose lanes 0-15 hold rows 16 (w % 4) .. +15 of D (M = 64)
// All waits are bounded (dev::mbar_wait); on a timeout the CTA records the
// error, drains its copies and MMAs (bounded) and frees its TMEM.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"
#include "tsm_plain.cuh"

namespace tsm {

struct SplitArgs {
  const float* A;
  const float* B;
  double* C;
  int64_t n;
  int m, k;
  int64_t ldc;
  int accumulate;
  int64_t rows_main;   // rows streamed by the pipeline; the rest (< 4) are added at the end
  int64_t num_chunks;  // ceil(rows_main / kRows)
  double* partials;    // gridDim.x * m * k
  unsigned* counter;
  unsigned* error;
};

namespace split {

constexpr int kRows = 64;         // rows per chunk (8 MMAs of K = 8)
constexpr int kFlush = 2;         // chunks accumulated in one TMEM buffer (128 rows) before a drain
constexpr int kRawStages = 4;
constexpr int kOpStages = 2;
constexpr int kConvWarps = 8;
constexpr int kEpiWarp0 = 10;     // warps 10..13
constexpr int kWarps = 14;
constexpr int kThreads = kWarps * 32;
constexpr int kRawStageBytes = 2 * kRows * 32 * 4;          // A and B, 32 floats per row (capacity)
constexpr int kOpHalfBytes = kRows * 128;                   // one part (hi or lo) of one operand
constexpr int kOpStageBytes = 4 * kOpHalfBytes;             // A hi, A lo, B hi, B lo
constexpr int kTmemCols = 128;                              // two 64-column accumulators
constexpr uint32_t kIdesc = dev::umma_idesc_tf32(64, 64, true, true);
// Shared memory map (operand ring first: 1024-byte aligned atoms).
constexpr size_t kOpOffset = 0;
constexpr size_t kRawOffset = kOpOffset + size_t(kOpStages) * kOpStageBytes;
constexpr size_t kBarOffset = kRawOffset + size_t(kRawStages) * kRawStageBytes;
constexpr int kNumBars = 2 * kRawStages + 2 * kOpStages + 4;
constexpr size_t kSmemBytes = kBarOffset + kNumBars * 8 + 32 + 1024;  // + alignment slack

// Byte offset, inside one part of one operand, of the 16-byte chunk c of data
// row r.  MN-major TF32 operands of tcgen05.mma use the 128-byte swizzle with
// 32-byte atomicity (layout type SWIZZLE_128B_BASE32B): atoms of 4 rows x
// 128 B (512 B, consecutive along K, so SBO = 512), the 32-byte chunk index
// XOR-ed with the row inside the atom.
constexpr uint32_t kLayout = 1;  // SWIZZLE_128B_BASE32B
constexpr uint32_t kSbo = 512;
__device__ __forceinline__ uint32_t op_offset(int r, int c) {
  return static_cast<uint32_t>((r >> 2) * 512 + (r & 3) * 128 + (((c >> 1) ^ (r & 3)) << 5) + ((c & 1) << 4));
}

}  // namespace split

// The end of both split kernels: the epilogue warps' FP64 sums (warps
// epi0..epi0+3, lanes 0-15: D row 16 (w % 4) + lane, 32 columns) -> `red`
// (16 KB of shared memory no longer in use), the CTA's m x k partial (D rows
// i and 32 + i -- the hi and lo parts of A's column i -- added) into the
// workspace, and the last CTA's fixed-order sum over CTAs (plus the rows
// [rows_main, n) the pipeline left) into C.
__device__ __forceinline__ void split_finish_ctas(const SplitArgs& p, int t, int nthreads, unsigned* s_is_last);

__device__ __forceinline__ void split_finish(const SplitArgs& p, const double (&acc)[32], double* red, int t,
                                             int nthreads, int epi0, unsigned* s_is_last) {
  const int warp = t >> 5, lane = t & 31;
  const int m = p.m, k = p.k;
  if (warp >= epi0 && warp < epi0 + 4 && lane < 16) {
    const int q = warp & 3;
#pragma unroll
    for (int j = 0; j < 32; ++j) red[(q * 16 + lane) * 32 + j] = acc[j];
  }
  __syncthreads();
  const int mk = m * k;
  double* mine = p.partials + static_cast<int64_t>(blockIdx.x) * mk;
  for (int e = t; e < mk; e += nthreads) {
    const int i = e / k, j = e - (e / k) * k;
    // row i of C: hi part in D row i (sub-partition i / 16), lo part in row 32 + i.
    const int hi_slot = (i >> 4) * 16 + (i & 15);
    const int lo_slot = (2 + (i >> 4)) * 16 + (i & 15);
    mine[e] = red[hi_slot * 32 + j] + red[lo_slot * 32 + j];
  }
  split_finish_ctas(p, t, nthreads, s_is_last);
}

// The CTA's partial is in the workspace (slot blockIdx.x): count the CTA in,
// and the last one sums the CTA partials in CTA order (plus the rows
// [rows_main, n) the pipeline left) into C.
__device__ __forceinline__ void split_finish_ctas(const SplitArgs& p, int t, int nthreads, unsigned* s_is_last) {
  const int m = p.m, k = p.k;
  const int mk = m * k;
  __threadfence();
  __syncthreads();
  if (t == 0) {
    const unsigned prev = atomicAdd(p.counter, 1u);
    *s_is_last = (prev == gridDim.x - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (*s_is_last == 0u) return;
  __threadfence();
  const int64_t G = gridDim.x;
  for (int e = t; e < mk; e += nthreads) {
    const int i = e / k, j = e - (e / k) * k;
    double s = dev::ld_cg(p.partials + e);
    for (int64_t b = 1; b < G; ++b) s += dev::ld_cg(p.partials + b * mk + e);
    for (int64_t r = p.rows_main; r < p.n; ++r)
      s += static_cast<double>(p.A[r * m + i]) * static_cast<double>(p.B[r * k + j]);
    double* c = p.C + static_cast<int64_t>(i) * p.ldc + j;
    *c = p.accumulate ? *c + s : s;
  }
  if (t == 0) *p.counter = 0u;
}

__global__ void __launch_bounds__(split::kThreads, 1) tsm_tn_split_tf32_kernel(const SplitArgs p) {
  using namespace split;
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte alignment for the swizzle atoms.
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char* op_ring = smem + kOpOffset;
  unsigned char* raw_ring = smem + kRawOffset;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kBarOffset);
  uint64_t* raw_full = bars;
  uint64_t* raw_empty = raw_full + kRawStages;
  uint64_t* op_full = raw_empty + kRawStages;
  uint64_t* op_empty = op_full + kOpStages;
  uint64_t* d_full = op_empty + kOpStages;
  uint64_t* d_empty = d_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kNumBars);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  unsigned* s_is_last = reinterpret_cast<unsigned*>(tmem_slot + 2);

  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  const int m = p.m, k = p.k;
  const int64_t G = gridDim.x;

  if (t == 0) {
    for (int s = 0; s < kRawStages; ++s) {
      dev::mbar_init(&raw_full[s], 1);
      dev::mbar_init(&raw_empty[s], kConvWarps);
    }
    for (int s = 0; s < kOpStages; ++s) {
      dev::mbar_init(&op_full[s], kConvWarps);
      dev::mbar_init(&op_empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
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

  double acc[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) acc[j] = 0.0;

  if (warp == 0) {
    // ---------------- TMA producer
    const uint64_t policy = dev::policy_evict_first();
    for (int64_t it = 0; it < nchunks_mine; ++it) {
      const int64_t c = blockIdx.x + it * G;
      const int s = static_cast<int>(it % kRawStages);
      bool ok = true;
      if (lane == 0) {
        if (it >= kRawStages)
          ok = dev::mbar_wait(&raw_empty[s], static_cast<uint32_t>(((it / kRawStages) - 1) & 1), abort);
        if (ok) {
          const int64_t r0 = c * kRows;
          const int64_t rows = (p.rows_main - r0) < kRows ? (p.rows_main - r0) : kRows;
          const uint32_t ba = static_cast<uint32_t>(rows * m * 4), bb = static_cast<uint32_t>(rows * k * 4);
          unsigned char* st = raw_ring + s * kRawStageBytes;
          dev::mbar_arrive_expect_tx(&raw_full[s], ba + bb);
          dev::bulk_g2s_evict_first(st, p.A + r0 * m, ba, &raw_full[s], policy);
          dev::bulk_g2s_evict_first(st + kRows * 32 * 4, p.B + r0 * k, bb, &raw_full[s], policy);
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (lane 0); the warp stays converged.
    const uint32_t op_base = dev::smem_u32(op_ring);
    for (int64_t it = 0; it < nchunks_mine; ++it) {
      const int o = static_cast<int>(it % kOpStages);
      const int64_t grp = it / kFlush;  // accumulator group: kFlush chunks into one TMEM buffer
      const int b = static_cast<int>(grp & 1);
      const bool first = (it % kFlush) == 0;
      const bool last = (it % kFlush) == kFlush - 1 || it == nchunks_mine - 1;
      bool ok = true;
      if (lane == 0) {
        ok = dev::mbar_wait(&op_full[o], static_cast<uint32_t>((it / kOpStages) & 1), abort);
        if (ok && first && grp >= 2)
          ok = dev::mbar_wait(&d_empty[b], static_cast<uint32_t>(((grp >> 1) - 1) & 1), abort);
        if (ok) {
          dev::tc_fence_after();
          const uint32_t a_base = op_base + o * kOpStageBytes;
          const uint32_t b_base = a_base + 2 * kOpHalfBytes;
#pragma unroll
          for (int g = 0; g < kRows / 8; ++g) {
            const uint64_t ad = dev::umma_smem_desc(a_base + g * 1024, kOpHalfBytes, kSbo, kLayout);
            const uint64_t bd = dev::umma_smem_desc(b_base + g * 1024, kOpHalfBytes, kSbo, kLayout);
            dev::umma_tf32(tmem + b * 64, ad, bd, kIdesc, (first && g == 0) ? 0u : 1u);
          }
          dev::umma_commit(&op_empty[o]);      // operands may be overwritten once these MMAs are done
          if (last) dev::umma_commit(&d_full[b]);  // accumulator b holds its group's rows
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else if (warp < kEpiWarp0) {
    // ---------------- converters: raw FP32 -> TF32 hi / lo operand tiles
    const int ct = t - 64;  // 0 .. 255
    for (int64_t it = 0; it < nchunks_mine; ++it) {
      const int64_t c = blockIdx.x + it * G;
      const int s = static_cast<int>(it % kRawStages);
      const int o = static_cast<int>(it % kOpStages);
      bool ok = dev::mbar_wait(&raw_full[s], static_cast<uint32_t>((it / kRawStages) & 1), abort);
      if (ok && it >= kOpStages)
        ok = dev::mbar_wait(&op_empty[o], static_cast<uint32_t>(((it / kOpStages) - 1) & 1), abort);
      if (!ok) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      const int64_t r0 = c * kRows;
      const int rows = static_cast<int>((p.rows_main - r0) < kRows ? (p.rows_main - r0) : kRows);
      const float* rawA = reinterpret_cast<const float*>(raw_ring + s * kRawStageBytes);
      const float* rawB = rawA + kRows * 32;
      unsigned char* opA = op_ring + o * kOpStageBytes;
      unsigned char* opB = opA + 2 * kOpHalfBytes;
      // 2 operands x 64 rows x 8 chunks = 1024 chunk jobs over 256 threads.
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int job = ct + q * 256;
        const int which = job >> 9;  // 0: A, 1: B
        const int r = (job >> 3) & 63;
        const int ch = job & 7;
        const int w = which ? k : m;
        const float* src = (which ? rawB : rawA) + r * w;
        float x[4];
        if (w == 32 && r < rows) {
          const float4 v = reinterpret_cast<const float4*>(src)[ch];
          x[0] = v.x;
          x[1] = v.y;
          x[2] = v.z;
          x[3] = v.w;
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) x[e] = (r < rows && 4 * ch + e < w) ? src[4 * ch + e] : 0.0f;
        }
        float4 hi, lo;
        hi.x = dev::to_tf32(x[0]);
        hi.y = dev::to_tf32(x[1]);
        hi.z = dev::to_tf32(x[2]);
        hi.w = dev::to_tf32(x[3]);
        lo.x = dev::to_tf32(x[0] - hi.x);
        lo.y = dev::to_tf32(x[1] - hi.y);
        lo.z = dev::to_tf32(x[2] - hi.z);
        lo.w = dev::to_tf32(x[3] - hi.w);
        unsigned char* dst = (which ? opB : opA) + split::op_offset(r, ch);
        *reinterpret_cast<float4*>(dst) = hi;
        *reinterpret_cast<float4*>(dst + kOpHalfBytes) = lo;
      }
      dev::fence_proxy_async_smem();  // make the operand stores visible to the tensor core
      __syncwarp();
      if (lane == 0) {
        dev::mbar_arrive(&raw_empty[s]);
        dev::mbar_arrive(&op_full[o]);
      }
    }
  } else {
    // ---------------- epilogue: TMEM -> FP64 sums (lanes 0-15 of each warp)
    const int q = warp & 3;
    const uint32_t lane_base = static_cast<uint32_t>(32 * q) << 16;
    const int64_t ngroups = (nchunks_mine + kFlush - 1) / kFlush;
    for (int64_t grp = 0; grp < ngroups; ++grp) {
      const int b = static_cast<int>(grp & 1);
      if (!dev::mbar_wait(&d_full[b], static_cast<uint32_t>((grp >> 1) & 1), abort)) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      dev::tc_fence_after();
      // Columns 0..31 hold x B_hi, 32..63 x B_lo (~2^-11 of the former): one
      // FP32 addition, then one conversion to FP64.
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
    // Bounded drains: copies still landing (producer), MMAs still running
    // (issuer).  A second timeout is only recorded.
    volatile int no_abort = 0;
    if (warp == 0) {
      for (int64_t it = nchunks_mine > kRawStages ? nchunks_mine - kRawStages : 0; it < nchunks_mine; ++it)
        if (!dev::mbar_wait(&raw_full[it % kRawStages], static_cast<uint32_t>((it / kRawStages) & 1), &no_abort))
          break;
    } else if (warp == 1) {
      const int64_t ngroups = (nchunks_mine + kFlush - 1) / kFlush;
      for (int64_t grp = ngroups > 2 ? ngroups - 2 : 0; grp < ngroups; ++grp)
        if (!dev::mbar_wait(&d_full[grp & 1], static_cast<uint32_t>((grp >> 1) & 1), &no_abort)) break;
    }
  }
  dev::tc_fence_before();
  __syncthreads();
  dev::tc_fence_after();
  if (warp == 1) dev::tmem_dealloc(tmem, kTmemCols);

  split_finish(p, acc, reinterpret_cast<double*>(raw_ring), t, kThreads, kEpiWarp0, s_is_last);
}

}  // namespace tsm
