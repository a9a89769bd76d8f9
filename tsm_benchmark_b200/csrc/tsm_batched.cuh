// tsm_batched.cuh -- many independent products C_p = A_p^T B_p in ONE
// persistent launch (the batching form; the reference runs one product per
// kernel submit).
//
// The host plan (tsm_batched.cu) concatenates the problems' rows and cuts
// that sequence into one contiguous byte range per CTA, so every CTA moves
// the same number of bytes.  A CTA's range is a short list of segments
// (problem, first row, end row); consecutive CTAs share at most the problem
// at their boundary.  Inside a CTA:
//   * the producer warp streams every segment's row chunks through one TMA
//     bulk-copy ring (as tsm_plain.cuh), without pausing between segments or
//     problems;
//   * the consumer warps switch, per segment, to the compile-time path of the
//     problem's width class (m, k in {4, 8, 16, 32}) and at the segment's end
//     reduce their tiles (a fixed-order sum over warps in a shared-memory
//     buffer separate from the ring) into the segment's FP64 partial.  Classes
//     with a width below 16 use SIMT register tiles over 1-D bulk copies
//     (16-byte rotated shared-memory loads); classes with m, k in {16, 32} use
//     the FP64 tensor cores (mma.sync m8n8k4 f64) over 2-D tiled TMA loads
//     with the 128-byte swizzle, through two tensor maps per problem kept in
//     the plan, with the fragment choice of tsm_dmma.cuh (conflict-free
//     16-byte loads); rows a box brings in beyond the segment are zeroed in
//     the fragments;
//   * a per-problem counter finds the last segment of a problem to finish;
//     that CTA sums the problem's partials in segment order and writes C_p.
// Results are deterministic for a given plan; there are no atomics on data.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"
#include "tsm_plain.cuh"

namespace tsm {

struct BatchedProblemDev {
  const double* A;
  const double* B;
  double* C;
  int64_t n;
  int m, k;
  int cls;  // width class index (kBatchedClasses order)
  int accumulate;
  int64_t ldc;
  int64_t seg_first;  // index of the problem's first segment
  int nseg;           // number of segments (>= 1)
  int path;           // consumer path of its class: kPathDefault or kPathSimt
};

struct BatchedSegmentDev {
  int problem;
  int pad;
  int64_t r0, r1;       // rows [r0, r1) of the problem
  int64_t partial_off;  // doubles from the start of the partials area
};

struct BatchedArgs {
  const BatchedProblemDev* problems;
  const CUtensorMap* maps;  // 2 per problem (A, B); set for the tensor-core classes
  const BatchedSegmentDev* segments;
  const int* cta_first;  // segments of CTA b: [cta_first[b], cta_first[b + 1])
  unsigned* counters;    // one per problem, zero between launches
  double* partials;
  unsigned* error;
};

namespace batched {

constexpr int kCW = 8;
constexpr int kCT = kCW * 32;
constexpr int kThreads = kCT + 32;
constexpr int kStages = 4;
constexpr int kStageBytes = 32768;
// Largest slots x m x k doubles over the classes: 8 warps x 32 x 32.
constexpr int kRedBytes = 65536;
constexpr size_t kBarOffset = size_t(kStages) * kStageBytes + kRedBytes;
// + 1024: the ring is aligned to 1024 bytes (the swizzle pattern's period).
constexpr size_t kSmemBytes = kBarOffset + 2 * kStages * sizeof(uint64_t) + 16 + 1024;

// Tensor-core classes: both widths 16 or 32.
__host__ __device__ constexpr bool dmma_class(int m, int k) { return m >= 16 && k >= 16; }

// Consumer paths.  Every class has its default path (the FP64 tensor cores
// for the tensor-core classes, SIMT register tiles for the others); the
// tensor-core classes also have the SIMT path (4 x 4 register tiles over 1-D
// bulk copies).  The plan picks one per class: the autotuned table, or the
// caller's override.
constexpr int kPathDefault = 0;
constexpr int kPathSimt = 1;
__host__ __device__ constexpr bool uses_dmma(int m, int k, int path) { return dmma_class(m, k) && path == kPathDefault; }

// 4 x 4 register tiles for every class: sixteen inlined class paths share
// one register budget, which nine warps per CTA cap at 168 per thread (three
// warps on one SM sub-partition); larger tiles would spill.
__host__ __device__ constexpr int tile_of(int) { return 4; }

// Rows per chunk for widths (m, k) on a path: ~32 KB stages.  SIMT paths:
// whole row-group passes.  Tensor-core path: (m + k) / 16 boxes of 128-byte
// rows, rows a multiple of 32 (4-row k-steps split evenly over the 8 warps).
__host__ __device__ constexpr int rows_of(int m, int k, int path = kPathDefault) {
  if (uses_dmma(m, k, path)) return (kStageBytes / (128 * ((m + k) / 16))) / 32 * 32;
  const int nt = (m / tile_of(m)) * (k / tile_of(k));
  const int rg = kCT / nt;
  const int rows = kStageBytes / (8 * (m + k));
  return rows / rg * rg;
}

// Width classes: m, k in {4, 8, 16, 32} -> index 4 * log2(m / 4) + log2(k / 4).
__host__ __device__ constexpr int class_of(int m, int k) {
  auto l = [](int w) { return w == 4 ? 0 : (w == 8 ? 1 : (w == 16 ? 2 : (w == 32 ? 3 : -1))); };
  return (l(m) < 0 || l(k) < 0) ? -1 : 4 * l(m) + l(k);
}

__device__ __forceinline__ void consumer_barrier() { asm volatile("bar.sync 1, %0;" ::"n"(kCT) : "memory"); }

// The end of a segment, after every consumer warp wrote its slot of the
// M x K sheets in `red`: the fixed-order sum over the SLOTS sheets into the
// segment's partial, then, for the problem's last segment to finish, the sum
// of the problem's partials in segment order into C.
template <int M, int K, int SLOTS>
__device__ __forceinline__ void finish_segment(const BatchedArgs& a, const BatchedSegmentDev& seg,
                                               const BatchedProblemDev& pr, double* red, unsigned* s_flag, int t) {
  static_assert(SLOTS * M * K * 8 <= kRedBytes, "reduction buffer too small for this class");
  consumer_barrier();
  double* part = a.partials + seg.partial_off;
  for (int e = t; e < M * K; e += kCT) {
    double sum = red[e];
#pragma unroll
    for (int q = 1; q < SLOTS; ++q) sum += red[q * M * K + e];
    part[e] = sum;
  }
  __threadfence();
  consumer_barrier();
  if (t == 0) {
    const unsigned prev = atomicAdd(a.counters + seg.problem, 1u);
    *s_flag = (prev == static_cast<unsigned>(pr.nseg - 1)) ? 1u : 0u;
  }
  consumer_barrier();
  if (*s_flag) {
    __threadfence();
    const double* base = a.partials + a.segments[pr.seg_first].partial_off;
    for (int e = t; e < M * K; e += kCT) {
      double sum = dev::ld_cg(base + e);
      for (int q = 1; q < pr.nseg; ++q) sum += dev::ld_cg(base + q * M * K + e);
      double* c = pr.C + (e / K) * pr.ldc + (e % K);
      *c = pr.accumulate ? *c + sum : sum;
    }
    if (t == 0) a.counters[seg.problem] = 0u;
  }
}

// Consumes one segment of a (M, K) problem: its chunks from the ring, then
// the CTA reduction into the segment's partial and, for the problem's last
// segment to finish, the final sum into C.
template <int M, int K>
__device__ __forceinline__ void consume_segment(const BatchedArgs& a, const BatchedSegmentDev& seg, const BatchedProblemDev& pr,
                                unsigned char* ring, double* red, uint64_t* full, uint64_t* empty,
                                volatile int* abort, unsigned* s_flag, int64_t& it, int t) {
  constexpr int TA = tile_of(M), TB = tile_of(K);
  using S = TileShape<M, K, TA, TB>;
  constexpr int RG = kCT / S::NT;
  constexpr int RS = rows_of(M, K, kPathSimt);
  constexpr int EPC = 2;
  constexpr bool VEC_A = TA % EPC == 0, VEC_B = TB % EPC == 0;
  constexpr int NCH_A = TA / EPC, NCH_B = TB / EPC;
  constexpr bool ROT_A = NCH_A > 1 && (RG * (M / EPC)) % (8 * NCH_A) == 0;
  constexpr bool ROT_B = NCH_B > 1 && (RG * (K / EPC)) % (8 * NCH_B) == 0;
  const int lane = t & 31;
  const int tile = t % S::NT;
  const int ta = tile % S::QA, tb = tile / S::QA;
  const int rg = t / S::NT;
  const int colA = ta * TA, colB = tb * TB;
  const int rotA = ROT_A ? ((rg * (M / EPC) + colA / EPC) / 8) & (NCH_A - 1) : 0;
  const int rotB = ROT_B ? ((rg * (K / EPC) + colB / EPC) / 8) & (NCH_B - 1) : 0;

  double acc[TA][TB];
#pragma unroll
  for (int i = 0; i < TA; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) acc[i][j] = 0.0;

  for (int64_t r0 = seg.r0; r0 < seg.r1; r0 += RS, ++it) {
    const int s = static_cast<int>(it % kStages);
    if (!*abort && !dev::mbar_wait(&full[s], static_cast<uint32_t>((it / kStages) & 1), abort)) {
      *abort = 1;
      atomicOr(a.error, dev::kErrTimeout);
    }
    if (!*abort) {
      const int rows = static_cast<int>((seg.r1 - r0) < RS ? (seg.r1 - r0) : RS);
      const double* sa = reinterpret_cast<const double*>(ring + s * kStageBytes) + colA;
      const double* sb = reinterpret_cast<const double*>(ring + s * kStageBytes) + RS * M + colB;
      for (int r = rg; r < rows; r += RG) {
        double av[TA], bv[TB];
        detail::load_row_seg<double, TA, VEC_A>(av, sa + r * M, TA, rotA);
        detail::load_row_seg<double, TB, VEC_B>(bv, sb + r * K, TB, rotB);
        detail::outer_fma<TA, TB>(acc, av, bv);
      }
    }
    __syncwarp();
    if (lane == 0) dev::mbar_arrive(&empty[s]);
  }

  // CTA reduction of this segment (consumer threads only; the producer keeps
  // streaming the next segment into the ring meanwhile).
  detail::unrotate_tile<EPC, TA, TB>(acc, rotA, rotB);
  if constexpr (S::NT < 32) {
#pragma unroll
    for (int off = S::NT; off < 32; off <<= 1)
#pragma unroll
      for (int i = 0; i < TA; ++i)
#pragma unroll
        for (int j = 0; j < TB; ++j) acc[i][j] += __shfl_xor_sync(0xffffffffu, acc[i][j], off);
  }
  constexpr int SLOTS = S::NT < 32 ? kCW : RG;
  static_assert(SLOTS * M * K * 8 <= kRedBytes, "reduction buffer too small for this class");
  static_assert(RS * (M + K) * 8 <= kStageBytes && RS > 0, "stage too small for this class");
  consumer_barrier();  // the previous segment's readers of `red` are done
  if (S::NT >= 32 || lane < S::NT) {
    const int slot = S::NT < 32 ? t / 32 : t / S::NT;
    double* dst = red + slot * M * K;
#pragma unroll
    for (int i = 0; i < TA; ++i)
#pragma unroll
      for (int j = 0; j < TB; ++j) dst[(colA + i) * K + colB + j] = acc[i][j];
  }
  finish_segment<M, K, SLOTS>(a, seg, pr, red, s_flag, t);
}

// Consumes one segment of a tensor-core class (M, K in {16, 32}): every warp
// holds all (M/8) x (K/8) 8x8 tiles of C and takes every 8th k-step (4 rows)
// of each chunk; rows at or past the segment's end read as zero.
template <int M, int K>
__device__ __forceinline__ void consume_segment_dmma(const BatchedArgs& a, const BatchedSegmentDev& seg,
                                                     const BatchedProblemDev& pr, unsigned char* ring, double* red,
                                                     uint64_t* full, uint64_t* empty, volatile int* abort,
                                                     unsigned* s_flag, int64_t& it, int t) {
  constexpr int MT = M / 8, NT = K / 8;  // tiles along m and k
  constexpr int MBA = M / 16;            // 16-column blocks of A (B's follow)
  constexpr int RS = rows_of(M, K);
  constexpr int BOX = RS * 128;
  constexpr int KSTEPS = RS / 4;
  static_assert(KSTEPS % kCW == 0, "k-steps must split evenly over the warps");
  static_assert((M / 16 + K / 16) * BOX <= kStageBytes, "stage too small for this class");
  const int warp = t >> 5, lane = t & 31;
  const int g = lane >> 2, tq = lane & 3;
  double acc[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  for (int64_t r0 = seg.r0; r0 < seg.r1; r0 += RS, ++it) {
    const int s = static_cast<int>(it % kStages);
    if (!*abort && !dev::mbar_wait(&full[s], static_cast<uint32_t>((it / kStages) & 1), abort)) {
      *abort = 1;
      atomicOr(a.error, dev::kErrTimeout);
    }
    if (!*abort) {
      const int rows = static_cast<int>((seg.r1 - r0) < RS ? (seg.r1 - r0) : RS);
      const unsigned char* stage = ring + s * kStageBytes;
#pragma unroll 2
      for (int ks = warp; ks < KSTEPS; ks += kCW) {
        const int row = 8 * (ks >> 1) + (ks & 1) + 2 * tq;
        if (8 * (ks >> 1) + (ks & 1) >= rows) break;  // the k-step's first row is past the segment (warp-uniform)
        const int off = row * 128 + ((g ^ (row & 7)) << 4);
        const bool live = row < rows;
        double av[MT], bv[NT];
#pragma unroll
        for (int i = 0; i < MT / 2; ++i) {
          const double2 v = *reinterpret_cast<const double2*>(stage + i * BOX + off);
          av[2 * i] = live ? v.x : 0.0;
          av[2 * i + 1] = live ? v.y : 0.0;
        }
#pragma unroll
        for (int j = 0; j < NT / 2; ++j) {
          const double2 v = *reinterpret_cast<const double2*>(stage + (MBA + j) * BOX + off);
          bv[2 * j] = v.x;
          bv[2 * j + 1] = v.y;
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) dev::dmma_m8n8k4(acc[i][j][0], acc[i][j][1], av[i], bv[j]);
      }
    }
    __syncwarp();
    if (lane == 0) dev::mbar_arrive(&empty[s]);
  }

  consumer_barrier();  // the previous segment's readers of `red` are done
  // Tile (i, j): C row 16 (i / 2) + 2 g + (i & 1), column 16 (j / 2) + 2 (2 tq + e) + (j & 1).
  double* dst = red + warp * M * K;
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int row = 16 * (i >> 1) + 2 * g + (i & 1);
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) dst[row * K + 16 * (j >> 1) + 2 * (2 * tq + e) + (j & 1)] = acc[i][j][e];
  }
  finish_segment<M, K, kCW>(a, seg, pr, red, s_flag, t);
}

}  // namespace batched

// SIMT_TC: the tensor-core classes may take their SIMT path (a plan that
// overrides one uses this instantiation; the default one leaves those paths
// out, which measured 1-5 % faster for the 512-problem batch).
template <bool SIMT_TC>
__global__ void __launch_bounds__(batched::kThreads, 1) tsm_tn_batched_kernel(const BatchedArgs a) {
  using namespace batched;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024u - (dev::smem_u32(smem_raw) & 1023u)) & 1023u);
  unsigned char* ring = smem;
  double* red = reinterpret_cast<double*>(smem + size_t(kStages) * kStageBytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kBarOffset);
  uint64_t* empty = full + kStages;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + kStages);
  unsigned* s_flag = reinterpret_cast<unsigned*>(empty + kStages) + 1;

  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  if (t == 0) {
    for (int s = 0; s < kStages; ++s) {
      dev::mbar_init(&full[s], 1);
      dev::mbar_init(&empty[s], kCW);
    }
    *abort = 0;
    dev::fence_mbar_init();
  }
  __syncthreads();
  const int first = a.cta_first[blockIdx.x], last = a.cta_first[blockIdx.x + 1];

  if (warp == kCW) {
    // ---------------- producer warp: chunks of every segment, in order.
    int64_t issued = 0;
    const uint64_t policy = dev::policy_evict_first();
    bool ok = true;
    for (int si = first; si < last && ok; ++si) {
      const BatchedSegmentDev seg = a.segments[si];
      const BatchedProblemDev& pr = a.problems[seg.problem];
      const int rs = rows_of(pr.m, pr.k, pr.path);
      const bool tc = uses_dmma(pr.m, pr.k, pr.path);
      const CUtensorMap* ta = a.maps + 2 * seg.problem;
      if (tc && lane == 0 && seg.r1 > seg.r0) {
        dev::fence_tensormap_acquire(ta);
        dev::fence_tensormap_acquire(ta + 1);
      }
      for (int64_t r0 = seg.r0; r0 < seg.r1 && ok; r0 += rs, ++issued) {
        const int s = static_cast<int>(issued % kStages);
        const int64_t round = issued / kStages;
        if (lane == 0) {
          if (round > 0) ok = dev::mbar_wait(&empty[s], static_cast<uint32_t>((round - 1) & 1), abort);
          if (ok && tc) {
            // Full 16-column x rs-row boxes (rows past n zero-filled; rows
            // past the segment are masked by the consumers).
            const int mba = pr.m / 16, mbb = pr.k / 16;
            const int box = rs * 128;
            unsigned char* st = ring + s * kStageBytes;
            const int y = static_cast<int>(r0);
            dev::mbar_arrive_expect_tx(&full[s], static_cast<uint32_t>((mba + mbb) * box));
            for (int b = 0; b < mba; ++b) dev::tma_load_2d(st + b * box, ta, 16 * b, y, &full[s], policy);
            for (int b = 0; b < mbb; ++b) dev::tma_load_2d(st + (mba + b) * box, ta + 1, 16 * b, y, &full[s], policy);
          } else if (ok) {
            const int64_t rows = (seg.r1 - r0) < rs ? (seg.r1 - r0) : rs;
            const uint32_t ba = static_cast<uint32_t>(rows * pr.m * sizeof(double));
            const uint32_t bb = static_cast<uint32_t>(rows * pr.k * sizeof(double));
            unsigned char* st = ring + s * kStageBytes;
            dev::mbar_arrive_expect_tx(&full[s], ba + bb);
            dev::bulk_g2s_evict_first(st, pr.A + r0 * pr.m, ba, &full[s], policy);
            dev::bulk_g2s_evict_first(st + size_t(rs) * pr.m * sizeof(double), pr.B + r0 * pr.k, bb, &full[s],
                                      policy);
          } else {
            *abort = 1;
            atomicOr(a.error, dev::kErrTimeout);
          }
        }
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      }
    }
  } else {
    // ---------------- consumer warps: one width-class path per segment.
    int64_t it = 0;
    for (int si = first; si < last; ++si) {
      const BatchedSegmentDev seg = a.segments[si];
      const BatchedProblemDev& pr = a.problems[seg.problem];
#define TSM_BATCHED_CASE(M, K)                                                                          \
  case class_of(M, K):                                                                                  \
    consume_segment<M, K>(a, seg, pr, ring, red, full, empty, abort, s_flag, it, t);                    \
    break;
#define TSM_BATCHED_TC_CASE(M, K)                                                                       \
  case class_of(M, K):                                                                                  \
    if (SIMT_TC && pr.path == kPathSimt)                                                                \
      consume_segment<M, K>(a, seg, pr, ring, red, full, empty, abort, s_flag, it, t);                  \
    else                                                                                                \
      consume_segment_dmma<M, K>(a, seg, pr, ring, red, full, empty, abort, s_flag, it, t);             \
    break;
      switch (pr.cls) {
        TSM_BATCHED_CASE(4, 4) TSM_BATCHED_CASE(4, 8) TSM_BATCHED_CASE(4, 16) TSM_BATCHED_CASE(4, 32)
        TSM_BATCHED_CASE(8, 4) TSM_BATCHED_CASE(8, 8) TSM_BATCHED_CASE(8, 16) TSM_BATCHED_CASE(8, 32)
        TSM_BATCHED_CASE(16, 4) TSM_BATCHED_CASE(16, 8) TSM_BATCHED_TC_CASE(16, 16) TSM_BATCHED_TC_CASE(16, 32)
        TSM_BATCHED_CASE(32, 4) TSM_BATCHED_CASE(32, 8) TSM_BATCHED_TC_CASE(32, 16) TSM_BATCHED_TC_CASE(32, 32)
        default:
          break;
      }
#undef TSM_BATCHED_TC_CASE
#undef TSM_BATCHED_CASE
    }
  }

  __syncthreads();
  if (*abort && warp == kCW && lane == 0) {
    // Bounded drain of the copies this CTA may still have in flight.
    int64_t issued = 0;
    for (int si = first; si < last; ++si) {
      const BatchedSegmentDev seg = a.segments[si];
      const BatchedProblemDev& pr = a.problems[seg.problem];
      const int rs = rows_of(pr.m, pr.k, pr.path);
      issued += (seg.r1 - seg.r0 + rs - 1) / rs;
    }
    volatile int no_abort = 0;
    for (int64_t q = issued > kStages ? issued - kStages : 0; q < issued; ++q)
      if (!dev::mbar_wait(&full[q % kStages], static_cast<uint32_t>((q / kStages) & 1), &no_abort)) break;
  }
}

}  // namespace tsm
