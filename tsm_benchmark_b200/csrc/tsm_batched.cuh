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
//     problem's width class (m, k in {4, 8, 16, 32}) -- exact register
//     tiles, 16-byte rotated shared-memory loads -- and at the segment's end
//     reduce their tiles (warp shuffles, then a fixed-order sum over warps in
//     a shared-memory buffer separate from the ring) into the segment's FP64
//     partial;
//   * a per-problem counter finds the last segment of a problem to finish;
//     that CTA sums the problem's partials in segment order and writes C_p.
// Results are deterministic for a given plan; there are no atomics on data.
#pragma once

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
  int pad;
};

struct BatchedSegmentDev {
  int problem;
  int pad;
  int64_t r0, r1;       // rows [r0, r1) of the problem
  int64_t partial_off;  // doubles from the start of the partials area
};

struct BatchedArgs {
  const BatchedProblemDev* problems;
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
// Largest slots x m x k doubles over the classes: 8 x 16 x 32 (and 4 x 32 x 32).
constexpr int kRedBytes = 32768;
constexpr size_t kBarOffset = size_t(kStages) * kStageBytes + kRedBytes;
constexpr size_t kSmemBytes = kBarOffset + 2 * kStages * sizeof(uint64_t) + 16;

// 4 x 4 register tiles for every class: sixteen inlined class paths share
// one register budget, which nine warps per CTA cap at 168 per thread (three
// warps on one SM sub-partition); larger tiles would spill.
__host__ __device__ constexpr int tile_of(int) { return 4; }

// Rows per chunk for widths (m, k): ~32 KB stages, whole row-group passes.
__host__ __device__ constexpr int rows_of(int m, int k) {
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
  constexpr int RS = rows_of(M, K);
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

}  // namespace batched

__global__ void __launch_bounds__(batched::kThreads, 1) tsm_tn_batched_kernel(const BatchedArgs a) {
  using namespace batched;
  extern __shared__ __align__(128) unsigned char smem[];
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
      const int rs = rows_of(pr.m, pr.k);
      for (int64_t r0 = seg.r0; r0 < seg.r1 && ok; r0 += rs, ++issued) {
        const int s = static_cast<int>(issued % kStages);
        const int64_t round = issued / kStages;
        if (lane == 0) {
          if (round > 0) ok = dev::mbar_wait(&empty[s], static_cast<uint32_t>((round - 1) & 1), abort);
          if (ok) {
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
      switch (pr.cls) {
        TSM_BATCHED_CASE(4, 4) TSM_BATCHED_CASE(4, 8) TSM_BATCHED_CASE(4, 16) TSM_BATCHED_CASE(4, 32)
        TSM_BATCHED_CASE(8, 4) TSM_BATCHED_CASE(8, 8) TSM_BATCHED_CASE(8, 16) TSM_BATCHED_CASE(8, 32)
        TSM_BATCHED_CASE(16, 4) TSM_BATCHED_CASE(16, 8) TSM_BATCHED_CASE(16, 16) TSM_BATCHED_CASE(16, 32)
        TSM_BATCHED_CASE(32, 4) TSM_BATCHED_CASE(32, 8) TSM_BATCHED_CASE(32, 16) TSM_BATCHED_CASE(32, 32)
        default:
          break;
      }
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
      const int rs = rows_of(pr.m, pr.k);
      issued += (seg.r1 - seg.r0 + rs - 1) / rs;
    }
    volatile int no_abort = 0;
    for (int64_t q = issued > kStages ? issued - kStages : 0; q < issued; ++q)
      if (!dev::mbar_wait(&full[q % kStages], static_cast<uint32_t>((q / kStages) & 1), &no_abort)) break;
  }
}

}  // namespace tsm
