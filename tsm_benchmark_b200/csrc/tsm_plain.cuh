// tsm_plain.cuh -- the plain TSMTTSM kernels, C (m x k) = A^T * B with
// A (n x m) and B (n x k) row-major, stored as T = double or float.
//
// Replaces the nine SYCL kernels of tsmttsm.hh (and the generated ones of
// sycl_codegen*.py).  All of them compute C[i][j] += sum_r A[r][i] * B[r][j]
// with a per-work-item register tile and FP64 atomics into C; here:
//
//   * tsm_tn_bulk_kernel  -- persistent CTAs (one per SM).  A producer warp
//     streams contiguous row chunks of A and B into a STAGES-deep ring of
//     shared-memory buffers with 1-D TMA bulk copies (cp.async.bulk, mbarrier
//     completion, L2 evict-first); CW consumer warps each own a TA x TB
//     register tile of C and walk the chunk's rows.  Needs lda == m,
//     ldb == k and 16-byte aligned A and B.
//   * tsm_tn_direct_kernel -- the same register tiles fed by plain read-only
//     global loads; any lda/ldb and any alignment.
//
// Accumulation: per thread in T (FP64 for double storage, FP32 for float);
// every cross-thread and cross-CTA sum is FP64.  Both kernels end in the same
// deterministic two-level reduction in place of the reference's atomics: warp
// shuffles and a fixed-order shared-memory sum give one m x k FP64 partial per
// CTA, written to the workspace; the last CTA to finish (a counter in the
// workspace) sums the partials in CTA order and writes C.  The result is
// bit-identical from run to run for a given variant and grid.  No value of C
// is ever updated atomically.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"

namespace tsm {

template <typename T>
struct PlainArgs {
  const T* A;
  const T* B;
  T* C;
  int64_t n;  // rows of A and B
  int m;      // columns of A = rows of C
  int k;      // columns of B = columns of C
  int64_t lda, ldb, ldc;
  int accumulate;      // 1: C += A^T B (the reference's semantics), 0: C = A^T B
  int symmetric;       // 1: B is A (m == k): C = A^T A is written from its upper triangle, mirrored
  int64_t rows_main;   // rows covered by the main loop; rows [rows_main, n) are added at the end
  int64_t num_chunks;  // bulk kernel: ceil(rows_main / RS)
  double* partials;    // workspace: gridDim.x * m * k doubles
  unsigned* counter;   // workspace: CTAs finished in this launch (zero between launches)
  unsigned* error;     // workspace: sticky error bits (dev::kErr*)
};

// Compile-time shape of one register-tiled variant.
//   WA, WB : widths (exact) or width capacities (EXACT == false; the actual
//            m <= WA, k <= WB come at run time and columns beyond are masked)
//   TA, TB : the per-thread tile of C, TA x TB
template <int WA, int WB, int TA, int TB>
struct TileShape {
  static_assert(WA % TA == 0 && WB % TB == 0, "tile must divide the width");
  static constexpr int QA = WA / TA;
  static constexpr int QB = WB / TB;
  static constexpr int NT = QA * QB;  // threads that together cover C once
  static_assert((NT & (NT - 1)) == 0, "tile count must be a power of two");
};

// 16-byte vector of T.
template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int N = 2;
  __device__ static void split(const double2& x, double* v) {
    v[0] = x.x;
    v[1] = x.y;
  }
};
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int N = 4;
  __device__ static void split(const float4& x, float* v) {
    v[0] = x.x;
    v[1] = x.y;
    v[2] = x.z;
    v[3] = x.w;
  }
};

namespace detail {

// Undoes the chunk rotation of load_row_seg on a thread's register tile:
// after loading with rotation `rot`, register group q (EPC elements, one
// 16-byte chunk) of a TW-wide segment holds the segment's chunk
// (q + rot) mod TW/EPC.  Rotating the groups right by `rot` (log2 stages of
// compile-time moves under a run-time predicate) puts chunk c back in group
// c, so that lanes with different rotations can then be summed register by
// register.
template <int EPC, int TA, int TB, typename ACC>
__device__ __forceinline__ void unrotate_tile(ACC (&acc)[TA][TB], int rotA, int rotB) {
  if constexpr (TA >= 2 * EPC && TA % EPC == 0 && ((TA / EPC) & (TA / EPC - 1)) == 0) {
    constexpr int N = TA / EPC;
#pragma unroll
    for (int b = 1; b < N; b <<= 1) {
      if (rotA & b) {
        ACC tmp[TA][TB];
#pragma unroll
        for (int c = 0; c < N; ++c)
#pragma unroll
          for (int e = 0; e < EPC; ++e)
#pragma unroll
            for (int j = 0; j < TB; ++j) tmp[EPC * c + e][j] = acc[EPC * ((c - b + N) % N) + e][j];
#pragma unroll
        for (int i = 0; i < TA; ++i)
#pragma unroll
          for (int j = 0; j < TB; ++j) acc[i][j] = tmp[i][j];
      }
    }
  }
  if constexpr (TB >= 2 * EPC && TB % EPC == 0 && ((TB / EPC) & (TB / EPC - 1)) == 0) {
    constexpr int N = TB / EPC;
#pragma unroll
    for (int b = 1; b < N; b <<= 1) {
      if (rotB & b) {
        ACC tmp[TA][TB];
#pragma unroll
        for (int i = 0; i < TA; ++i)
#pragma unroll
          for (int c = 0; c < N; ++c)
#pragma unroll
            for (int e = 0; e < EPC; ++e) tmp[i][EPC * c + e] = acc[i][EPC * ((c - b + N) % N) + e];
#pragma unroll
        for (int i = 0; i < TA; ++i)
#pragma unroll
          for (int j = 0; j < TB; ++j) acc[i][j] = tmp[i][j];
      }
    }
  }
}

template <typename T>
__device__ __forceinline__ void finish_partials(const PlainArgs<T>& p, const double* red, int slots, int t,
                                                int nthreads, unsigned* s_is_last);

// Sums the per-thread tiles of one CTA into `red`, then into this CTA's slot
// of the workspace; the last CTA then writes C.  `red` must hold
// slots * m * k doubles.  Called by all threads of the CTA (nthreads), of
// which the first `cthreads` carry tiles.
template <typename T, int EPC, int TA, int TB, int NT, bool EXACT, int WA, int WB, typename ACC>
__device__ __forceinline__ void finish_tiles(const PlainArgs<T>& p, ACC (&acc_in)[TA][TB], int t, int cthreads,
                                             int nthreads, double* red, unsigned* s_is_last, int rotA = 0,
                                             int rotB = 0) {
  const int m = EXACT ? WA : p.m;
  const int k = EXACT ? WB : p.k;
  const int mk = m * k;
  const int lane = t & 31;
  const int tile = t % NT;
  const int ta = tile % (WA / TA), tb = tile / (WA / TA);
  const bool carrier = t < cthreads;
  if (carrier) unrotate_tile<EPC, TA, TB>(acc_in, rotA, rotB);
  double acc[TA][TB];
#pragma unroll
  for (int i = 0; i < TA; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) acc[i][j] = static_cast<double>(acc_in[i][j]);

  // 1. Warp level: lanes that share a tile differ by multiples of NT.
  if (carrier && NT < 32) {
#pragma unroll
    for (int off = NT; off < 32; off <<= 1)
#pragma unroll
      for (int i = 0; i < TA; ++i)
#pragma unroll
        for (int j = 0; j < TB; ++j) acc[i][j] += __shfl_xor_sync(0xffffffffu, acc[i][j], off);
  }
  // 2. One slot per warp (NT < 32) or per row group (NT >= 32).
  const int slots = NT < 32 ? cthreads / 32 : cthreads / NT;
  if (carrier && (NT >= 32 || lane < NT)) {
    const int slot = NT < 32 ? t / 32 : t / NT;
    double* dst = red + slot * mk;
#pragma unroll
    for (int i = 0; i < TA; ++i) {
      const int row = ta * TA + i;
#pragma unroll
      for (int j = 0; j < TB; ++j) {
        const int col = tb * TB + j;
        if (EXACT || (row < m && col < k)) dst[row * k + col] = acc[i][j];
      }
    }
  }
  __syncthreads();
  finish_partials(p, red, slots, t, nthreads, s_is_last);
}

// Steps 3 and 4 of the reduction: the CTA's `slots` m x k FP64 partial sums
// in `red` (shared memory, complete: the caller synchronised) are summed in
// slot order into this CTA's workspace slot; the last CTA to arrive sums the
// CTA partials in CTA order (plus the rows [rows_main, n) the main loop left)
// and writes C.  Called by all `nthreads` threads of the CTA.
template <typename T>
__device__ __forceinline__ void finish_partials(const PlainArgs<T>& p, const double* red, int slots, int t,
                                                int nthreads, unsigned* s_is_last) {
  const int m = p.m, k = p.k;
  const int mk = m * k;
  // 3. Fixed-order sum over the slots -> this CTA's partial in the workspace.
  double* mine = p.partials + static_cast<int64_t>(blockIdx.x) * mk;
  for (int e = t; e < mk; e += nthreads) {
    double s = red[e];
    for (int q = 1; q < slots; ++q) s += red[q * mk + e];
    mine[e] = s;
  }
  __threadfence();
  __syncthreads();
  if (t == 0) {
    const unsigned prev = atomicAdd(p.counter, 1u);
    *s_is_last = (prev == gridDim.x - 1) ? 1u : 0u;
  }
  __syncthreads();
  if (*s_is_last == 0u) return;

  // 4. Last CTA: partials in CTA order, then the leftover rows, then C.
  //    Symmetric (Gram): the upper triangle is summed and written to both
  //    (i, j) and (j, i), so C is exactly symmetric.
  __threadfence();
  const int G = gridDim.x;
  for (int e = t; e < mk; e += nthreads) {
    const int i = e / k, j = e - (e / k) * k;
    if (p.symmetric && i > j) continue;
    double s = dev::ld_cg(p.partials + e);
    for (int b = 1; b < G; ++b) s += dev::ld_cg(p.partials + static_cast<int64_t>(b) * mk + e);
    for (int64_t r = p.rows_main; r < p.n; ++r)
      s += static_cast<double>(p.A[r * p.lda + i]) * static_cast<double>(p.B[r * p.ldb + j]);
    T* c = p.C + static_cast<int64_t>(i) * p.ldc + j;
    *c = static_cast<T>(p.accumulate ? static_cast<double>(*c) + s : s);
    if (p.symmetric && i != j) {
      T* ct = p.C + static_cast<int64_t>(j) * p.ldc + i;
      *ct = static_cast<T>(p.accumulate ? static_cast<double>(*ct) + s : s);
    }
  }
  if (t == 0) *p.counter = 0u;  // ready for the next launch on this workspace
}

// acc += a (TA) x b (TB) outer product.
template <int TA, int TB, typename ACC>
__device__ __forceinline__ void outer_fma(ACC (&acc)[TA][TB], const ACC (&a)[TA], const ACC (&b)[TB]) {
#pragma unroll
  for (int i = 0; i < TA; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
}

// Loads W consecutive elements from shared memory (16-byte vector loads where
// the layout allows) or, in capacity mode, up to `valid` of them (rest = 0).
// With vector loads, 16-byte chunk c of the segment goes to register group
// (c - rot) mod (W / EPC): threads whose rows share shared-memory banks then
// read different banks in the same instruction (the rows of a warp are a
// whole number of 128-byte bank rows apart for row pitches of 64, 128, 256
// and 512 bytes).  The accumulators follow the registers, so the rotation is
// undone once, on the finished tile (unrotate_tile).
template <typename T, int W, bool VEC>
__device__ __forceinline__ void load_row_seg(T (&v)[W], const T* src, int valid, int rot = 0) {
  if constexpr (VEC) {
    using V = Vec16<T>;
    constexpr int N = W / V::N;
    static_assert(W % V::N == 0 && (N & (N - 1)) == 0,
                  "vector segments hold a power-of-two number of 16-byte chunks");
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const typename V::type x = reinterpret_cast<const typename V::type*>(src)[(i + rot) & (N - 1)];
      V::split(x, v + V::N * i);
    }
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = (i < valid) ? src[i] : T(0);
  }
}

}  // namespace detail

// --------------------------------------------------------------------------
// Bulk (TMA) pipelined kernel.
// --------------------------------------------------------------------------
// GRAM: B is A (C = A^T A): only A's rows are streamed and the B tile reads
// the same stage.
template <typename T, int WA, int WB, int TA, int TB, int CW, int STAGES, int RS, int UNROLL, bool EXACT,
          bool GRAM = false>
struct BulkKernel {
  static_assert(!GRAM || (WA == WB && EXACT), "Gram variants are exact and square");
  using S = TileShape<WA, WB, TA, TB>;
  static constexpr int EPC = 16 / int(sizeof(T));  // elements per 16-byte chunk
  static constexpr int CT = CW * 32;               // consumer threads
  static constexpr int THREADS = CT + 32;          // + one producer warp
  static_assert(CT % S::NT == 0, "consumer threads must cover whole tiles");
  static constexpr int RG = CT / S::NT;  // row groups
  static_assert(RS % EPC == 0, "chunk rows must keep every bulk copy a multiple of 16 bytes");
  static constexpr int STAGE_A = RS * WA;  // elements (capacity)
  static constexpr int STAGE_B = GRAM ? 0 : RS * WB;
  static constexpr int SLOTS = S::NT < 32 ? CW : RG;
  static constexpr size_t RING_BYTES = size_t(STAGES) * (STAGE_A + STAGE_B) * sizeof(T);
  static constexpr size_t RED_BYTES = size_t(SLOTS) * WA * WB * sizeof(double);
  static constexpr size_t DATA_BYTES = RING_BYTES > RED_BYTES ? RING_BYTES : RED_BYTES;
  static constexpr size_t BAR_OFFSET = (DATA_BYTES + 127) / 128 * 128;
  static constexpr size_t SMEM_BYTES = BAR_OFFSET + 2 * STAGES * sizeof(uint64_t) + 16;
  static constexpr bool VEC_A = EXACT && TA % EPC == 0 && WA % EPC == 0;
  static constexpr bool VEC_B = EXACT && TB % EPC == 0 && WB % EPC == 0;
  // Chunk rotation (load_row_seg): a thread's rows r = rg + i*RG must all
  // map to the same rotation, i.e. RG row pitches span whole multiples of
  // 8 * (chunks per segment) 16-byte units.
  static constexpr int NCH_A = TA / EPC > 0 ? TA / EPC : 1;
  static constexpr int NCH_B = TB / EPC > 0 ? TB / EPC : 1;
  static constexpr bool ROT_A = VEC_A && NCH_A > 1 && (RG * (WA / EPC)) % (8 * NCH_A) == 0;
  static constexpr bool ROT_B = VEC_B && NCH_B > 1 && (RG * (WB / EPC)) % (8 * NCH_B) == 0;
  // Rotation of a thread whose first row in a stage is rg and whose segment
  // starts at column col: spreads the rows and column segments of one warp
  // over the eight 16-byte bank groups.
  __device__ static int rotation(int rg, int col, int width, int nch) {
    return ((rg * (width / EPC) + col / EPC) / 8) & (nch - 1);
  }
};

template <typename T, int WA, int WB, int TA, int TB, int CW, int STAGES, int RS, int UNROLL, bool EXACT,
          bool GRAM = false>
__global__ void __launch_bounds__(BulkKernel<T, WA, WB, TA, TB, CW, STAGES, RS, UNROLL, EXACT, GRAM>::THREADS, 1)
    tsm_tn_bulk_kernel(const PlainArgs<T> p) {
  using K = BulkKernel<T, WA, WB, TA, TB, CW, STAGES, RS, UNROLL, EXACT, GRAM>;
  using S = typename K::S;
  extern __shared__ __align__(128) unsigned char smem[];
  T* ringA = reinterpret_cast<T*>(smem);
  T* ringB = ringA + STAGES * K::STAGE_A;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + K::BAR_OFFSET);
  uint64_t* empty = full + STAGES;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + STAGES);
  unsigned* s_is_last = reinterpret_cast<unsigned*>(empty + STAGES) + 1;

  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  const int m = EXACT ? WA : p.m;
  const int k = EXACT ? WB : p.k;

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
  T acc[TA][TB];
#pragma unroll
  for (int i = 0; i < TA; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) acc[i][j] = T(0);

  if (warp == CW) {
    // ---------------- producer warp: lane 0 issues, the warp stays converged.
    int64_t issued = 0;
    const uint64_t policy = dev::policy_evict_first();
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++issued) {
      const int s = static_cast<int>(issued % STAGES);
      const int64_t round = issued / STAGES;
      bool ok = true;
      if (lane == 0) {
        if (round > 0) ok = dev::mbar_wait(&empty[s], static_cast<uint32_t>((round - 1) & 1), abort);
        if (ok) {
          const int64_t r0 = c * RS;
          const int64_t rows = (p.rows_main - r0) < RS ? (p.rows_main - r0) : RS;
          const uint32_t ba = static_cast<uint32_t>(rows * m * sizeof(T));
          const uint32_t bb = GRAM ? 0u : static_cast<uint32_t>(rows * k * sizeof(T));
          dev::mbar_arrive_expect_tx(&full[s], ba + bb);
          dev::bulk_g2s_evict_first(ringA + s * K::STAGE_A, p.A + r0 * m, ba, &full[s], policy);
          if (!GRAM) dev::bulk_g2s_evict_first(ringB + s * K::STAGE_B, p.B + r0 * k, bb, &full[s], policy);
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else {
    // ---------------- consumer warps.
    const int tile = t % S::NT;
    const int ta = tile % S::QA, tb = tile / S::QA;
    const int rg = t / S::NT;
    const int colA = ta * TA, colB = tb * TB;
    const int validA = m - colA, validB = k - colB;
    const int rotA = K::ROT_A ? K::rotation(rg, colA, WA, K::NCH_A) : 0;
    const int rotB = K::ROT_B ? K::rotation(rg, colB, WB, K::NCH_B) : 0;
    int64_t it = 0;
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++it) {
      const int s = static_cast<int>(it % STAGES);
      if (!dev::mbar_wait(&full[s], static_cast<uint32_t>((it / STAGES) & 1), abort)) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      const int64_t r0 = c * RS;
      const int rows = static_cast<int>((p.rows_main - r0) < RS ? (p.rows_main - r0) : RS);
      const T* sa = ringA + s * K::STAGE_A + colA;
      const T* sb = (GRAM ? ringA + s * K::STAGE_A : ringB + s * K::STAGE_B) + colB;
      if (rows == RS) {
        static_assert((RS / K::RG) % UNROLL == 0 || RS < K::RG, "unroll must divide the rows per thread");
#pragma unroll UNROLL
        for (int r = rg; r < RS; r += K::RG) {
          T a[TA], b[TB];
          detail::load_row_seg<T, TA, K::VEC_A>(a, sa + r * m, validA, rotA);
          detail::load_row_seg<T, TB, K::VEC_B>(b, sb + r * k, validB, rotB);
          detail::outer_fma<TA, TB>(acc, a, b);
        }
      } else {
        for (int r = rg; r < rows; r += K::RG) {
          T a[TA], b[TB];
          detail::load_row_seg<T, TA, K::VEC_A>(a, sa + r * m, validA, rotA);
          detail::load_row_seg<T, TB, K::VEC_B>(b, sb + r * k, validB, rotB);
          detail::outer_fma<TA, TB>(acc, a, b);
        }
      }
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&empty[s]);
    }
  }

  __syncthreads();
  if (*abort && warp == CW && lane == 0) {
    // Let every bulk copy this CTA issued land before the ring is reused or
    // the CTA exits.  Bounded as well; a second timeout is only recorded.
    int64_t issued = 0;
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G) ++issued;
    volatile int no_abort = 0;
    for (int64_t q = issued > STAGES ? issued - STAGES : 0; q < issued; ++q)
      if (!dev::mbar_wait(&full[q % STAGES], static_cast<uint32_t>((q / STAGES) & 1), &no_abort)) break;
  }
  __syncthreads();

  int rotA = 0, rotB = 0;
  if (warp < CW) {
    const int tile = t % S::NT;
    const int rg = t / S::NT;
    rotA = K::ROT_A ? K::rotation(rg, (tile % S::QA) * TA, WA, K::NCH_A) : 0;
    rotB = K::ROT_B ? K::rotation(rg, (tile / S::QA) * TB, WB, K::NCH_B) : 0;
  }
  detail::finish_tiles<T, K::EPC, TA, TB, S::NT, EXACT, WA, WB>(p, acc, t, K::CT, K::THREADS,
                                                                  reinterpret_cast<double*>(smem), s_is_last,
                                                                  rotA, rotB);
}

// --------------------------------------------------------------------------
// Direct-load kernel (strided or unaligned operands).
// --------------------------------------------------------------------------
template <typename T, int WA, int WB, int TA, int TB, int THREADS, bool EXACT>
struct DirectKernel {
  using S = TileShape<WA, WB, TA, TB>;
  static_assert(THREADS % S::NT == 0 && THREADS % 32 == 0, "threads must cover whole tiles");
  static constexpr int RG = THREADS / S::NT;
  static constexpr int SLOTS = S::NT < 32 ? THREADS / 32 : RG;
  static constexpr size_t SMEM_BYTES = size_t(SLOTS) * WA * WB * sizeof(double) + 16;
};

template <typename T, int WA, int WB, int TA, int TB, int THREADS, bool EXACT>
__global__ void __launch_bounds__(THREADS) tsm_tn_direct_kernel(const PlainArgs<T> p) {
  using K = DirectKernel<T, WA, WB, TA, TB, THREADS, EXACT>;
  using S = typename K::S;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned* s_is_last = reinterpret_cast<unsigned*>(smem + K::SMEM_BYTES - 16);

  const int t = threadIdx.x;
  const int m = EXACT ? WA : p.m;
  const int k = EXACT ? WB : p.k;
  const int tile = t % S::NT;
  const int ta = tile % S::QA, tb = tile / S::QA;
  const int colA = ta * TA, colB = tb * TB;
  const int validA = m - colA, validB = k - colB;

  T acc[TA][TB];
#pragma unroll
  for (int i = 0; i < TA; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) acc[i][j] = T(0);

  const int64_t rstep = static_cast<int64_t>(gridDim.x) * K::RG;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * K::RG + t / S::NT; r < p.rows_main; r += rstep) {
    const T* ar = p.A + r * p.lda + colA;
    const T* br = p.B + r * p.ldb + colB;
    T a[TA], b[TB];
#pragma unroll
    for (int i = 0; i < TA; ++i) a[i] = (EXACT || i < validA) ? __ldg(ar + i) : T(0);
#pragma unroll
    for (int j = 0; j < TB; ++j) b[j] = (EXACT || j < validB) ? __ldg(br + j) : T(0);
    detail::outer_fma<TA, TB>(acc, a, b);
  }
  detail::finish_tiles<T, 16 / int(sizeof(T)), TA, TB, S::NT, EXACT, WA, WB>(
      p, acc, t, THREADS, THREADS, reinterpret_cast<double*>(smem), s_is_last);
}

}  // namespace tsm
