// tsm_strided.cuh -- C (m x k) = A^T B for operands in other element
// layouts than the row-major one of tsm_plain.cuh / tsm_dmma.cuh.  Element
// (r, i) of A (row r < n, column i < m) is A[r * a_row + i * a_col].
//
// Column-major operands (a_row = 1): A is stored as the row-major m x n
// matrix A^T with pitch a_col >= n, each column of A one contiguous run of
// n values.  The contraction index r is then the contiguous one, so the
// kernels stream chunks of RS consecutive r for all m (k) columns at once.
//
// Both pipelined kernels load 2-D TMA boxes of the map {n, m} (x = r, y =
// column), unswizzled; columns beyond m (k) and r beyond n are zero-filled by
// the TMA unit, so every chunk is processed whole.
//
//   * tsm_tn_cm_simt_kernel<WA, WB, RS, STAGES> -- width capacities with
//     WA * WB <= 64: boxes of min(RS, 256) r x WA columns; each
//     consumer thread takes whole r values (consecutive threads consecutive
//     r, so the shared loads are conflict-free) and keeps all WA x WB sums.
//   * tsm_tn_cm_dmma_kernel<WA, WB, MT, NT, CW, STAGES, RS> -- capacities in
//     {8, 16, 32, 48, 64}: FP64 tensor cores (mma.m8n8k4.f64).  One
//     unswizzled box per operand and chunk, RS + 2 values x WA columns: the
//     shared rows land RS * 8 + 16 bytes apart, so consecutive rows start one
//     16-byte bank group apart (the 2 extra values, the next chunk's first,
//     are ignored).  Measured on 2^26 x 32 x 32: runs of 128 bytes per
//     column (boxes with the 128-byte swizzle) streamed at 4.6 TB/s, one 1-D
//     bulk copy per column and chunk at ~35 ns a copy; whole-chunk boxes
//     have neither limit.  A DMMA's A operand is 8 columns x 4 values of r:
//     lane 4 g + t holds A[r(t)][i0 + g], B[r(t)][j0 + g].  One 16-byte load
//     of chunk 2 t + s of a 16-value group of row i0 + g gives a lane the
//     values r = 4 t + 2 s and 4 t + 2 s + 1 of the group -- two k-steps,
//     each a permutation of r (the same in both operands); the 8 lanes of a
//     16-byte load phase (g, g + 1; t = 0..3) then hit bank groups
//     g + 2 t + s mod 8, all different.  A warp region is MT x NT tiles of
//     C; each (group, s) unit costs MT + NT shared loads for 2 MT NT DMMAs.
//   * tsm_tn_strided_kernel<WA, WB, TA, TB, THREADS> -- any positive
//     strides (mixed layouts, odd pitches, unaligned bases): TA x TB register
//     tiles fed by read-only global loads, one row per thread group.
//
// All three end in the deterministic two-level reduction of tsm_plain.cuh
// (finish_partials): per-CTA partials in the workspace, the last CTA sums
// them in CTA order.  Every wait is bounded (dev::mbar_wait); a timeout sets
// the error word, drains the CTA's copies (bounded) and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"
#include "tsm_plain.cuh"

namespace tsm {

struct StridedArgs {
  PlainArgs<double> p;  // A, B, C, n, m, k, ldc, accumulate, workspace; rows_main = n
  int64_t a_row, a_col, b_row, b_col;
};

struct CmArgs {
  PlainArgs<double> p;  // num_chunks = ceil(n / RS); rows_main = n
  CUtensorMap ta;       // A^T: {n, m}, pitch a_col
  CUtensorMap tb;       // B^T: {n, k}, pitch b_col
};

// ------------------------------------------------------------------ SIMT
template <int WA, int WB, int RS, int STAGES>
struct CmSimt {
  static_assert(WA * WB <= 64, "register tile of all of C: at most 64 sums per thread");
  static_assert(RS % 32 == 0 && (RS <= 256 || RS % 256 == 0), "chunk: whole warps of r, boxes of <= 256 r");
  static constexpr int BOX_R = RS < 256 ? RS : 256;  // r per box
  static constexpr int NBOX = RS / BOX_R;            // boxes per operand and chunk
  static constexpr int CW = 8;                       // consumer warps
  static constexpr int THREADS = CW * 32 + 32;       // + the producer warp (last)
  static constexpr int STAGE_BYTES = RS * (WA + WB) * 8;
  static_assert((BOX_R * 8) % 128 == 0, "boxes start on 128-byte boundaries");
  static constexpr size_t RING_BYTES = size_t(STAGES) * STAGE_BYTES;
  static constexpr size_t RED_BYTES = size_t(CW) * WA * WB * sizeof(double);
  static constexpr size_t DATA_BYTES = RING_BYTES > RED_BYTES ? RING_BYTES : RED_BYTES;
  static constexpr size_t BAR_OFFSET = (DATA_BYTES + 127) / 128 * 128;
  static constexpr size_t SMEM_BYTES = 128 + BAR_OFFSET + 2 * STAGES * sizeof(uint64_t) + 16;
};

namespace detail {

// Producer side of both column-major kernels: lane 0 of the calling warp
// fills stage s with chunk c (NBA boxes of A^T then NBB of B^T, box_r r
// apart; each box box_bytes_a / box_bytes_b).  Returns false on a timeout.
__device__ __forceinline__ bool cm_produce(const CmArgs& args, unsigned char* stage, uint64_t* full, uint64_t* empty,
                                           int64_t issued, int stages, int stage_bytes, int nba, int nbb, int box_r,
                                           int box_bytes_a, int box_bytes_b, int64_t r0, uint64_t policy,
                                           volatile int* abort) {
  const int s = static_cast<int>(issued % stages);
  const int64_t round = issued / stages;
  if (round > 0 && !dev::mbar_wait(&empty[s], static_cast<uint32_t>((round - 1) & 1), abort)) return false;
  dev::mbar_arrive_expect_tx(&full[s], static_cast<uint32_t>(stage_bytes));
  for (int b = 0; b < nba; ++b)
    dev::tma_load_2d(stage + b * box_bytes_a, &args.ta, static_cast<int>(r0 + b * box_r), 0, &full[s], policy);
  unsigned char* stb = stage + nba * box_bytes_a;
  for (int b = 0; b < nbb; ++b)
    dev::tma_load_2d(stb + b * box_bytes_b, &args.tb, static_cast<int>(r0 + b * box_r), 0, &full[s], policy);
  return true;
}

// After an abort: lets every tensor load this CTA issued land before the
// shared memory is reused (bounded; a second timeout is only recorded).
__device__ __forceinline__ void cm_drain(uint64_t* full, int64_t num_chunks, int stages) {
  int64_t issued = 0;
  for (int64_t c = blockIdx.x; c < num_chunks; c += gridDim.x) ++issued;
  volatile int no_abort = 0;
  for (int64_t q = issued > stages ? issued - stages : 0; q < issued; ++q)
    if (!dev::mbar_wait(&full[q % stages], static_cast<uint32_t>((q / stages) & 1), &no_abort)) break;
}

}  // namespace detail

template <int WA, int WB, int RS, int STAGES>
__global__ void __launch_bounds__(CmSimt<WA, WB, RS, STAGES>::THREADS, 1)
    tsm_tn_cm_simt_kernel(const __grid_constant__ CmArgs args) {
  using K = CmSimt<WA, WB, RS, STAGES>;
  const PlainArgs<double>& p = args.p;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (dev::smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + K::BAR_OFFSET);
  uint64_t* empty = full + STAGES;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + STAGES);
  unsigned* s_is_last = reinterpret_cast<unsigned*>(empty + STAGES) + 1;

  const int t = threadIdx.x;
  const int warp = t >> 5, lane = t & 31;
  if (t == 0) {
    for (int s = 0; s < STAGES; ++s) {
      dev::mbar_init(&full[s], 1);
      dev::mbar_init(&empty[s], K::CW);
    }
    *abort = 0;
    dev::fence_mbar_init();
  }
  if (warp == K::CW && lane == 0 && blockIdx.x < p.num_chunks) {
    dev::prefetch_tensormap(&args.ta);
    dev::prefetch_tensormap(&args.tb);
  }
  __syncthreads();

  const int64_t G = gridDim.x;
  double acc[WA][WB];
#pragma unroll
  for (int i = 0; i < WA; ++i)
#pragma unroll
    for (int j = 0; j < WB; ++j) acc[i][j] = 0.0;

  if (warp == K::CW) {
    // ---------------- producer warp: lane 0 issues the tensor loads.
    int64_t issued = 0;
    const uint64_t policy = dev::policy_evict_first();
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++issued) {
      bool ok = true;
      if (lane == 0) {
        ok = detail::cm_produce(args, smem + (issued % STAGES) * K::STAGE_BYTES, full, empty, issued, STAGES,
                                K::STAGE_BYTES, K::NBOX, K::NBOX, K::BOX_R, K::BOX_R * WA * 8, K::BOX_R * WB * 8,
                                c * RS, policy, abort);
        if (!ok) {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else {
    // ---------------- consumers: thread t takes r = t, t + 256, ... of each chunk.
    int64_t it = 0;
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++it) {
      const int s = static_cast<int>(it % STAGES);
      if (!dev::mbar_wait(&full[s], static_cast<uint32_t>((it / STAGES) & 1), abort)) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      const double* sa = reinterpret_cast<const double*>(smem + s * K::STAGE_BYTES);
      const double* sb = sa + RS * WA;
      for (int r = t; r < RS; r += K::CW * 32) {
        const int box = r / K::BOX_R, rr = r % K::BOX_R;
        const double* pa = sa + box * (K::BOX_R * WA) + rr;
        const double* pb = sb + box * (K::BOX_R * WB) + rr;
        // The narrower operand's values stay in registers, the wider one's
        // are streamed through (64 sums + a few values: no spills at 168
        // registers a thread).
        if constexpr (WA >= WB) {
          double b[WB];
#pragma unroll
          for (int j = 0; j < WB; ++j) b[j] = pb[j * K::BOX_R];
#pragma unroll
          for (int i = 0; i < WA; ++i) {
            const double a = pa[i * K::BOX_R];
#pragma unroll
            for (int j = 0; j < WB; ++j) acc[i][j] = fma(a, b[j], acc[i][j]);
          }
        } else {
          double a[WA];
#pragma unroll
          for (int i = 0; i < WA; ++i) a[i] = pa[i * K::BOX_R];
#pragma unroll
          for (int j = 0; j < WB; ++j) {
            const double b = pb[j * K::BOX_R];
#pragma unroll
            for (int i = 0; i < WA; ++i) acc[i][j] = fma(a[i], b, acc[i][j]);
          }
        }
      }
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&empty[s]);
    }
  }

  __syncthreads();
  if (*abort && warp == K::CW && lane == 0) detail::cm_drain(full, p.num_chunks, STAGES);
  __syncthreads();
  // Each consumer thread holds all of C: a warp shuffle sum, one slot per
  // consumer warp (the producer warp carries nothing), then the CTA sum.
  double* red = reinterpret_cast<double*>(smem);
  const int m = p.m, k = p.k;
  if (warp < K::CW) {
#pragma unroll
    for (int i = 0; i < WA; ++i)
#pragma unroll
      for (int j = 0; j < WB; ++j) {
        double v = acc[i][j];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0 && i < m && j < k) red[warp * m * k + i * k + j] = v;
      }
  }
  __syncthreads();
  detail::finish_partials(p, red, K::CW, t, K::THREADS, s_is_last);
}

// ------------------------------------------------------------------ DMMA
template <int WA, int WB, int MT, int NT, int CW, int STAGES, int RS>
struct CmDmma {
  static_assert(WA % 8 == 0 && WB % 8 == 0 && WA <= 64 && WB <= 64, "capacities: multiples of 8 up to 64");
  static_assert(RS % 16 == 0 && RS + 2 <= 256, "chunk: whole 16-value groups, box of RS + 2 <= 256 values");
  static constexpr int MTA = WA / 8, NTB = WB / 8;  // 8 x 8 tiles of C along m and k
  static_assert(MTA % MT == 0 && NTB % NT == 0 && MT * NT <= 16, "region: tile counts dividing the widths");
  static constexpr int RA = MTA / MT, RB = NTB / NT;
  static constexpr int R = RA * RB;  // regions
  static_assert(CW % R == 0, "consumer warps must cover whole regions");
  static constexpr int S = CW / R;      // unit slots
  static constexpr int UNITS = RS / 8;  // (16-value group, half) units per chunk
  // A box row is RS + 2 values: the 2 extra ones (the next chunk's first,
  // ignored) make consecutive shared rows start one 16-byte bank group apart.
  static constexpr int BOX_R = RS + 2;
  static constexpr int PITCH = BOX_R * 8;
  static_assert((PITCH / 16) % 8 == 1, "row pitch: one bank group of skew per row");
  static constexpr int TILE_A = WA * PITCH, TILE_B = WB * PITCH;  // multiples of 128
  static constexpr int STAGE_BYTES = TILE_A + TILE_B;
  static constexpr int THREADS = CW * 32 + 32;
  static constexpr size_t RING_BYTES = size_t(STAGES) * STAGE_BYTES;
  static constexpr size_t RED_BYTES = size_t(S) * WA * WB * sizeof(double);
  static constexpr size_t DATA_BYTES = RING_BYTES > RED_BYTES ? RING_BYTES : RED_BYTES;
  static constexpr size_t BAR_OFFSET = (DATA_BYTES + 127) / 128 * 128;
  static constexpr size_t SMEM_BYTES = 128 + BAR_OFFSET + 2 * STAGES * sizeof(uint64_t) + 16;
};

template <int WA, int WB, int MT, int NT, int CW, int STAGES, int RS>
__global__ void __launch_bounds__(CmDmma<WA, WB, MT, NT, CW, STAGES, RS>::THREADS, 1)
    tsm_tn_cm_dmma_kernel(const __grid_constant__ CmArgs args) {
  using K = CmDmma<WA, WB, MT, NT, CW, STAGES, RS>;
  const PlainArgs<double>& p = args.p;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (dev::smem_u32(smem_raw) & 127u)) & 127u);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + K::BAR_OFFSET);
  uint64_t* empty = full + STAGES;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + STAGES);
  unsigned* s_is_last = reinterpret_cast<unsigned*>(empty + STAGES) + 1;

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
  if (warp == CW && lane == 0 && blockIdx.x < p.num_chunks) {
    dev::prefetch_tensormap(&args.ta);
    dev::prefetch_tensormap(&args.tb);
  }
  __syncthreads();

  const int64_t G = gridDim.x;
  const int region = warp % K::R, slot = warp / K::R;
  const int ra = region % K::RA, rb = region / K::RA;
  double acc[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  if (warp == CW) {
    int64_t issued = 0;
    const uint64_t policy = dev::policy_evict_first();
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++issued) {
      bool ok = true;
      if (lane == 0) {
        ok = detail::cm_produce(args, smem + (issued % STAGES) * K::STAGE_BYTES, full, empty, issued, STAGES,
                                K::STAGE_BYTES, 1, 1, K::BOX_R, K::TILE_A, K::TILE_B, c * RS, policy, abort);
        if (!ok) {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else {
    const int g = lane >> 2, tq = lane & 3;
    const int a_row0 = 8 * ra * MT + g, b_row0 = 8 * rb * NT + g;
    int64_t it = 0;
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++it) {
      const int s = static_cast<int>(it % STAGES);
      if (!dev::mbar_wait(&full[s], static_cast<uint32_t>((it / STAGES) & 1), abort)) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      const unsigned char* sa = smem + s * K::STAGE_BYTES;
      const unsigned char* sb = sa + K::TILE_A;
#pragma unroll 2
      for (int u = slot; u < K::UNITS; u += K::S) {
        // Lane (g, tq) reads values 2 (2 tq + half) and + 1 of 16-value
        // group u / 2: 16-byte chunk 8 group + 2 tq + half of its row.
        const int off = 16 * (8 * (u >> 1) + 2 * tq + (u & 1));
        double2 a[MT], b[NT];
#pragma unroll
        for (int i = 0; i < MT; ++i) a[i] = *reinterpret_cast<const double2*>(sa + (a_row0 + 8 * i) * K::PITCH + off);
#pragma unroll
        for (int j = 0; j < NT; ++j) b[j] = *reinterpret_cast<const double2*>(sb + (b_row0 + 8 * j) * K::PITCH + off);
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) {
            dev::dmma_m8n8k4(acc[i][j][0], acc[i][j][1], a[i].x, b[j].x);
            dev::dmma_m8n8k4(acc[i][j][0], acc[i][j][1], a[i].y, b[j].y);
          }
      }
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&empty[s]);
    }
  }

  __syncthreads();
  if (*abort && warp == CW && lane == 0) detail::cm_drain(full, p.num_chunks, STAGES);
  __syncthreads();

  // Tile (i, j) of the warp: D[g][2 tq + e] is C[8 (ra MT + i) + g][8 (rb NT + j) + 2 tq + e].
  const int m = p.m, k = p.k, mk = m * k;
  double* red = reinterpret_cast<double*>(smem);
  if (warp < CW) {
    const int g = lane >> 2, tq = lane & 3;
    double* sheet = red + slot * mk;
#pragma unroll
    for (int i = 0; i < MT; ++i) {
      const int row = 8 * (ra * MT + i) + g;
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = 8 * (rb * NT + j) + 2 * tq + e;
          if (row < m && col < k) sheet[row * k + col] = acc[i][j][e];
        }
    }
  }
  __syncthreads();
  detail::finish_partials(p, red, K::S, t, K::THREADS, s_is_last);
}

// ------------------------------------------------------- any strides
template <int WA, int WB, int TA, int TB, int THREADS>
struct StridedKernel {
  using S = TileShape<WA, WB, TA, TB>;
  static_assert(THREADS % S::NT == 0 && THREADS % 32 == 0, "whole row groups, whole warps");
  static constexpr int RG = THREADS / S::NT;  // rows per CTA step
  static constexpr int SLOTS = S::NT < 32 ? THREADS / 32 : RG;
  static constexpr size_t SMEM_BYTES = size_t(SLOTS) * WA * WB * sizeof(double) + 16;
};

template <int WA, int WB, int TA, int TB, int THREADS>
__global__ void __launch_bounds__(THREADS) tsm_tn_strided_kernel(const StridedArgs args) {
  using K = StridedKernel<WA, WB, TA, TB, THREADS>;
  using S = typename K::S;
  const PlainArgs<double>& p = args.p;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned* s_is_last = reinterpret_cast<unsigned*>(smem + K::SMEM_BYTES - 16);

  const int t = threadIdx.x;
  const int tile = t % S::NT;
  const int ta = tile % S::QA, tb = tile / S::QA;
  const int colA = ta * TA, colB = tb * TB;
  const int validA = p.m - colA, validB = p.k - colB;

  double acc[TA][TB];
#pragma unroll
  for (int i = 0; i < TA; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) acc[i][j] = 0.0;

  const int64_t rstep = static_cast<int64_t>(gridDim.x) * K::RG;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * K::RG + t / S::NT; r < p.n; r += rstep) {
    const double* ar = p.A + r * args.a_row + colA * args.a_col;
    const double* br = p.B + r * args.b_row + colB * args.b_col;
    double a[TA], b[TB];
#pragma unroll
    for (int i = 0; i < TA; ++i) a[i] = i < validA ? __ldg(ar + i * args.a_col) : 0.0;
#pragma unroll
    for (int j = 0; j < TB; ++j) b[j] = j < validB ? __ldg(br + j * args.b_col) : 0.0;
    detail::outer_fma<TA, TB>(acc, a, b);
  }
  detail::finish_tiles<double, 2, TA, TB, S::NT, false, WA, WB>(p, acc, t, THREADS, THREADS,
                                                                 reinterpret_cast<double*>(smem), s_is_last);
}

}  // namespace tsm
