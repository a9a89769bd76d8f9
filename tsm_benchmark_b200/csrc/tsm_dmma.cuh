// tsm_dmma.cuh -- FP64 TSMTTSM, C (m x k) = A^T B, on the FP64 tensor cores
// (mma.sync m8n8k4 .f64, "DMMA"; tcgen05 has no FP64 kind).  For the wide
// shapes (m, k in {16, 32, 48, 64}) where the SIMT register-tile kernels of
// tsm_plain.cuh are bound by FMA issue rather than by HBM: one DMMA is 256
// FMAs in one warp instruction.
//
// Contraction over rows.  A DMMA multiplies an 8 x 4 block of A^T (8
// columns of A, 4 rows) by a 4 x 8 block of B (4 rows, 8 columns of B) into
// an 8 x 8 tile of C.  Fragments (PTX ISA, mma.m8n8k4 .f64; lane = 4 g + t):
// lane holds A^T[g][t] = A[row(t)][col(g)], B[row(t)][col'(g)] and
// D[g][2t], D[g][2t + 1].  Both the rows of a k-step and the columns of a
// tile may be permuted freely (the same way in both operands / tracked in the
// output), which this kernel uses twice:
//   * a tile's 8 columns are every other column of a 16-column block
//     (parity 0 or 1), so ONE 16-byte shared load gives a lane its values
//     for two tiles (the even and the odd one);
//   * the 4 rows of a k-step are rows s, s+2, s+4, s+6 of an 8-row group
//     (s = 0, 1): with the 128-byte swizzle below, the 8 lanes of each
//     16-byte load phase then hit 8 different bank groups.
//
// Data movement.  A producer warp streams RS-row chunks of A and B with 2-D
// tiled TMA loads (tensor maps built on the host, 16 x RS boxes of 128-byte
// rows, CU_TENSOR_MAP_SWIZZLE_128B: 16-byte chunk c of box row r is stored
// at chunk c ^ (r mod 8)) into a STAGES-deep shared-memory ring with
// mbarrier completion, as in tsm_plain.cuh.  Rows beyond n are zero-filled by
// the TMA unit, so every chunk is processed in full and no rows are left for
// an epilogue.
//
// Warps.  C's 8 x 8 tiles are split into R regions of MT x NT tiles (<= 16
// tiles, 32 FP64 accumulators per lane; a k-step costs MT/2 + NT/2 shared
// loads for MT x NT DMMAs, so the generator picks the region that maximises
// that ratio); the CW consumer warps are R regions x S row slots.  A warp walks the k-steps of its slot in every chunk.  At the
// end each warp writes its tiles into its slot's m x k sheet in shared
// memory, and the deterministic two-level reduction of tsm_plain.cuh
// (finish_partials) sums slots in order, then CTAs in order.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tsm_device.cuh"
#include "tsm_plain.cuh"

namespace tsm {

struct DmmaArgs {
  PlainArgs<double> p;
  CUtensorMap ta;  // A: {m columns, n rows}, box {16, RS}, 128-byte swizzle
  CUtensorMap tb;  // B: {k columns, n rows}, box {16, RS}, 128-byte swizzle
};

// A chunk of RS rows is loaded as dmma_boxes(RS) tensor boxes of
// dmma_box_rows(RS) rows per 16-column block (a box spans at most 256 rows;
// each box is a whole number of 8-row swizzle groups, 1024-byte aligned, so
// the block's rows lie in shared memory exactly as one taller box would put
// them).  The host encodes the tensor maps with the same box height.
__host__ __device__ constexpr int dmma_boxes(int rs) { return (rs + 255) / 256; }
__host__ __device__ constexpr int dmma_box_rows(int rs) { return rs / dmma_boxes(rs); }
__host__ __device__ constexpr bool dmma_rows_ok(int rs) {
  return rs > 0 && rs % 8 == 0 && rs <= 1024 && rs % dmma_boxes(rs) == 0 && dmma_box_rows(rs) % 8 == 0;
}

template <int WA, int WB, int MT, int NT, int CW, int STAGES, int RS>
struct DmmaTn {
  static_assert(WA % 16 == 0 && WB % 16 == 0 && WA <= 64 && WB <= 64, "widths: multiples of 16 up to 64");
  static_assert(dmma_rows_ok(RS), "chunk rows: equal boxes of whole 8-row swizzle groups, <= 256 rows each");
  static constexpr int NBOX = dmma_boxes(RS), BOX_ROWS = dmma_box_rows(RS);
  static constexpr int MBA = WA / 16, MBB = WB / 16;  // 16-column blocks per chunk
  static constexpr int MTA = WA / 8, NTB = WB / 8;    // 8 x 8 tiles of C along m and k
  // MT x NT tiles per warp (region): even (whole 16-column blocks), dividing
  // the widths, at most 16 tiles (32 accumulators per lane).
  static_assert(MT % 2 == 0 && NT % 2 == 0 && MTA % MT == 0 && NTB % NT == 0 && MT * NT <= 16,
                "region: even tile counts dividing the widths, <= 16 tiles");
  static constexpr int RA = MTA / MT, RB = NTB / NT;
  static constexpr int R = RA * RB;  // regions
  static_assert(CW % R == 0, "consumer warps must cover whole regions");
  static constexpr int S = CW / R;  // row slots
  static constexpr int KSTEPS = RS / 4;
  static constexpr int BOX_BYTES = RS * 128;  // one 16-column block of the chunk (NBOX tensor boxes)
  static constexpr int STAGE_BYTES = (MBA + MBB) * BOX_BYTES;  // a multiple of 1024
  static constexpr int THREADS = CW * 32 + 32;
  static constexpr size_t RING_BYTES = size_t(STAGES) * STAGE_BYTES;
  static constexpr size_t RED_BYTES = size_t(S) * WA * WB * sizeof(double);
  static constexpr size_t DATA_BYTES = RING_BYTES > RED_BYTES ? RING_BYTES : RED_BYTES;
  static constexpr size_t BAR_OFFSET = (DATA_BYTES + 127) / 128 * 128;
  // + 1024: the ring is aligned to 1024 bytes (the swizzle pattern's period).
  static constexpr size_t SMEM_BYTES = 1024 + BAR_OFFSET + 2 * STAGES * sizeof(uint64_t) + 16;
};

template <int WA, int WB, int MT, int NT, int CW, int STAGES, int RS>
__global__ void __launch_bounds__(DmmaTn<WA, WB, MT, NT, CW, STAGES, RS>::THREADS, 1)
    tsm_tn_dmma_kernel(const __grid_constant__ DmmaArgs args) {
  using K = DmmaTn<WA, WB, MT, NT, CW, STAGES, RS>;
  const PlainArgs<double>& p = args.p;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024u - (dev::smem_u32(smem_raw) & 1023u)) & 1023u);
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
    // ---------------- producer warp: lane 0 issues the tensor loads.
    int64_t issued = 0;
    const uint64_t policy = dev::policy_evict_first();
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++issued) {
      const int s = static_cast<int>(issued % STAGES);
      const int64_t round = issued / STAGES;
      bool ok = true;
      if (lane == 0) {
        if (round > 0) ok = dev::mbar_wait(&empty[s], static_cast<uint32_t>((round - 1) & 1), abort);
        if (ok) {
          unsigned char* stage = smem + s * K::STAGE_BYTES;
          const int y = static_cast<int>(c * RS);
          dev::mbar_arrive_expect_tx(&full[s], K::STAGE_BYTES);
#pragma unroll
          for (int q = 0; q < K::NBOX; ++q) {
            const int off = q * K::BOX_ROWS * 128, yq = y + q * K::BOX_ROWS;
#pragma unroll
            for (int b = 0; b < K::MBA; ++b)
              dev::tma_load_2d(stage + b * K::BOX_BYTES + off, &args.ta, 16 * b, yq, &full[s], policy);
#pragma unroll
            for (int b = 0; b < K::MBB; ++b)
              dev::tma_load_2d(stage + (K::MBA + b) * K::BOX_BYTES + off, &args.tb, 16 * b, yq, &full[s], policy);
          }
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else {
    // ---------------- consumer warps: k-steps of this warp's row slot.
    const int g = lane >> 2, tq = lane & 3;
    const int a_blk0 = ra * (MT / 2), b_blk0 = K::MBA + rb * (NT / 2);
    int64_t it = 0;
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++it) {
      const int s = static_cast<int>(it % STAGES);
      if (!dev::mbar_wait(&full[s], static_cast<uint32_t>((it / STAGES) & 1), abort)) {
        *abort = 1;
        atomicOr(p.error, dev::kErrTimeout);
        break;
      }
      const unsigned char* stage = smem + s * K::STAGE_BYTES;
#pragma unroll 2
      for (int ks = slot; ks < K::KSTEPS; ks += K::S) {
        // rows s, s+2, s+4, s+6 of 8-row group ks/2 (s = ks & 1); lane tq's row:
        const int row = 8 * (ks >> 1) + (ks & 1) + 2 * tq;
        const int off = row * 128 + ((g ^ (row & 7)) << 4);  // column pair (2g, 2g+1), swizzled
        double a[MT], b[NT];
#pragma unroll
        for (int i = 0; i < MT / 2; ++i) {
          const double2 v = *reinterpret_cast<const double2*>(stage + (a_blk0 + i) * K::BOX_BYTES + off);
          a[2 * i] = v.x;
          a[2 * i + 1] = v.y;
        }
#pragma unroll
        for (int j = 0; j < NT / 2; ++j) {
          const double2 v = *reinterpret_cast<const double2*>(stage + (b_blk0 + j) * K::BOX_BYTES + off);
          b[2 * j] = v.x;
          b[2 * j + 1] = v.y;
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) dev::dmma_m8n8k4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
      __syncwarp();
      if (lane == 0) dev::mbar_arrive(&empty[s]);
    }
  }

  __syncthreads();
  if (*abort && warp == CW && lane == 0) {
    // Let every tensor load this CTA issued land before the ring is reused.
    int64_t issued = 0;
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G) ++issued;
    volatile int no_abort = 0;
    for (int64_t q = issued > STAGES ? issued - STAGES : 0; q < issued; ++q)
      if (!dev::mbar_wait(&full[q % STAGES], static_cast<uint32_t>((q / STAGES) & 1), &no_abort)) break;
  }
  __syncthreads();

  // Each warp's tiles -> its slot's m x k sheet.  Tile (i, j) of the warp:
  // C row 16 (a block) + 2 g + (i & 1), C column 16 (b block) + 2 n + (j & 1)
  // for D column n = 2 tq + e.
  double* red = reinterpret_cast<double*>(smem);
  if (warp < CW) {
    const int g = lane >> 2, tq = lane & 3;
    double* sheet = red + slot * (WA * WB);
#pragma unroll
    for (int i = 0; i < MT; ++i) {
      const int row = 16 * (ra * (MT / 2) + (i >> 1)) + 2 * g + (i & 1);
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = 16 * (rb * (NT / 2) + (j >> 1)) + 2 * (2 * tq + e) + (j & 1);
          sheet[row * WB + col] = acc[i][j][e];
        }
    }
  }
  __syncthreads();
  detail::finish_partials(p, red, K::S, t, K::THREADS, s_is_last);
}

}  // namespace tsm

namespace tsm {

// ---------------------------------------------------------------------------
// Gram C = A^T A on the FP64 tensor cores, upper triangle only.
//
// The 16-column blocks b of A give 8x8 tiles 2b (even columns) and 2b + 1
// (odd columns).  Only block pairs (bi, bj) with bi <= bj are computed -- 4
// tiles each off the diagonal, 3 on it (tile (1, 0) of a diagonal pair is
// the transpose of tile (0, 1); gram_store writes it from that one) -- so
// C's upper triangle is complete and the lower one is written by mirroring
// (finish_partials with symmetric = 1).  Per k-step a warp loads each 16-column
// block its region touches ONCE and feeds both DMMA operands from it (B is A).
// Regions (lists of block pairs, DMMA tiles per k-step, <= 20 per region):
//   W = 16: {(0,0)}                                         1 region
//   W = 32: {(0,0),(0,1),(1,1)}                             1 region, 10 of 16 tiles
//   W = 48: {(0,0),(0,1),(1,1)}, {(0,2),(1,2),(2,2)}        21 of 36 tiles
//   W = 64: {(0,0),(0,1),(0,2),(0,3),(1,1)},
//           {(1,2),(1,3),(2,2),(2,3),(3,3)}                 36 of 64 tiles
// A pair is coded 4 bi + bj, four bits per pair.
__host__ __device__ constexpr int gram_regions(int W) { return W >= 48 ? 2 : 1; }
__host__ __device__ constexpr int gram_npairs(int W, int) { return W == 16 ? 1 : (W == 64 ? 5 : 3); }
__host__ __device__ constexpr unsigned gram_pair_codes(int W, int r) {
  return W == 16   ? 0x0u
         : W == 32 ? (0x0u | (0x1u << 4) | (0x5u << 8))
         : W == 48 ? (r == 0 ? (0x0u | (0x1u << 4) | (0x5u << 8)) : (0x2u | (0x6u << 4) | (0xAu << 8)))
         : r == 0  ? (0x0u | (0x1u << 4) | (0x2u << 8) | (0x3u << 12) | (0x5u << 16))
                   : (0x6u | (0x7u << 4) | (0xAu << 8) | (0xBu << 12) | (0xFu << 16));
}
constexpr int kGramMaxPairs = 5;
__host__ __device__ constexpr int gram_pair(int W, int r, int p) {
  return static_cast<int>((gram_pair_codes(W, r) >> (4 * p)) & 0xFu);
}
// Blocks a region touches (bit b: 16-column block b).
__host__ __device__ constexpr unsigned gram_block_mask(int W, int r) {
  unsigned mask = 0;
  for (int p = 0; p < gram_npairs(W, r); ++p) mask |= (1u << (gram_pair(W, r, p) >> 2)) | (1u << (gram_pair(W, r, p) & 3));
  return mask;
}

template <int W, int CW, int STAGES, int RS>
struct GramDmma {
  static_assert(W % 16 == 0 && W >= 16 && W <= 64, "width: multiple of 16 up to 64");
  static_assert(dmma_rows_ok(RS), "chunk rows: equal boxes of whole 8-row swizzle groups, <= 256 rows each");
  static constexpr int NBOX = dmma_boxes(RS), BOX_ROWS = dmma_box_rows(RS);
  static constexpr int NB = W / 16;
  static constexpr int R = gram_regions(W);
  static_assert(CW % R == 0, "consumer warps must cover whole regions");
  static constexpr int S = CW / R;
  static constexpr int KSTEPS = RS / 4;
  static constexpr int BOX_BYTES = RS * 128;  // one 16-column block of the chunk (NBOX tensor boxes)
  static constexpr int STAGE_BYTES = NB * BOX_BYTES;
  static constexpr int THREADS = CW * 32 + 32;
  static constexpr size_t RING_BYTES = size_t(STAGES) * STAGE_BYTES;
  static constexpr size_t RED_BYTES = size_t(S) * W * W * sizeof(double);
  static constexpr size_t DATA_BYTES = RING_BYTES > RED_BYTES ? RING_BYTES : RED_BYTES;
  static constexpr size_t BAR_OFFSET = (DATA_BYTES + 127) / 128 * 128;
  static constexpr size_t SMEM_BYTES = 1024 + BAR_OFFSET + 2 * STAGES * sizeof(uint64_t) + 16;
};

namespace detail {

// One consumer warp of region REG: every chunk's k-steps of its slot, then
// its tiles into the slot's sheet of `red` (after the caller's barrier).
template <int W, int CW, int STAGES, int RS, int REG>
__device__ __forceinline__ void gram_consume(const PlainArgs<double>& p, unsigned char* smem, uint64_t* full,
                                             uint64_t* empty, volatile int* abort, int slot, int lane,
                                             double (&out)[kGramMaxPairs][2][2][2]) {
  using K = GramDmma<W, CW, STAGES, RS>;
  constexpr int NP = gram_npairs(W, REG);
  constexpr unsigned MASK = gram_block_mask(W, REG);
  const int g = lane >> 2, tq = lane & 3;
  const int64_t G = gridDim.x;
#pragma unroll
  for (int q = 0; q < kGramMaxPairs; ++q)
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) out[q][a][b][0] = out[q][a][b][1] = 0.0;
  int64_t it = 0;
  for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++it) {
    const int s = static_cast<int>(it % STAGES);
    if (!dev::mbar_wait(&full[s], static_cast<uint32_t>((it / STAGES) & 1), abort)) {
      *abort = 1;
      atomicOr(p.error, dev::kErrTimeout);
      break;
    }
    const unsigned char* stage = smem + s * K::STAGE_BYTES;
#pragma unroll 2
    for (int ks = slot; ks < K::KSTEPS; ks += K::S) {
      const int row = 8 * (ks >> 1) + (ks & 1) + 2 * tq;
      const int off = row * 128 + ((g ^ (row & 7)) << 4);
      double v[K::NB][2];
#pragma unroll
      for (int b = 0; b < K::NB; ++b) {
        if (MASK & (1u << b)) {
          const double2 x = *reinterpret_cast<const double2*>(stage + b * K::BOX_BYTES + off);
          v[b][0] = x.x;
          v[b][1] = x.y;
        } else {
          v[b][0] = v[b][1] = 0.0;
        }
      }
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        const int bi = gram_pair(W, REG, q) >> 2, bj = gram_pair(W, REG, q) & 3;
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            if (bi == bj && a == 1 && b == 0) continue;  // the transpose of tile (0, 1): stored from it
            dev::dmma_m8n8k4(out[q][a][b][0], out[q][a][b][1], v[bi][a], v[bj][b]);
          }
      }
    }
    __syncwarp();
    if (lane == 0) dev::mbar_arrive(&empty[s]);
  }
}

// Tile (pair q, parities a, b) -> C row 16 bi + 2 g + a, column 16 bj + 2 n + b
// for D column n = 2 tq + e.  On a diagonal pair (bi = bj), tile (1, 0) is
// the transpose of tile (0, 1) -- entry (g, n) of one is entry (n, g) of the
// other, the same products summed over the same rows -- so the consumer
// skips its DMMAs and tile (0, 1) is stored a second time, transposed, in
// its place.  That brings the tiles per k-step to the upper triangle of the
// 8 x 8 tiles: 3 of 4 at W = 16, 10 of 16 at 32, 21 of 36 at 48, 36 of 64 at
// 64 (12, 24 and 40 before).
template <int W, int REG>
__device__ __forceinline__ void gram_store(double* sheet, int lane, const double (&out)[kGramMaxPairs][2][2][2]) {
  constexpr int NP = gram_npairs(W, REG);
  const int g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int q = 0; q < NP; ++q) {
    const int bi = gram_pair(W, REG, q) >> 2, bj = gram_pair(W, REG, q) & 3;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          if (bi == bj && a == 1 && b == 0)  // C[16 bi + 2 n + 1][16 bi + 2 g] = tile (0, 1) entry (g, n)
            sheet[(16 * bi + 2 * (2 * tq + e) + 1) * W + 16 * bi + 2 * g] = out[q][0][1][e];
          else
            sheet[(16 * bi + 2 * g + a) * W + 16 * bj + 2 * (2 * tq + e) + b] = out[q][a][b][e];
        }
  }
}

}  // namespace detail

template <int W, int CW, int STAGES, int RS>
__global__ void __launch_bounds__(GramDmma<W, CW, STAGES, RS>::THREADS, 1)
    tsm_gram_dmma_kernel(const __grid_constant__ DmmaArgs args) {
  using K = GramDmma<W, CW, STAGES, RS>;
  const PlainArgs<double>& p = args.p;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024u - (dev::smem_u32(smem_raw) & 1023u)) & 1023u);
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
  if (warp == CW && lane == 0 && blockIdx.x < p.num_chunks) dev::prefetch_tensormap(&args.ta);
  __syncthreads();

  const int64_t G = gridDim.x;
  const int region = warp % K::R, slot = warp / K::R;
  double out[kGramMaxPairs][2][2][2];

  if (warp == CW) {
    // ---------------- producer warp: A's boxes only.
    int64_t issued = 0;
    const uint64_t policy = dev::policy_evict_first();
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G, ++issued) {
      const int s = static_cast<int>(issued % STAGES);
      const int64_t round = issued / STAGES;
      bool ok = true;
      if (lane == 0) {
        if (round > 0) ok = dev::mbar_wait(&empty[s], static_cast<uint32_t>((round - 1) & 1), abort);
        if (ok) {
          unsigned char* stage = smem + s * K::STAGE_BYTES;
          const int y = static_cast<int>(c * RS);
          dev::mbar_arrive_expect_tx(&full[s], K::STAGE_BYTES);
#pragma unroll
          for (int q = 0; q < K::NBOX; ++q)
#pragma unroll
            for (int b = 0; b < K::NB; ++b)
              dev::tma_load_2d(stage + b * K::BOX_BYTES + q * K::BOX_ROWS * 128, &args.ta, 16 * b,
                               y + q * K::BOX_ROWS, &full[s], policy);
        } else {
          *abort = 1;
          atomicOr(p.error, dev::kErrTimeout);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
    }
  } else if (region == 0) {
    detail::gram_consume<W, CW, STAGES, RS, 0>(p, smem, full, empty, abort, slot, lane, out);
  } else {
    detail::gram_consume<W, CW, STAGES, RS, (K::R > 1 ? 1 : 0)>(p, smem, full, empty, abort, slot, lane, out);
  }

  __syncthreads();
  if (*abort && warp == CW && lane == 0) {
    int64_t issued = 0;
    for (int64_t c = blockIdx.x; c < p.num_chunks; c += G) ++issued;
    volatile int no_abort = 0;
    for (int64_t q = issued > STAGES ? issued - STAGES : 0; q < issued; ++q)
      if (!dev::mbar_wait(&full[q % STAGES], static_cast<uint32_t>((q / STAGES) & 1), &no_abort)) break;
  }
  __syncthreads();

  // Tiles -> the slot's W x W sheet (the upper triangle is complete; cells
  // below the diagonal blocks are never read by the symmetric finish).
  double* red = reinterpret_cast<double*>(smem);
  if (warp < CW) {
    double* sheet = red + slot * (W * W);
    if (region == 0)
      detail::gram_store<W, 0>(sheet, lane, out);
    else
      detail::gram_store<W, (K::R > 1 ? 1 : 0)>(sheet, lane, out);
  }
  __syncthreads();
  detail::finish_partials(p, red, K::S, t, K::THREADS, s_is_last);
}

}  // namespace tsm
