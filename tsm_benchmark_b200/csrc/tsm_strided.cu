// tsm_strided.cu -- C ABI of the general-layout product,
// tsm_gemm_tn_strided_f64: A's element (r, i) at A[r * a_row + i * a_col],
// B's (r, j) at B[r * b_row + j * b_col].
//
// Routing:
//   * both operands row-major (unit column stride, row pitch >= width):
//     tsm_gemm_tn_f64, the tuned plain path (Gram detection included);
//   * both column-major (unit row stride, column pitch >= n; A stored as
//     the m x n row-major A^T) with 16-byte aligned bases and even pitches:
//     the tensor-map kernels of tsm_strided.cuh -- SIMT when the width
//     capacities (powers of two) hold WA * WB <= 64, FP64 tensor cores with
//     capacities 8, 16, 32, 48 or 64 otherwise;
//   * anything else (mixed layouts, odd pitches, unaligned bases, overlapping
//     strides): the register-tile kernel with plain strided loads.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/tsm.h"
#include "tsm_errors.h"
#include "tsm_strided.cuh"
#include "tsm_tmap.h"

namespace tsm {
namespace {

constexpr size_t kWsHeader = 256;  // [counter u32][error u32][pad]; partials follow
constexpr int kMaxCtasPerSm = 4;   // workspace: sms * 4 partials of m x k
constexpr int kMaxDevices = 64;

tsm_status strided_fail(cudaError_t e, const char* what) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  last_error() = buf;
  return TSM_ERROR_CUDA;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Compile-time launch shapes.
// SIMT: chunks of up to ~96 KB (whole boxes of 256 values of r above 256,
// whole warps of r below, at least 64), two stages.  At n = 2^26 three
// stages of ~64 KB ran 1-3.4 % faster than six of ~32 KB, and two of ~96 KB
// 2-3.5 % faster again at 2 x 2, 8 x 8, 2 x 32 and 1 x 64 (1 x 1, 4 x 4 and
// 4 x 16 within 0.5 %).
constexpr int cm_simt_rs(int wa, int wb) {
  return 12288 / (wa + wb) >= 256 ? std::min(6144, 12288 / (wa + wb) / 256 * 256)
                                  : std::max(64, 12288 / (wa + wb) / 32 * 32);
}
constexpr int kCmSimtStages = 2;
// DMMA: regions of at most 4 x 4 tiles, 8 consumer warps, chunks of whole
// 16-value groups sized for two ~98 KB stages (boxes of RS + 2 <= 242
// values), as many stages as fit 220 KB (2 to 4).  Against ~64 KB chunks
// (three interleaved rounds, one B200): 32 x 32 at 2^25 7143-7159 vs
// 6894-6944 GB/s, 32 x 64 at 2^24 6227-6282 vs 5957-6038, 64 x 64 at 2^23
// 4186-4210 vs 4148-4169; 16 x 16 and narrower keep their 240-value chunks.
constexpr int cm_tiles(int w) {
  return (w / 8) % 4 == 0 ? 4 : (w / 8) % 3 == 0 ? 3 : (w / 8) % 2 == 0 ? 2 : 1;
}
constexpr int cm_dmma_rs(int wa, int wb) { return std::min(240, std::max(16, (12544 / (wa + wb) - 2) / 16 * 16)); }
constexpr int cm_dmma_stages(int wa, int wb) {
  return std::max(2, std::min(4, (220 * 1024) / ((wa + wb) * 8 * (cm_dmma_rs(wa, wb) + 2))));
}

struct Kernel {
  int wa, wb;    // capacities
  int rs;        // values of r per chunk (tensor-map kernels)
  int threads;
  size_t smem;
  const void* fn;
};

#define CM_SIMT(WA, WB)                                                                                     \
  Kernel {                                                                                                  \
    WA, WB, cm_simt_rs(WA, WB), CmSimt<WA, WB, cm_simt_rs(WA, WB), kCmSimtStages>::THREADS,                 \
        CmSimt<WA, WB, cm_simt_rs(WA, WB), kCmSimtStages>::SMEM_BYTES,                                      \
        reinterpret_cast<const void*>(&tsm_tn_cm_simt_kernel<WA, WB, cm_simt_rs(WA, WB), kCmSimtStages>) \
  }
#define CM_SIMT_ROW(WA) CM_SIMT(WA, 1), CM_SIMT(WA, 2), CM_SIMT(WA, 4), CM_SIMT(WA, 8)

const Kernel kCmSimt[] = {
    CM_SIMT_ROW(1), CM_SIMT(1, 16), CM_SIMT(1, 32), CM_SIMT(1, 64),
    CM_SIMT_ROW(2), CM_SIMT(2, 16), CM_SIMT(2, 32),
    CM_SIMT_ROW(4), CM_SIMT(4, 16),
    CM_SIMT_ROW(8),
    CM_SIMT(16, 1), CM_SIMT(16, 2), CM_SIMT(16, 4),
    CM_SIMT(32, 1), CM_SIMT(32, 2),
    CM_SIMT(64, 1),
};

#define CM_DMMA_T(WA, WB)                                                                                    \
  tsm_tn_cm_dmma_kernel<WA, WB, cm_tiles(WA), cm_tiles(WB), 8, cm_dmma_stages(WA, WB), cm_dmma_rs(WA, WB)>
#define CM_DMMA(WA, WB)                                                                                      \
  Kernel {                                                                                                   \
    WA, WB, cm_dmma_rs(WA, WB),                                                                              \
        CmDmma<WA, WB, cm_tiles(WA), cm_tiles(WB), 8, cm_dmma_stages(WA, WB), cm_dmma_rs(WA, WB)>::THREADS,  \
        CmDmma<WA, WB, cm_tiles(WA), cm_tiles(WB), 8, cm_dmma_stages(WA, WB), cm_dmma_rs(WA, WB)>::SMEM_BYTES, \
        reinterpret_cast<const void*>(&CM_DMMA_T(WA, WB))                                                   \
  }
#define CM_DMMA_ROW(WA) CM_DMMA(WA, 8), CM_DMMA(WA, 16), CM_DMMA(WA, 32), CM_DMMA(WA, 48), CM_DMMA(WA, 64)

// Capacity 8 (one tile) keeps 4 x 32 or 8 x 16 from padding to 16 x ...
const Kernel kCmDmma[] = {CM_DMMA(8, 16), CM_DMMA(8, 32), CM_DMMA(8, 48), CM_DMMA(8, 64), CM_DMMA(16, 8),
                          CM_DMMA(32, 8), CM_DMMA(48, 8), CM_DMMA(64, 8), CM_DMMA_ROW(16), CM_DMMA_ROW(32),
                          CM_DMMA_ROW(48), CM_DMMA_ROW(64)};

#define STRIDED(WA, WB)                                                                                     \
  Kernel {                                                                                                  \
    WA, WB, 0, 256, StridedKernel<WA, WB, 8, 8, 256>::SMEM_BYTES,                                           \
        reinterpret_cast<const void*>(&tsm_tn_strided_kernel<WA, WB, 8, 8, 256>)                           \
  }
const Kernel kStrided[] = {STRIDED(8, 8), STRIDED(8, 64), STRIDED(64, 8), STRIDED(64, 64)};

constexpr int kNumCmSimt = sizeof(kCmSimt) / sizeof(Kernel);
constexpr int kNumCmDmma = sizeof(kCmDmma) / sizeof(Kernel);
constexpr int kNumStrided = sizeof(kStrided) / sizeof(Kernel);
constexpr int kNumKernels = kNumCmSimt + kNumCmDmma + kNumStrided;

struct DeviceInfo {
  int sms = 0;
  signed char ready[kNumKernels] = {};  // 1: attribute set, -1: failed
  int ctas[kNumKernels] = {};           // resident CTAs per SM (<= kMaxCtasPerSm)
};

std::mutex g_mu;
DeviceInfo g_dev[kMaxDevices];

const Kernel* kernel_at(int idx) {
  if (idx < kNumCmSimt) return &kCmSimt[idx];
  if (idx < kNumCmSimt + kNumCmDmma) return &kCmDmma[idx - kNumCmSimt];
  return &kStrided[idx - kNumCmSimt - kNumCmDmma];
}

int find_kernel(const Kernel* table, int count, int base, int wa, int wb) {
  for (int i = 0; i < count; ++i)
    if (table[i].wa == wa && table[i].wb == wb) return base + i;
  return -1;
}

// Tensor-core capacities: 8, 16, 32, 48, 64.
int dmma_capacity(int w) { return w <= 8 ? 8 : w <= 16 ? 16 : w <= 32 ? 32 : w <= 48 ? 48 : 64; }

int pow2_ceil(int x) {
  int p = 1;
  while (p < x) p *= 2;
  return p;
}

tsm_status prepare(int dev, int idx, int* sms, int* ctas) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceInfo& d = g_dev[dev];
  cudaError_t e;
  if (d.sms == 0) {
    e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return strided_fail(e, "cudaDeviceGetAttribute");
  }
  *sms = d.sms;
  if (d.ready[idx] == -1) return TSM_ERROR_UNSUPPORTED;
  if (d.ready[idx] == 0) {
    const Kernel* k = kernel_at(idx);
    e = cudaFuncSetAttribute(k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(k->smem));
    if (e != cudaSuccess) {
      d.ready[idx] = -1;
      return strided_fail(e, "cudaFuncSetAttribute(strided)");
    }
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k->fn, k->threads, k->smem);
    if (e != cudaSuccess) return strided_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (occ < 1) {
      d.ready[idx] = -1;
      return TSM_ERROR_UNSUPPORTED;
    }
    d.ctas[idx] = std::min(occ, kMaxCtasPerSm);
    d.ready[idx] = 1;
  }
  *ctas = d.ctas[idx];
  return TSM_SUCCESS;
}

// Map of an operand stored transposed (w rows of n values, pitch ld >= n):
// boxes of box_r values x box_w rows.
bool encode_transposed(CUtensorMap* map, const double* base, int64_t n, int w, int64_t ld, int box_r, int box_w,
                       CUtensorMapSwizzle swizzle) {
  return encode_rowmajor_map(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, base, w, static_cast<int>(n), ld, box_r, box_w,
                             swizzle, &last_error());
}

}  // namespace
}  // namespace tsm

using namespace tsm;

extern "C" tsm_status tsm_gemm_tn_strided_f64(tsm_stream_t stream, int64_t n, int m, int k, const double* A,
                                              int64_t a_row, int64_t a_col, const double* B, int64_t b_row,
                                              int64_t b_col, double* C, int64_t ldc, int accumulate,
                                              void* workspace, size_t workspace_bytes) {
  if (n < 0 || m < 1 || k < 1 || m > 64 || k > 64 || ldc < k || C == nullptr) return TSM_ERROR_INVALID_VALUE;
  if (a_row < 1 || a_col < 1 || b_row < 1 || b_col < 1) return TSM_ERROR_INVALID_VALUE;
  if (n > 0 && (A == nullptr || B == nullptr)) return TSM_ERROR_INVALID_VALUE;
  // A stride along an extent of one is never used.
  if (m == 1) a_col = 1;
  if (k == 1) b_col = 1;

  // 1. Row-major operands: the plain path.
  if (a_col == 1 && b_col == 1 && a_row >= m && b_row >= k)
    return tsm_gemm_tn_f64(stream, n, m, k, A, a_row, B, b_row, C, ldc, accumulate, workspace, workspace_bytes);

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return strided_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return TSM_ERROR_UNSUPPORTED;

  // 2. Column-major operands that tensor maps can describe.
  const bool cm_a = (a_row == 1 || n == 1) && (m == 1 || (a_col >= n && a_col % 2 == 0));
  const bool cm_b = (b_row == 1 || n == 1) && (k == 1 || (b_col >= n && b_col % 2 == 0));
  // Box coordinates are 32-bit: the last chunk's boxes start below n + RS
  // (RS <= 6144), so n leaves that much room below INT_MAX.
  const bool tma_ok = aligned16(A) && aligned16(B) && n <= static_cast<int64_t>(INT_MAX) - 8192;
  int idx = -1;
  if (cm_a && cm_b && tma_ok) {
    const int wa = pow2_ceil(m), wb = pow2_ceil(k);
    if (wa * wb <= 64) {
      idx = find_kernel(kCmSimt, kNumCmSimt, 0, wa, wb);
    } else {
      idx = find_kernel(kCmDmma, kNumCmDmma, kNumCmSimt, dmma_capacity(m), dmma_capacity(k));
    }
  }
  const bool tensor_maps = idx >= 0;
  if (!tensor_maps) {
    idx = find_kernel(kStrided, kNumStrided, kNumCmSimt + kNumCmDmma, m <= 8 ? 8 : 64, k <= 8 ? 8 : 64);
    if (idx < 0) return TSM_ERROR_UNSUPPORTED;
  }

  int sms = 0, ctas = 0;
  tsm_status s = prepare(dev, idx, &sms, &ctas);
  if (s != TSM_SUCCESS) return s;
  const size_t need = kWsHeader + static_cast<size_t>(sms) * kMaxCtasPerSm * m * k * sizeof(double);
  if (workspace == nullptr || workspace_bytes < need || !aligned16(workspace)) return TSM_ERROR_WORKSPACE;

  const Kernel* kern = kernel_at(idx);
  PlainArgs<double> p{};
  p.A = A;
  p.B = B;
  p.C = C;
  p.n = n;
  p.m = m;
  p.k = k;
  p.lda = m;  // unused: rows_main = n leaves no rows to the reduction epilogue
  p.ldb = k;
  p.ldc = ldc;
  p.accumulate = accumulate ? 1 : 0;
  p.symmetric = 0;
  p.rows_main = n;
  unsigned char* base = static_cast<unsigned char*>(workspace);
  p.counter = reinterpret_cast<unsigned*>(base);
  p.error = reinterpret_cast<unsigned*>(base) + 1;
  p.partials = reinterpret_cast<double*>(base + kWsHeader);
  const int64_t max_grid = static_cast<int64_t>(sms) * ctas;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);

  if (tensor_maps) {
    CmArgs a{};
    p.num_chunks = (n + kern->rs - 1) / kern->rs;
    a.p = p;
    if (n > 0) {  // n = 0: no chunks, the maps are never read
      // A single column (m = 1) has no pitch of its own; any legal one will do.
      const int64_t lda = m == 1 ? (n + 1) / 2 * 2 : a_col;
      const int64_t ldb = k == 1 ? (n + 1) / 2 * 2 : b_col;
      // SIMT: boxes of up to 256 values; DMMA: RS + 2 (row skew).
      const int box_r = idx < kNumCmSimt ? std::min(kern->rs, 256) : kern->rs + 2;
      if (!encode_transposed(&a.ta, A, n, m, lda, box_r, kern->wa, CU_TENSOR_MAP_SWIZZLE_NONE) ||
          !encode_transposed(&a.tb, B, n, k, ldb, box_r, kern->wb, CU_TENSOR_MAP_SWIZZLE_NONE))
        return TSM_ERROR_CUDA;
    }
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(p.num_chunks, max_grid));
    void* args[] = {&a};
    e = cudaLaunchKernel(kern->fn, dim3(static_cast<unsigned>(grid)), dim3(kern->threads), args, kern->smem, cs);
    if (e != cudaSuccess) return strided_fail(e, "cudaLaunchKernel(column-major)");
    return TSM_SUCCESS;
  }

  StridedArgs a{};
  p.num_chunks = 0;
  a.p = p;
  a.a_row = a_row;
  a.a_col = a_col;
  a.b_row = b_row;
  a.b_col = b_col;
  const int tiles = (kern->wa / 8) * (kern->wb / 8);
  const int64_t row_groups = kern->threads / tiles;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((n + row_groups - 1) / row_groups, max_grid));
  void* args[] = {&a};
  e = cudaLaunchKernel(kern->fn, dim3(static_cast<unsigned>(grid)), dim3(kern->threads), args, kern->smem, cs);
  if (e != cudaSuccess) return strided_fail(e, "cudaLaunchKernel(strided)");
  return TSM_SUCCESS;
}
