// tsm_split.cu -- C ABI of the precision form (FP32 storage, hi/lo parts on
// the tcgen05 tensor cores, FP64 reductions).  TF32 parts: tsm_split_tma.cuh
// (widths that are multiples of 4: 2-D TMA straight into the MMA layout) and
// tsm_split.cuh (any width: 1-D bulk copies and a converter pass).  BF16
// parts (two or three): tsm_split_bf16.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/tsm.h"
#include "tsm_errors.h"
#include "tsm_split.cuh"
#include "tsm_split_bf16.cuh"
#include "tsm_split_tma.cuh"
#include "tsm_tmap.h"

namespace tsm {
namespace {

std::mutex g_split_mu;
int g_split_sms[64] = {};
bool g_split_attr[64] = {};
bool g_split_tma_attr[64] = {};

tsm_status split_fail(cudaError_t e, const char* what) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  last_error() = buf;
  return TSM_ERROR_CUDA;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Rows per chunk of the TMA kernel, and chunks an issuer accumulates in TMEM
// before the epilogue drains them (FP32 accumulation over 256 rows).  Timed
// at n = 2^25, 32 x 32 on one B200 against the FP64 oracle: 64-row chunks
// 2.35-2.6 ms (the per-chunk handshakes and drains cost more than the finer
// stages win); drains every chunk 1.77 ms sustained, 1.9e-7 normwise error;
// every 2 chunks 1.62 ms, 4.9e-7; every 4 chunks 1.60 ms but 1.3e-6, above
// the stated 1e-6.
constexpr int kTmaRows = 128;
constexpr int kTmaDrain = 2;
using TmaCfg = split2::Cfg<kTmaRows>;

int64_t rows_for_bulk(int64_t n, int m, int k) {
  auto need = [](int w) {
    const int bytes = 4 * w;
    int g = 16, b = bytes;
    while (b) {
      const int t = g % b;
      g = b;
      b = t;
    }
    return static_cast<int64_t>(16 / g);
  };
  const int64_t r0 = std::max(need(m), need(k));
  return n - n % r0;
}

}  // namespace
}  // namespace tsm

using namespace tsm;

extern "C" tsm_status tsm_gemm_tn_f32_split(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                                            const float* B, int64_t ldb, double* C, int64_t ldc, int accumulate,
                                            void* workspace, size_t workspace_bytes) {
  if (n < 0 || m < 1 || k < 1 || m > 32 || k > 32 || ldc < k || C == nullptr) return TSM_ERROR_INVALID_VALUE;
  if (n > 0 && (A == nullptr || B == nullptr)) return TSM_ERROR_INVALID_VALUE;
  if (lda != m || ldb != k || !aligned16(A) || !aligned16(B)) return TSM_ERROR_UNSUPPORTED;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return split_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return TSM_ERROR_UNSUPPORTED;
  {
    std::lock_guard<std::mutex> lk(g_split_mu);
    if (g_split_sms[dev] == 0) {
      e = cudaDeviceGetAttribute(&g_split_sms[dev], cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return split_fail(e, "cudaDeviceGetAttribute");
    }
    if (!g_split_attr[dev]) {
      e = cudaFuncSetAttribute(reinterpret_cast<const void*>(&tsm_tn_split_tf32_kernel),
                               cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(split::kSmemBytes));
      if (e != cudaSuccess) return split_fail(e, "cudaFuncSetAttribute(split)");
      g_split_attr[dev] = true;
    }
  }
  const int sms = g_split_sms[dev];
  const size_t need = 256 + static_cast<size_t>(sms) * 4 * m * k * sizeof(double);
  if (workspace == nullptr || workspace_bytes < need || !aligned16(workspace)) return TSM_ERROR_WORKSPACE;
  // Widths that are multiples of 4 floats (16-byte row pitches): tensor maps.
  const bool tma = m % 4 == 0 && k % 4 == 0 && n <= static_cast<int64_t>(INT_MAX) - TmaCfg::kRows;
  SplitArgs p{};
  p.A = A;
  p.B = B;
  p.C = C;
  p.n = n;
  p.m = m;
  p.k = k;
  p.ldc = ldc;
  p.accumulate = accumulate ? 1 : 0;
  unsigned char* base = static_cast<unsigned char*>(workspace);
  p.counter = reinterpret_cast<unsigned*>(base);
  p.error = reinterpret_cast<unsigned*>(base) + 1;
  p.partials = reinterpret_cast<double*>(base + 256);
  if (tma) {
    {
      std::lock_guard<std::mutex> lk(g_split_mu);
      if (!g_split_tma_attr[dev]) {
        e = cudaFuncSetAttribute(reinterpret_cast<const void*>(&tsm_tn_split_tf32_tma_kernel<kTmaRows, kTmaDrain>),
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(TmaCfg::kSmemBytes));
        if (e != cudaSuccess) return split_fail(e, "cudaFuncSetAttribute(split tma)");
        g_split_tma_attr[dev] = true;
      }
    }
    SplitTmaArgs a{};
    p.rows_main = n;  // the tensor maps zero-fill past row n
    p.num_chunks = (n + TmaCfg::kRows - 1) / TmaCfg::kRows;
    a.p = p;
    if (n > 0) {  // n = 0: no chunks, the maps are never read
      if (!encode_rowmajor_map(&a.ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, A, n, m, lda, 32, TmaCfg::kRows,
                               CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, &last_error()) ||
          !encode_rowmajor_map(&a.tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, B, n, k, ldb, 32, TmaCfg::kRows,
                               CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, &last_error()))
        return TSM_ERROR_CUDA;
    }
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(p.num_chunks, sms));
    void* args[] = {&a};
    e = cudaLaunchKernel(reinterpret_cast<const void*>(&tsm_tn_split_tf32_tma_kernel<kTmaRows, kTmaDrain>),
                         dim3(static_cast<unsigned>(grid)), dim3(TmaCfg::kThreads), args, TmaCfg::kSmemBytes,
                         static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return split_fail(e, "cudaLaunchKernel(split tma)");
    return TSM_SUCCESS;
  }
  p.rows_main = rows_for_bulk(n, m, k);
  p.num_chunks = (p.rows_main + split::kRows - 1) / split::kRows;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(p.num_chunks, sms));
  void* args[] = {&p};
  e = cudaLaunchKernel(reinterpret_cast<const void*>(&tsm_tn_split_tf32_kernel), dim3(static_cast<unsigned>(grid)),
                       dim3(split::kThreads), args, split::kSmemBytes, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return split_fail(e, "cudaLaunchKernel(split)");
  return TSM_SUCCESS;
}

// ---------------------------------------------------------------------------
// BF16 parts (tsm_split_bf16.cuh): 2 (hi/lo) or 3 (hi/mid/lo) parts.
namespace tsm {
namespace {
bool g_split16_attr[64][2] = {};
}  // namespace
}  // namespace tsm

extern "C" tsm_status tsm_gemm_tn_f32_split_bf16(tsm_stream_t stream, int64_t n, int m, int k, const float* A,
                                                 int64_t lda, const float* B, int64_t ldb, double* C, int64_t ldc,
                                                 int accumulate, int parts, void* workspace,
                                                 size_t workspace_bytes) {
  if (n < 0 || m < 1 || k < 1 || m > 32 || k > 32 || ldc < k || C == nullptr) return TSM_ERROR_INVALID_VALUE;
  if (parts != 2 && parts != 3) return TSM_ERROR_INVALID_VALUE;
  if (n > 0 && (A == nullptr || B == nullptr)) return TSM_ERROR_INVALID_VALUE;
  // Tensor maps: 16-byte row pitches and bases, 32-bit row coordinates.
  if (lda != m || ldb != k || m % 4 != 0 || k % 4 != 0 || !aligned16(A) || !aligned16(B) ||
      n > static_cast<int64_t>(INT_MAX) - split16::kRows)
    return TSM_ERROR_UNSUPPORTED;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return split_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return TSM_ERROR_UNSUPPORTED;
  const void* fn = parts == 2 ? reinterpret_cast<const void*>(&tsm_tn_split_bf16_kernel<2, split16::kFlushDefault>)
                              : reinterpret_cast<const void*>(&tsm_tn_split_bf16_kernel<3, split16::kFlushDefault>);
  const size_t smem = parts == 2 ? split16::Shape<2>::SMEM_BYTES : split16::Shape<3>::SMEM_BYTES;
  {
    std::lock_guard<std::mutex> lk(g_split_mu);
    if (g_split_sms[dev] == 0) {
      e = cudaDeviceGetAttribute(&g_split_sms[dev], cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return split_fail(e, "cudaDeviceGetAttribute");
    }
    if (!g_split16_attr[dev][parts - 2]) {
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e != cudaSuccess) return split_fail(e, "cudaFuncSetAttribute(split bf16)");
      g_split16_attr[dev][parts - 2] = true;
    }
  }
  const int sms = g_split_sms[dev];
  const size_t need = 256 + static_cast<size_t>(sms) * 4 * m * k * sizeof(double);
  if (workspace == nullptr || workspace_bytes < need || !aligned16(workspace)) return TSM_ERROR_WORKSPACE;
  SplitTmaArgs a{};
  SplitArgs& p = a.p;
  p.A = A;
  p.B = B;
  p.C = C;
  p.n = n;
  p.m = m;
  p.k = k;
  p.ldc = ldc;
  p.accumulate = accumulate ? 1 : 0;
  unsigned char* base = static_cast<unsigned char*>(workspace);
  p.counter = reinterpret_cast<unsigned*>(base);
  p.error = reinterpret_cast<unsigned*>(base) + 1;
  p.partials = reinterpret_cast<double*>(base + 256);
  p.rows_main = n;  // the tensor maps zero-fill past row n
  p.num_chunks = (n + split16::kRows - 1) / split16::kRows;
  if (n > 0) {  // n = 0: no chunks, the maps are never read
    if (!encode_rowmajor_map(&a.ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, A, n, m, lda, 32, split16::kRows,
                             CU_TENSOR_MAP_SWIZZLE_NONE, &last_error()) ||
        !encode_rowmajor_map(&a.tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, B, n, k, ldb, 32, split16::kRows,
                             CU_TENSOR_MAP_SWIZZLE_NONE, &last_error()))
      return TSM_ERROR_CUDA;
  }
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(p.num_chunks, sms));
  void* args[] = {&a};
  e = cudaLaunchKernel(fn, dim3(static_cast<unsigned>(grid)), dim3(split16::kThreads), args, smem,
                       static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return split_fail(e, "cudaLaunchKernel(split bf16)");
  return TSM_SUCCESS;
}
