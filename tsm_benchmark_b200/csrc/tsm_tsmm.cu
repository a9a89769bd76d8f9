// tsm_tsmm.cu -- C ABI of the backward products (TSMM) and of the fused
// backward of C = A^T B.  Kernels: csrc/tsm_tsmm.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/tsm.h"
#include "tsm_errors.h"
#include "tsm_tsmm.cuh"
#include "tsm_tsmm_dmma.cuh"

namespace tsm {
namespace {

// Two CTAs per SM where registers allow (3 stages of ~32 KB each): 1-2 %
// faster on the fused backward than one CTA with 4 stages.
constexpr int kCW = 8, kStages = 3, kCtasPerSm = 2;

// SIMT kernels with direct loads: X with any row stride or alignment.
struct TsmmEntry {
  int dtype;  // 0 f64, 1 f32
  int cap;
  const void* direct;
};

#define TSM_TSMM_ENTRY(T, DT, C) \
  TsmmEntry { DT, C, reinterpret_cast<const void*>(&tsm_tsmm_direct_kernel<T, C, 256>) }

const TsmmEntry kTsmm[] = {
    TSM_TSMM_ENTRY(double, 0, 1),  TSM_TSMM_ENTRY(double, 0, 2),  TSM_TSMM_ENTRY(double, 0, 4),
    TSM_TSMM_ENTRY(double, 0, 8),  TSM_TSMM_ENTRY(double, 0, 16), TSM_TSMM_ENTRY(double, 0, 32),
    TSM_TSMM_ENTRY(double, 0, 64), TSM_TSMM_ENTRY(float, 1, 1),   TSM_TSMM_ENTRY(float, 1, 2),
    TSM_TSMM_ENTRY(float, 1, 4),   TSM_TSMM_ENTRY(float, 1, 8),   TSM_TSMM_ENTRY(float, 1, 16),
    TSM_TSMM_ENTRY(float, 1, 32),  TSM_TSMM_ENTRY(float, 1, 64),
};
constexpr int kTsmmCount = sizeof(kTsmm) / sizeof(kTsmm[0]);

// FP64 tensor-core (DMMA) kernels for dense, aligned X, FP64 or FP32
// storage: capacities P, Q in {4, 8, 16, 32, 64}, ~32 KB stages.
struct DmmaEntry {
  int dtype;  // 0 f64, 1 f32
  int P, Q;
  bool ys;  // Y += X W with the old Y rows staged beside X (beta = 1, dense Y)
  const void* fn;
  int threads;
  size_t smem;
  int rows;
};

template <typename T, int P>
constexpr int dmma_rows() {
  // FP32 X with P >= 16: 64 KB stages (one CTA per SM by occupancy), 5-7 %
  // faster than 32 KB at 16 x 16 and 32 x 32, 5 % slower at 8 x 8.
  return (sizeof(T) == 4 && P >= 16 ? 65536 : 32768) / (P * int(sizeof(T)));
}

// Staged-Y kernels (beta = 1, dense Y): stages of ~64 KB holding the X rows
// and the old Y rows of a chunk; rows a power of two.
template <typename T, int P, int Q>
constexpr int dmma_ys_rows() {
  int r = 1;
  while (2 * r * (P + Q) * int(sizeof(T)) <= 65536) r *= 2;
  return r;
}

#define TSM_DMMA_ENTRY(T, DT, P, Q)                                                                            \
  DmmaEntry {                                                                                                  \
    DT, P, Q, false,                                                                                           \
        reinterpret_cast<const void*>(&tsm_tsmm_dmma_kernel<T, P, Q, kCW, kStages, dmma_rows<T, P>()>),         \
        TsmmDmmaKernel<T, P, Q, kCW, kStages, dmma_rows<T, P>()>::THREADS,                                      \
        TsmmDmmaKernel<T, P, Q, kCW, kStages, dmma_rows<T, P>()>::SMEM_BYTES, dmma_rows<T, P>()                 \
  }
#define TSM_DMMA_YS_ENTRY(T, DT, P, Q)                                                                            \
  DmmaEntry {                                                                                                     \
    DT, P, Q, true,                                                                                               \
        reinterpret_cast<const void*>(&tsm_tsmm_dmma_kernel<T, P, Q, kCW, kStages, dmma_ys_rows<T, P, Q>(), true>), \
        TsmmDmmaKernel<T, P, Q, kCW, kStages, dmma_ys_rows<T, P, Q>(), true>::THREADS,                             \
        TsmmDmmaKernel<T, P, Q, kCW, kStages, dmma_ys_rows<T, P, Q>(), true>::SMEM_BYTES,                          \
        dmma_ys_rows<T, P, Q>()                                                                                   \
  }
#define TSM_DMMA_ROW(T, DT, P)                                                                              \
  TSM_DMMA_ENTRY(T, DT, P, 4), TSM_DMMA_ENTRY(T, DT, P, 8), TSM_DMMA_ENTRY(T, DT, P, 16),                   \
      TSM_DMMA_ENTRY(T, DT, P, 32), TSM_DMMA_ENTRY(T, DT, P, 64)
#define TSM_DMMA_YS_ROW(T, DT, P)                                                                           \
  TSM_DMMA_YS_ENTRY(T, DT, P, 4), TSM_DMMA_YS_ENTRY(T, DT, P, 8), TSM_DMMA_YS_ENTRY(T, DT, P, 16),          \
      TSM_DMMA_YS_ENTRY(T, DT, P, 32), TSM_DMMA_YS_ENTRY(T, DT, P, 64)

const DmmaEntry kDmma[] = {
    TSM_DMMA_ROW(double, 0, 4),     TSM_DMMA_ROW(double, 0, 8),     TSM_DMMA_ROW(double, 0, 16),
    TSM_DMMA_ROW(double, 0, 32),    TSM_DMMA_ROW(double, 0, 64),    TSM_DMMA_ROW(float, 1, 4),
    TSM_DMMA_ROW(float, 1, 8),      TSM_DMMA_ROW(float, 1, 16),     TSM_DMMA_ROW(float, 1, 32),
    TSM_DMMA_ROW(float, 1, 64),     TSM_DMMA_YS_ROW(double, 0, 4),  TSM_DMMA_YS_ROW(double, 0, 8),
    TSM_DMMA_YS_ROW(double, 0, 16), TSM_DMMA_YS_ROW(double, 0, 32), TSM_DMMA_YS_ROW(double, 0, 64),
    TSM_DMMA_YS_ROW(float, 1, 4),   TSM_DMMA_YS_ROW(float, 1, 8),   TSM_DMMA_YS_ROW(float, 1, 16),
    TSM_DMMA_YS_ROW(float, 1, 32),  TSM_DMMA_YS_ROW(float, 1, 64),
};
constexpr int kDmmaCount = sizeof(kDmma) / sizeof(kDmma[0]);

std::mutex g_tsmm_mu;
int g_sms[64] = {};
signed char g_dmma_ready[64][kDmmaCount] = {};
int g_dmma_ctas[64][kDmmaCount] = {};  // resident CTAs per SM, <= kCtasPerSm

tsm_status fail(cudaError_t e, const char* what) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  last_error() = buf;
  return TSM_ERROR_CUDA;
}

int cap_of(int w) {
  int c = 1;
  while (c < w) c <<= 1;
  return c;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int64_t tsmm_bulk_rows(int64_t n, int p, size_t esize) {
  const size_t bytes = static_cast<size_t>(p) * esize;
  size_t g = 16, b = bytes;
  while (b) {
    const size_t t = g % b;
    g = b;
    b = t;
  }
  const int64_t r0 = static_cast<int64_t>(16 / g);
  return n - n % r0;
}

// Splits the problems' streamed rows into chunks of `rows` rows.
template <typename T>
void set_chunks(TsmmArgs<T>& a, int rows) {
  int64_t total = 0;
  for (int i = 0; i < a.nprob; ++i) {
    TsmmProblem<T>& pr = a.prob[i];
    pr.rows_main = tsmm_bulk_rows(pr.n, pr.p, sizeof(T));
    pr.num_chunks = (pr.rows_main + rows - 1) / rows;
    if (i == 0) a.split = pr.num_chunks;
    total += pr.num_chunks;
  }
  if (a.nprob == 1) a.split = total;
  a.total_chunks = total;
}

int dmma_index(int dtype, int p, int q, bool ys) {
  const int P = std::max(4, cap_of(p)), Q = std::max(4, cap_of(q));
  for (int i = 0; i < kDmmaCount; ++i)
    if (kDmma[i].dtype == dtype && kDmma[i].P == P && kDmma[i].Q == Q && kDmma[i].ys == ys) return i;
  return -1;
}

// Y += X W can stage the old Y rows through the ring when Y is dense (ldy =
// q), 16-byte aligned and each row a multiple of 16 bytes.
template <typename T>
bool stages_y(const TsmmProblem<T>& pr) {
  return pr.beta && pr.ldy == pr.q && (pr.q * sizeof(T)) % 16 == 0 && aligned16(pr.Y);
}

// Bulk path on the FP64 tensor cores: one launch when both problems share
// capacities (the fused backward of square or same-capacity shapes), else
// one launch per problem.
template <typename T>
tsm_status launch_dmma(cudaStream_t stream, int dev, int sms, const TsmmProblem<T>* probs, int nprob,
                       unsigned* error) {
  constexpr int dtype = sizeof(T) == 8 ? 0 : 1;
  bool ys = true;  // every problem of the launch stages its old Y rows
  for (int i = 0; i < nprob; ++i) ys = ys && stages_y(probs[i]);
  int idx[2] = {dmma_index(dtype, probs[0].p, probs[0].q, ys),
                nprob > 1 ? dmma_index(dtype, probs[1].p, probs[1].q, ys) : -1};
  const bool together = nprob == 1 || idx[0] == idx[1];
  for (int l = 0; l < (together ? 1 : nprob); ++l) {
    const DmmaEntry& e = kDmma[idx[l]];
    {
      std::lock_guard<std::mutex> lk(g_tsmm_mu);
      if (!g_dmma_ready[dev][idx[l]]) {
        const cudaError_t ce =
            cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(e.smem));
        if (ce != cudaSuccess) return fail(ce, "cudaFuncSetAttribute(dmma)");
        // A grid larger than what is resident would run its extra CTAs as a
        // second wave: cap it at the measured occupancy.
        int occ = 0;
        const cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, e.fn, e.threads, e.smem);
        if (oe != cudaSuccess) return fail(oe, "cudaOccupancyMaxActiveBlocksPerMultiprocessor(dmma)");
        g_dmma_ctas[dev][idx[l]] = std::max(1, std::min(occ, kCtasPerSm));
        g_dmma_ready[dev][idx[l]] = 1;
      }
    }
    TsmmArgs<T> a{};
    a.error = error;
    if (together) {
      a.nprob = nprob;
      for (int i = 0; i < nprob; ++i) a.prob[i] = probs[i];
    } else {
      a.nprob = 1;
      a.prob[0] = probs[l];
    }
    set_chunks(a, e.rows);
    if (a.total_chunks == 0 && a.prob[0].n == 0 && (a.nprob < 2 || a.prob[1].n == 0)) continue;
    const int64_t grid =
        std::max<int64_t>(1, std::min<int64_t>(a.total_chunks, int64_t(sms) * g_dmma_ctas[dev][idx[l]]));
    void* args[] = {&a};
    const cudaError_t le =
        cudaLaunchKernel(e.fn, dim3(static_cast<unsigned>(grid)), dim3(e.threads), args, e.smem, stream);
    if (le != cudaSuccess) return fail(le, "cudaLaunchKernel(tsmm dmma)");
  }
  return TSM_SUCCESS;
}

template <typename T>
tsm_status launch_tsmm(cudaStream_t stream, TsmmProblem<T>* probs, int nprob, void* ws, size_t ws_bytes) {
  constexpr int dtype = sizeof(T) == 8 ? 0 : 1;
  if (ws == nullptr || ws_bytes < 256 || !aligned16(ws)) return TSM_ERROR_WORKSPACE;
  int cap = 1;
  bool bulk = true;
  for (int i = 0; i < nprob; ++i) {
    const TsmmProblem<T>& pr = probs[i];
    if (pr.n < 0 || pr.p < 1 || pr.q < 1 || pr.p > 64 || pr.q > 64) return TSM_ERROR_INVALID_VALUE;
    if (pr.ldx < pr.p || pr.ldy < pr.q || pr.W == nullptr) return TSM_ERROR_INVALID_VALUE;
    if (pr.n > 0 && (pr.X == nullptr || pr.Y == nullptr)) return TSM_ERROR_INVALID_VALUE;
    cap = std::max(cap, std::max(cap_of(pr.p), cap_of(pr.q)));
    if (pr.ldx != pr.p || !aligned16(pr.X)) bulk = false;
  }
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return fail(ce, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return TSM_ERROR_UNSUPPORTED;
  {
    std::lock_guard<std::mutex> lk(g_tsmm_mu);
    if (g_sms[dev] == 0) {
      ce = cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev);
      if (ce != cudaSuccess) return fail(ce, "cudaDeviceGetAttribute");
    }
  }
  const int sms = g_sms[dev];
  if (bulk) return launch_dmma<T>(stream, dev, sms, probs, nprob, reinterpret_cast<unsigned*>(ws) + 1);

  int idx = -1;
  for (int i = 0; i < kTsmmCount; ++i)
    if (kTsmm[i].dtype == dtype && kTsmm[i].cap == cap) idx = i;
  if (idx < 0) return TSM_ERROR_UNSUPPORTED;
  TsmmArgs<T> a{};
  a.nprob = nprob;
  a.error = reinterpret_cast<unsigned*>(ws) + 1;
  for (int i = 0; i < nprob; ++i) a.prob[i] = probs[i];
  int64_t nmax = 0;
  for (int i = 0; i < nprob; ++i) nmax = std::max(nmax, a.prob[i].n);
  const int rgn = cap >= 32 ? (8 / (cap / 32)) : 8 * (32 / cap);
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((nmax + rgn - 1) / rgn, int64_t(sms) * 8));
  void* args[] = {&a};
  const cudaError_t le = cudaLaunchKernel(kTsmm[idx].direct, dim3(static_cast<unsigned>(grid)), dim3(256), args, 0, stream);
  if (le != cudaSuccess) return fail(le, "cudaLaunchKernel(tsmm)");
  return TSM_SUCCESS;
}

template <typename T>
tsm_status tsmm_entry(tsm_stream_t stream, int64_t n, int p, int q, const T* X, int64_t ldx, const T* W,
                      int64_t w_row, int64_t w_col, T* Y, int64_t ldy, int beta, void* ws, size_t ws_bytes) {
  TsmmProblem<T> pr{};
  pr.X = X;
  pr.ldx = ldx;
  pr.W = W;
  pr.w_row = w_row;
  pr.w_col = w_col;
  pr.Y = Y;
  pr.ldy = ldy;
  pr.n = n;
  pr.p = p;
  pr.q = q;
  pr.beta = beta ? 1 : 0;
  return launch_tsmm<T>(static_cast<cudaStream_t>(stream), &pr, 1, ws, ws_bytes);
}

template <typename T>
tsm_status backward_entry(tsm_stream_t stream, int64_t n, int m, int k, const T* A, int64_t lda, const T* B,
                          int64_t ldb, const T* dC, int64_t lddc, T* dA, int64_t ldda, T* dB, int64_t lddb, int beta,
                          void* ws, size_t ws_bytes) {
  if (m < 1 || k < 1 || m > 64 || k > 64 || lddc < k || dC == nullptr) return TSM_ERROR_INVALID_VALUE;
  TsmmProblem<T> pr[2] = {};
  int np = 0;
  if (dA != nullptr) {  // dA (n x m) = B (n x k) * dC^T: W[a][b] = dC[b][a]
    TsmmProblem<T>& x = pr[np++];
    x.X = B;
    x.ldx = ldb;
    x.W = dC;
    x.w_row = 1;
    x.w_col = lddc;
    x.Y = dA;
    x.ldy = ldda;
    x.n = n;
    x.p = k;
    x.q = m;
    x.beta = beta ? 1 : 0;
  }
  if (dB != nullptr) {  // dB (n x k) = A (n x m) * dC
    TsmmProblem<T>& x = pr[np++];
    x.X = A;
    x.ldx = lda;
    x.W = dC;
    x.w_row = lddc;
    x.w_col = 1;
    x.Y = dB;
    x.ldy = lddb;
    x.n = n;
    x.p = m;
    x.q = k;
    x.beta = beta ? 1 : 0;
  }
  if (np == 0) return TSM_SUCCESS;
  return launch_tsmm<T>(static_cast<cudaStream_t>(stream), pr, np, ws, ws_bytes);
}

}  // namespace
}  // namespace tsm

using namespace tsm;

extern "C" {

tsm_status tsm_tsmm_f64(tsm_stream_t stream, int64_t n, int p, int q, const double* X, int64_t ldx, const double* W,
                        int64_t w_row, int64_t w_col, double* Y, int64_t ldy, int beta, void* workspace,
                        size_t workspace_bytes) {
  return tsmm_entry<double>(stream, n, p, q, X, ldx, W, w_row, w_col, Y, ldy, beta, workspace, workspace_bytes);
}

tsm_status tsm_tsmm_f32(tsm_stream_t stream, int64_t n, int p, int q, const float* X, int64_t ldx, const float* W,
                        int64_t w_row, int64_t w_col, float* Y, int64_t ldy, int beta, void* workspace,
                        size_t workspace_bytes) {
  return tsmm_entry<float>(stream, n, p, q, X, ldx, W, w_row, w_col, Y, ldy, beta, workspace, workspace_bytes);
}

tsm_status tsm_block_orth_f64(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda, double* B,
                             int64_t ldb, double* C, int64_t ldc, void* workspace, size_t workspace_bytes) {
  if (B == nullptr && n > 0) return TSM_ERROR_INVALID_VALUE;
  // 1. C = A^T B.
  tsm_status s = tsm_gemm_tn_f64(stream, n, m, k, A, lda, B, ldb, C, ldc, 0, workspace, workspace_bytes);
  if (s != TSM_SUCCESS) return s;
  // 2. B -= A C: TSMM with X = A (p = m), W = C (m x k, row-major, pitch ldc) read negated, Y = B, beta = 1;
  //    stream order makes step 1's C visible.
  TsmmProblem<double> pr{};
  pr.X = A;
  pr.ldx = lda;
  pr.W = C;
  pr.w_row = ldc;
  pr.w_col = 1;
  pr.Y = B;
  pr.ldy = ldb;
  pr.n = n;
  pr.p = m;
  pr.q = k;
  pr.beta = 1;
  pr.negate = 1;
  return launch_tsmm<double>(static_cast<cudaStream_t>(stream), &pr, 1, workspace, workspace_bytes);
}

tsm_status tsm_gemm_tn_backward_f64(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                                    const double* B, int64_t ldb, const double* dC, int64_t lddc, double* dA,
                                    int64_t ldda, double* dB, int64_t lddb, int beta, void* workspace,
                                    size_t workspace_bytes) {
  return backward_entry<double>(stream, n, m, k, A, lda, B, ldb, dC, lddc, dA, ldda, dB, lddb, beta, workspace,
                                workspace_bytes);
}

tsm_status tsm_gemm_tn_backward_f32(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                                    const float* B, int64_t ldb, const float* dC, int64_t lddc, float* dA,
                                    int64_t ldda, float* dB, int64_t lddb, int beta, void* workspace,
                                    size_t workspace_bytes) {
  return backward_entry<float>(stream, n, m, k, A, lda, B, ldb, dC, lddc, dA, ldda, dB, lddb, beta, workspace,
                               workspace_bytes);
}

}  // extern "C"
