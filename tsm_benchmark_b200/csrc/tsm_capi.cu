// tsm_capi.cu -- the C ABI (include/tsm.h): argument checks, variant choice,
// grid sizing and launches for the plain FP64 path.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/tsm.h"
#include "tsm_errors.h"
#include "tsm_registry.cuh"
#include "tsm_tmap.h"

namespace tsm {
namespace {
thread_local std::string g_last_cuda_error;
}  // namespace

std::string& last_error() { return g_last_cuda_error; }

namespace {

tsm_status cuda_fail(cudaError_t e, const char* what) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  g_last_cuda_error = buf;
  return TSM_ERROR_CUDA;
}

// Workspace layout: [counter u32][error u32][pad to 256 B][partials].
constexpr size_t kWsHeader = 256;
constexpr int kMaxCtasPerSm = 4;

struct DeviceState {
  int sms = 0;
  std::vector<signed char> attr_done;  // per variant: smem attribute set / failed
  std::vector<int> occupancy;          // per variant: CTAs per SM (0 = unknown)
};

std::mutex g_mu;
std::unordered_map<int, DeviceState> g_devices;

const std::vector<const Variant*>& variants() {
  static const std::vector<const Variant*> all = [] {
    std::vector<const Variant*> v;
    for (int p = 0; p < kVariantPartCount; ++p)
      for (int i = 0; i < kVariantParts[p].count; ++i) v.push_back(&kVariantParts[p].rows[i]);
    return v;
  }();
  return all;
}

tsm_status current_device(int* dev, DeviceState** st) {
  cudaError_t e = cudaGetDevice(dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState& s = g_devices[*dev];
  if (s.sms == 0) {
    e = cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, *dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    s.attr_done.assign(variants().size(), 0);
    s.occupancy.assign(variants().size(), 0);
  }
  *st = &s;
  return TSM_SUCCESS;
}

// Sets the dynamic shared-memory limit of a variant once per device and
// caches how many of its CTAs fit on one SM.
tsm_status prepare_variant(DeviceState* st, int idx) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (st->attr_done[idx] == 1) return TSM_SUCCESS;
  if (st->attr_done[idx] == -1) return TSM_ERROR_UNSUPPORTED;
  const Variant* v = variants()[idx];
  cudaError_t e = cudaFuncSetAttribute(v->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(v->smem));
  if (e != cudaSuccess) {
    st->attr_done[idx] = -1;
    return cuda_fail(e, "cudaFuncSetAttribute");
  }
  int occ = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v->kernel, v->threads, v->smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) {
    st->attr_done[idx] = -1;
    return TSM_ERROR_UNSUPPORTED;
  }
  st->occupancy[idx] = std::min(occ, kMaxCtasPerSm);
  st->attr_done[idx] = 1;
  return TSM_SUCCESS;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// C = A^T A: B is the same matrix as A (same data, pitch and width).
bool is_gram(int m, int k, const void* A, int64_t lda, const void* B, int64_t ldb) {
  return A == B && lda == ldb && m == k;
}

bool applicable(const Variant* v, int dtype, int64_t n, int m, int k, const void* A, int64_t lda, const void* B,
                int64_t ldb) {
  if (v->dtype != dtype) return false;
  if (v->gram && !is_gram(m, k, A, lda, B, ldb)) return false;
  if (v->exact ? (m != v->wa || k != v->wb) : (m > v->wa || k > v->wb)) return false;
  if (v->kind == kKindBulk) {
    if (lda != m || ldb != k) return false;
    if (!aligned16(A) || !aligned16(B)) return false;
  }
  if (v->kind == kKindDmma) {
    // Tensor maps: 16-byte aligned bases and row pitches, 32-bit row
    // coordinates.
    if ((lda * 8) % 16 != 0 || (ldb * 8) % 16 != 0) return false;
    if (!aligned16(A) || !aligned16(B)) return false;
    if (n > static_cast<int64_t>(INT_MAX) - v->rows) return false;
  }
  return true;
}

// Tensor map of a row-major FP64 operand (rows x width, pitch ld elements)
// with boxes of 16 columns x `box_rows` rows and the 128-byte swizzle the
// DMMA kernels read with.
tsm_status encode_operand_map(CUtensorMap* map, const double* base, int64_t rows, int width, int64_t ld,
                              int box_rows) {
  if (!encode_rowmajor_map(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, base, rows, width, ld, 16, box_rows,
                           CU_TENSOR_MAP_SWIZZLE_128B, &g_last_cuda_error))
    return TSM_ERROR_CUDA;
  return TSM_SUCCESS;
}

// Generated: preferred variant per (m, k, n) from the tuning table.
}  // namespace

extern const char* const kTunedDefaults[];  // "m k nmin name", null-terminated
extern const int kTunedDefaultCount;
extern const char* const kTunedGram[];  // "w nmin name": Gram variants, null-terminated
extern const int kTunedGramCount;

namespace {

int find_variant(const char* name) {
  const auto& vs = variants();
  for (size_t i = 0; i < vs.size(); ++i)
    if (std::strcmp(vs[i]->name, name) == 0) return static_cast<int>(i);
  return -1;
}

int default_variant(int dtype, int64_t n, int m, int k, const void* A, int64_t lda, const void* B, int64_t ldb) {
  const auto& vs = variants();
  // 0. C = A^T A: a Gram variant (A streamed once): the tuned entry with the
  //    largest nmin <= n for width m, else the first in table order.
  if (is_gram(m, k, A, lda, B, ldb)) {
    int best = -1;
    long long best_nmin = -1;
    for (int i = 0; i < kTunedGramCount; ++i) {
      int tw = 0;
      long long nmin = 0;
      char name[96] = {0};
      if (std::sscanf(kTunedGram[i], "%d %lld %95s", &tw, &nmin, name) != 3) continue;
      if (tw != m || nmin > n || nmin < best_nmin) continue;
      const int idx = find_variant(name);
      if (idx >= 0 && vs[idx]->gram && applicable(vs[idx], dtype, n, m, k, A, lda, B, ldb)) {
        best = idx;
        best_nmin = nmin;
      }
    }
    if (best >= 0) return best;
    for (size_t i = 0; i < vs.size(); ++i)
      if (vs[i]->gram && applicable(vs[i], dtype, n, m, k, A, lda, B, ldb)) return static_cast<int>(i);
  }
  // 1. The tuning table: the entry with the largest nmin <= n for (m, k).
  int best = -1;
  long long best_nmin = -1;
  for (int i = 0; i < kTunedDefaultCount; ++i) {
    int tm = 0, tk = 0;
    long long nmin = 0;
    char name[96] = {0};
    if (std::sscanf(kTunedDefaults[i], "%d %d %lld %95s", &tm, &tk, &nmin, name) != 4) continue;
    if (tm != m || tk != k || nmin > n || nmin < best_nmin) continue;
    const int idx = find_variant(name);
    if (idx >= 0 && applicable(vs[idx], dtype, n, m, k, A, lda, B, ldb)) {
      best = idx;
      best_nmin = nmin;
    }
  }
  if (best >= 0) return best;
  // 2. Table order: the generator lists exact bulk variants first, then
  //    capacity bulk variants from the smallest capacity up, then direct ones.
  for (size_t i = 0; i < vs.size(); ++i)
    if (applicable(vs[i], dtype, n, m, k, A, lda, B, ldb)) return static_cast<int>(i);
  return -1;
}

// Rows the bulk kernels stream: every copy of rows * width elements must be a
// multiple of 16 bytes, so up to three final rows may be left to the epilogue.
int64_t bulk_rows(int64_t n, int m, int k, size_t esize) {
  auto need = [esize](int w) {
    const size_t bytes = static_cast<size_t>(w) * esize;
    size_t g = 16;
    size_t b = bytes;
    while (b) {
      const size_t t = g % b;
      g = b;
      b = t;
    }
    return static_cast<int64_t>(16 / g);
  };
  const int64_t ra = need(m), rb = need(k);
  const int64_t r0 = ra > rb ? ra : rb;  // both are powers of two
  return n - n % r0;
}

tsm_status check_args(int64_t n, int m, int k, const void* A, int64_t lda, const void* B, int64_t ldb,
                      const void* C, int64_t ldc) {
  if (n < 0 || m < 1 || k < 1 || m > 64 || k > 64) return TSM_ERROR_INVALID_VALUE;
  if (lda < m || ldb < k || ldc < k) return TSM_ERROR_INVALID_VALUE;
  if (C == nullptr) return TSM_ERROR_INVALID_VALUE;
  if (n > 0 && (A == nullptr || B == nullptr)) return TSM_ERROR_INVALID_VALUE;
  return TSM_SUCCESS;
}

size_t workspace_bytes_for(int sms, int m, int k) {
  return kWsHeader + static_cast<size_t>(sms) * kMaxCtasPerSm * m * k * sizeof(double);
}

// Rows the main loop streams, chunk count and grid for variant v (p.n, p.m,
// p.k set).  Bulk: 16-byte copies leave up to three final rows of an
// odd-width operand to the reduction epilogue.  DMMA: the tensor maps
// zero-fill past row n, so every row is streamed.
template <typename T>
int64_t plan_grid(const Variant* v, const DeviceState* st, int idx, PlainArgs<T>& p) {
  const int64_t max_grid = static_cast<int64_t>(st->sms) * st->occupancy[idx];
  if (v->kind == kKindBulk || v->kind == kKindDmma) {
    p.rows_main = v->kind == kKindBulk ? bulk_rows(p.n, p.m, p.k, sizeof(T)) : p.n;
    p.num_chunks = (p.rows_main + v->rows - 1) / v->rows;
    return std::max<int64_t>(1, std::min<int64_t>(p.num_chunks, max_grid));
  }
  p.rows_main = p.n;
  p.num_chunks = 0;
  const int tiles = (v->wa / v->ta) * (v->wb / v->tb);
  const int64_t row_groups = v->threads / tiles;
  return std::max<int64_t>(1, std::min<int64_t>((p.n + row_groups - 1) / row_groups, max_grid));
}

template <typename T>
tsm_status launch_variant(const Variant* v, const PlainArgs<T>& p, int64_t grid, cudaStream_t stream) {
  cudaError_t e;
  if (v->kind == kKindDmma) {
    if constexpr (sizeof(T) == 8) {
      DmmaArgs d{};
      d.p = p;
      d.p.symmetric = is_gram(p.m, p.k, p.A, p.lda, p.B, p.ldb) ? 1 : 0;
      if (p.n > 0) {  // n = 0: no chunks, the maps are never read
        const int box_rows = dmma_box_rows(v->rows);
        tsm_status s = encode_operand_map(&d.ta, p.A, p.n, p.m, p.lda, box_rows);
        if (s == TSM_SUCCESS && !v->gram) s = encode_operand_map(&d.tb, p.B, p.n, p.k, p.ldb, box_rows);
        if (s != TSM_SUCCESS) return s;
      }
      void* args[] = {&d};
      e = cudaLaunchKernel(v->kernel, dim3(static_cast<unsigned>(grid)), dim3(v->threads), args, v->smem, stream);
    } else {
      return TSM_ERROR_UNSUPPORTED;
    }
  } else {
    PlainArgs<T> q = p;
    q.symmetric = is_gram(p.m, p.k, p.A, p.lda, p.B, p.ldb) ? 1 : 0;  // C = A^T A: written exactly symmetric
    void* args[] = {&q};
    e = cudaLaunchKernel(v->kernel, dim3(static_cast<unsigned>(grid)), dim3(v->threads), args, v->smem, stream);
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaLaunchKernel");
  return TSM_SUCCESS;
}

template <typename T>
tsm_status launch_plain(cudaStream_t stream, int64_t n, int m, int k, const T* A, int64_t lda, const T* B,
                        int64_t ldb, T* C, int64_t ldc, int accumulate, void* ws, size_t ws_bytes, int variant,
                        int64_t max_ctas = 0) {
  constexpr int dtype = DTypeOf<T>::value;
  tsm_status s = check_args(n, m, k, A, lda, B, ldb, C, ldc);
  if (s != TSM_SUCCESS) return s;
  int dev = 0;
  DeviceState* st = nullptr;
  if ((s = current_device(&dev, &st)) != TSM_SUCCESS) return s;
  if (ws == nullptr || ws_bytes < workspace_bytes_for(st->sms, m, k) || !aligned16(ws))
    return TSM_ERROR_WORKSPACE;

  const auto& vs = variants();
  int idx = variant;
  if (idx < 0) {
    idx = default_variant(dtype, n, m, k, A, lda, B, ldb);
    if (idx < 0) return TSM_ERROR_UNSUPPORTED;
  } else if (idx >= static_cast<int>(vs.size()) || !applicable(vs[idx], dtype, n, m, k, A, lda, B, ldb)) {
    return TSM_ERROR_UNSUPPORTED;
  }
  if ((s = prepare_variant(st, idx)) != TSM_SUCCESS) return s;
  const Variant* v = vs[idx];

  PlainArgs<T> p{};
  p.A = A;
  p.B = B;
  p.C = C;
  p.n = n;
  p.m = m;
  p.k = k;
  p.lda = lda;
  p.ldb = ldb;
  p.ldc = ldc;
  p.accumulate = accumulate ? 1 : 0;
  unsigned char* base = static_cast<unsigned char*>(ws);
  p.counter = reinterpret_cast<unsigned*>(base);
  p.error = reinterpret_cast<unsigned*>(base) + 1;
  p.partials = reinterpret_cast<double*>(base + kWsHeader);

  int64_t grid = plan_grid(v, st, idx, p);
  if (max_ctas > 0) grid = std::min(grid, max_ctas);  // every kernel deals its rows over any grid >= 1
  return launch_variant(v, p, grid, stream);
}

// ------------------------------------------------------- timeout self-test
// One thread waits on an mbarrier that nothing ever arrives on, through the
// same bounded wait every pipeline uses, then records the timeout in the
// workspace's error word -- the failure path of the kernels, exercised on
// purpose (a wait that runs out; no fault, no trap).
__global__ void selftest_wait_kernel(unsigned* error, uint64_t limit_ns) {
  __shared__ uint64_t bar;
  __shared__ int abort;
  if (threadIdx.x == 0) {
    dev::mbar_init(&bar, 1);
    abort = 0;
    dev::fence_mbar_init();
    if (!dev::mbar_wait_for(&bar, 0, &abort, limit_ns)) atomicOr(error, dev::kErrTimeout);
  }
}

// ----------------------------------------------------------------- fills
__global__ void fill_uniform_kernel(double* x, int64_t count, uint64_t seed, uint64_t stream_id) {
  const int64_t step = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += step) {
    uint64_t z = seed + ((stream_id << 40) + static_cast<uint64_t>(i) + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = static_cast<double>(z >> 11) * 0x1.0p-53;
    x[i] = 2.0 * u - 1.0;
  }
}

}  // namespace
}  // namespace tsm

using namespace tsm;

extern "C" {

int tsm_version(void) { return 100; }

const char* tsm_status_string(tsm_status s) {
  switch (s) {
    case TSM_SUCCESS: return "success";
    case TSM_ERROR_INVALID_VALUE: return "invalid value (shape, pointer or leading dimension)";
    case TSM_ERROR_WORKSPACE: return "workspace missing, unaligned or too small";
    case TSM_ERROR_CUDA: return "CUDA runtime error";
    case TSM_ERROR_UNSUPPORTED: return "no compiled variant supports this request";
    case TSM_ERROR_DEVICE_TIMEOUT: return "a kernel gave up a bounded wait";
  }
  return "unknown status";
}

const char* tsm_last_cuda_error(void) { return g_last_cuda_error.c_str(); }

size_t tsm_gemm_tn_workspace_size(int64_t n, int m, int k) {
  (void)n;
  if (m < 1 || k < 1 || m > 64 || k > 64) return 0;
  int dev = 0;
  DeviceState* st = nullptr;
  if (current_device(&dev, &st) != TSM_SUCCESS) return 0;
  return workspace_bytes_for(st->sms, m, k);
}

tsm_status tsm_gemm_tn_f64(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                           const double* B, int64_t ldb, double* C, int64_t ldc, int accumulate, void* workspace,
                           size_t workspace_bytes) {
  return launch_plain<double>(static_cast<cudaStream_t>(stream), n, m, k, A, lda, B, ldb, C, ldc, accumulate,
                              workspace, workspace_bytes, -1);
}

tsm_status tsm_gram_f64(tsm_stream_t stream, int64_t n, int m, const double* A, int64_t lda, double* C, int64_t ldc,
                        int accumulate, void* workspace, size_t workspace_bytes) {
  return launch_plain<double>(static_cast<cudaStream_t>(stream), n, m, m, A, lda, A, lda, C, ldc, accumulate,
                              workspace, workspace_bytes, -1);
}

tsm_status tsm_gemm_tn_f64_variant(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                                   const double* B, int64_t ldb, double* C, int64_t ldc, int accumulate,
                                   void* workspace, size_t workspace_bytes, int variant) {
  return launch_plain<double>(static_cast<cudaStream_t>(stream), n, m, k, A, lda, B, ldb, C, ldc, accumulate,
                              workspace, workspace_bytes, variant);
}

tsm_status tsm_gemm_tn_f64_launch(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                                  const double* B, int64_t ldb, double* C, int64_t ldc, int accumulate,
                                  void* workspace, size_t workspace_bytes, int variant, int64_t max_ctas) {
  return launch_plain<double>(static_cast<cudaStream_t>(stream), n, m, k, A, lda, B, ldb, C, ldc, accumulate,
                              workspace, workspace_bytes, variant, max_ctas);
}

tsm_status tsm_gemm_tn_f32(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                           const float* B, int64_t ldb, float* C, int64_t ldc, int accumulate, void* workspace,
                           size_t workspace_bytes) {
  return launch_plain<float>(static_cast<cudaStream_t>(stream), n, m, k, A, lda, B, ldb, C, ldc, accumulate,
                             workspace, workspace_bytes, -1);
}

tsm_status tsm_gemm_tn_f32_variant(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                                   const float* B, int64_t ldb, float* C, int64_t ldc, int accumulate,
                                   void* workspace, size_t workspace_bytes, int variant) {
  return launch_plain<float>(static_cast<cudaStream_t>(stream), n, m, k, A, lda, B, ldb, C, ldc, accumulate,
                             workspace, workspace_bytes, variant);
}

int tsm_gemm_tn_default_variant(int dtype, int64_t n, int m, int k, const void* A, int64_t lda, const void* B,
                                int64_t ldb) {
  if (dtype != kF64 && dtype != kF32) return -1;
  if (check_args(n, m, k, A, lda, B, ldb, A ? A : B, k) != TSM_SUCCESS) return -1;
  return default_variant(dtype, n, m, k, A, lda, B, ldb);
}

int tsm_variant_count(void) { return static_cast<int>(variants().size()); }

tsm_status tsm_variant_get_info(int index, tsm_variant_info* info) {
  if (index < 0 || index >= tsm_variant_count() || info == nullptr) return TSM_ERROR_INVALID_VALUE;
  const Variant* v = variants()[index];
  std::memset(info, 0, sizeof(*info));
  std::strncpy(info->name, v->name, sizeof(info->name) - 1);
  info->kind = v->kind;
  info->dtype = v->dtype;
  info->wa = v->wa;
  info->wb = v->wb;
  info->ta = v->ta;
  info->tb = v->tb;
  info->exact = v->exact;
  info->threads = v->threads;
  info->stages = v->stages;
  info->rows = v->rows;
  info->unroll = v->unroll;
  info->smem_bytes = v->smem;
  info->gram = v->gram;
  return TSM_SUCCESS;
}

tsm_status tsm_selftest_wait_timeout(tsm_stream_t stream, void* workspace, size_t workspace_bytes,
                                     unsigned limit_us) {
  if (workspace == nullptr || workspace_bytes < kWsHeader || !aligned16(workspace)) return TSM_ERROR_WORKSPACE;
  if (limit_us == 0 || limit_us > 2000000u) return TSM_ERROR_INVALID_VALUE;
  unsigned* error = reinterpret_cast<unsigned*>(workspace) + 1;
  selftest_wait_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(error, uint64_t(limit_us) * 1000u);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "selftest_wait_kernel");
  return TSM_SUCCESS;
}

tsm_status tsm_workspace_check(tsm_stream_t stream, void* workspace, unsigned* bits) {
  if (workspace == nullptr) return TSM_ERROR_WORKSPACE;
  unsigned host = 0;
  unsigned* err = static_cast<unsigned*>(workspace) + 1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(&host, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(unsigned), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "tsm_workspace_check");
  if (bits) *bits = host;
  return host ? TSM_ERROR_DEVICE_TIMEOUT : TSM_SUCCESS;
}

tsm_status tsm_fill_uniform_f64(tsm_stream_t stream, double* x, int64_t count, uint64_t seed, uint64_t stream_id) {
  if (count < 0 || (count > 0 && x == nullptr)) return TSM_ERROR_INVALID_VALUE;
  if (count == 0) return TSM_SUCCESS;
  int dev = 0;
  DeviceState* st = nullptr;
  tsm_status s = current_device(&dev, &st);
  if (s != TSM_SUCCESS) return s;
  const int64_t blocks = std::min<int64_t>((count + 255) / 256, static_cast<int64_t>(st->sms) * 16);
  fill_uniform_kernel<<<static_cast<unsigned>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, count, seed,
                                                                                                    stream_id);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fill_uniform_kernel");
  return TSM_SUCCESS;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point: tsm_gemm_tn_f64_noalloc.
//
// Some callers cannot hand the library a workspace.  A plugin loaded into a
// host program that owns every device allocation (its own pool, no
// cudaMalloc from plug-ins), or a latency-bound loop where a cudaMalloc --
// which may synchronise the whole device -- is not allowed after start-up,
// can still call this.  The scratch the kernels need (a launch counter, an
// error word and one m x k partial per CTA) lives in the file-scope array
// below instead, which every GPU that loads this library holds until the
// process exits.
//
// Limits and sharing:
//   * kStaticScratchBytes (4 MiB) bounds a call: 256 B of header plus
//     (CTAs launched) * m * k * 8 B of partials.  A request that would need
//     more returns TSM_ERROR_WORKSPACE and runs nothing.
//   * All calls on a device share the one array and it keeps whatever the
//     last call left.  The launch counter must start at zero, so each call
//     zeroes it (stream-ordered) before its launch.  Calls that overlap on
//     the GPU (different streams, other threads) race on the array and give
//     wrong results: serialise them.
//   * The first call on each device looks the array's device address up
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture.  Like every per-device state of the
//     library, that address does not survive cudaDeviceReset: do not reset a
//     device while the library is in use on it.
//   * A kernel that gives up a bounded wait sets a bit in the array's error
//     word; tsm_noalloc_check reads and clears it.
// ---------------------------------------------------------------------------
namespace tsm {
namespace {
constexpr size_t kStaticScratchBytes = size_t(4) << 20;
constexpr int kStaticScratchDevices = 64;
}  // namespace
}  // namespace tsm

static __device__ __align__(256) unsigned char tsm_static_scratch[tsm::kStaticScratchBytes];

namespace tsm {
namespace {

std::mutex g_static_mu;
void* g_static_ptr[kStaticScratchDevices] = {};

// Device address of tsm_static_scratch on device `dev` (current), looked up
// once per device.  In host code the array's name is only a host-side
// stand-in, never a device address.
tsm_status static_scratch(int dev, void** out) {
  if (dev < 0 || dev >= kStaticScratchDevices) return TSM_ERROR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (g_static_ptr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, tsm_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(tsm_static_scratch)");
    g_static_ptr[dev] = p;
  }
  *out = g_static_ptr[dev];
  return TSM_SUCCESS;
}

}  // namespace
}  // namespace tsm

extern "C" tsm_status tsm_gemm_tn_f64_noalloc(tsm_stream_t stream, int64_t n, int m, int k, const double* A,
                                              int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc,
                                              int accumulate) {
  using namespace tsm;
  tsm_status s = check_args(n, m, k, A, lda, B, ldb, C, ldc);
  if (s != TSM_SUCCESS) return s;
  int dev = 0;
  DeviceState* st = nullptr;
  if ((s = current_device(&dev, &st)) != TSM_SUCCESS) return s;
  void* scratch = nullptr;
  if ((s = static_scratch(dev, &scratch)) != TSM_SUCCESS) return s;

  // Same variant and grid as tsm_gemm_tn_f64 would use.
  const int idx = default_variant(kF64, n, m, k, A, lda, B, ldb);
  if (idx < 0) return TSM_ERROR_UNSUPPORTED;
  if ((s = prepare_variant(st, idx)) != TSM_SUCCESS) return s;
  const Variant* v = variants()[idx];

  PlainArgs<double> p{};
  p.A = A;
  p.B = B;
  p.C = C;
  p.n = n;
  p.m = m;
  p.k = k;
  p.lda = lda;
  p.ldb = ldb;
  p.ldc = ldc;
  p.accumulate = accumulate ? 1 : 0;
  const int64_t grid = plan_grid(v, st, idx, p);
  const size_t need = kWsHeader + static_cast<size_t>(grid) * m * k * sizeof(double);
  if (need > kStaticScratchBytes) return TSM_ERROR_WORKSPACE;

  unsigned char* base = static_cast<unsigned char*>(scratch);
  p.counter = reinterpret_cast<unsigned*>(base);
  p.error = reinterpret_cast<unsigned*>(base) + 1;
  p.partials = reinterpret_cast<double*>(base + kWsHeader);

  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(p.counter, 0, sizeof(unsigned), cs);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(static scratch counter)");
  return launch_variant(v, p, grid, cs);
}

// Reads and clears the error word of the static scratch: the counterpart of
// tsm_workspace_check for tsm_gemm_tn_f64_noalloc, whose kernels record a
// bounded wait that ran out there instead of in a caller's workspace.  The
// word is sticky across calls until read.  Allocates nothing.
extern "C" tsm_status tsm_noalloc_check(tsm_stream_t stream, unsigned* bits) {
  using namespace tsm;
  int dev = 0;
  DeviceState* st = nullptr;
  tsm_status s = current_device(&dev, &st);
  if (s != TSM_SUCCESS) return s;
  void* scratch = nullptr;
  if ((s = static_scratch(dev, &scratch)) != TSM_SUCCESS) return s;
  return tsm_workspace_check(stream, scratch, bits);
}
