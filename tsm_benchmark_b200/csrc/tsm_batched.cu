// tsm_batched.cu -- C ABI of the batched form: a plan (schedule of row
// segments per CTA, built once on the host and copied to caller-owned device
// memory) and a single-launch execution that a CUDA graph can capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tsm.h"
#include "tsm_errors.h"
#include "tsm_batched.cuh"
#include "tsm_tmap.h"

namespace tsm {
namespace {

constexpr size_t kAlign = 256;
constexpr uint32_t kMagic = 0x54534d42u;  // "TSMB"

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

struct Layout {
  size_t problems, maps, segments, cta_first, counters, partials, total;
};

Layout layout(int count, int nseg, int grid, size_t partial_doubles) {
  Layout l{};
  size_t off = kAlign;  // header: magic, error word
  l.problems = off;
  off = align_up(off + sizeof(BatchedProblemDev) * count);
  l.maps = off;  // 2 tensor maps per problem (64-byte aligned: kAlign is 256)
  off = align_up(off + sizeof(CUtensorMap) * 2 * count);
  l.segments = off;
  off = align_up(off + sizeof(BatchedSegmentDev) * nseg);
  l.cta_first = off;
  off = align_up(off + sizeof(int) * (grid + 1));
  l.counters = off;
  off = align_up(off + sizeof(unsigned) * count);
  l.partials = off;
  off = align_up(off + sizeof(double) * partial_doubles);
  l.total = off;
  return l;
}

struct Schedule {
  std::vector<BatchedProblemDev> problems;
  std::vector<BatchedSegmentDev> segments;
  std::vector<int> cta_first;
  size_t partial_doubles = 0;
  int grid = 0;
};


tsm_status fail(cudaError_t e, const char* what) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  last_error() = buf;
  return TSM_ERROR_CUDA;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

// Autotuned consumer path per width class: "m k path" lines written by the
// generator from tuned.json (csrc/generated/variants_index.cu).
extern const char* const kTunedBatchedPaths[];
extern const int kTunedBatchedPathCount;

namespace {

// The consumer path of class (m, k): the caller's override when given
// (class_paths[class] >= 0), else the tuned table's, else the default.
int class_path(int m, int k, const int* class_paths) {
  const int cls = batched::class_of(m, k);
  int path = batched::kPathDefault;
  if (class_paths != nullptr && class_paths[cls] >= 0) {
    path = class_paths[cls];
  } else {
    for (int i = 0; i < kTunedBatchedPathCount; ++i) {
      int tm = 0, tk = 0, tp = 0;
      if (std::sscanf(kTunedBatchedPaths[i], "%d %d %d", &tm, &tk, &tp) == 3 && tm == m && tk == k) path = tp;
    }
  }
  // The SIMT path is the default of the classes below the tensor cores.
  return batched::dmma_class(m, k) ? path : batched::kPathDefault;
}

// Cuts the concatenated rows of all problems into one contiguous byte range
// per CTA (one CTA per SM): CTA b gets bytes [b T / G, (b + 1) T / G).
tsm_status build_schedule(int count, const tsm_batched_problem_f64* in, int sms, Schedule* out,
                          const int* class_paths = nullptr) {
  if (count < 1 || in == nullptr) return TSM_ERROR_INVALID_VALUE;
  if (class_paths != nullptr)
    for (int c = 0; c < 16; ++c)
      if (class_paths[c] < -1 || class_paths[c] > batched::kPathSimt) return TSM_ERROR_INVALID_VALUE;
  Schedule s;
  s.grid = sms;
  s.problems.resize(count);
  double total = 0;
  for (int p = 0; p < count; ++p) {
    const tsm_batched_problem_f64& q = in[p];
    if (q.n < 0 || q.C == nullptr || q.ldc < q.k) return TSM_ERROR_INVALID_VALUE;
    if (q.n > 0 && (q.A == nullptr || q.B == nullptr)) return TSM_ERROR_INVALID_VALUE;
    const int cls = batched::class_of(q.m, q.k);
    if (cls < 0) return TSM_ERROR_UNSUPPORTED;  // widths outside {4, 8, 16, 32}
    if (q.n > 0 && (!aligned16(q.A) || !aligned16(q.B))) return TSM_ERROR_UNSUPPORTED;
    const int path = class_path(q.m, q.k, class_paths);
    // The tensor-core path addresses rows with 32-bit tensor-map coordinates.
    if (batched::uses_dmma(q.m, q.k, path) && q.n > static_cast<int64_t>(INT_MAX) - 256) return TSM_ERROR_UNSUPPORTED;
    BatchedProblemDev& d = s.problems[p];
    d.path = path;
    d.A = q.A;
    d.B = q.B;
    d.C = q.C;
    d.n = q.n;
    d.m = q.m;
    d.k = q.k;
    d.cls = cls;
    d.accumulate = q.accumulate ? 1 : 0;
    d.ldc = q.ldc;
    total += 8.0 * q.n * (q.m + q.k);
  }
  const double per = total > 0 ? total / sms : 1.0;
  int cta = 0;
  double used = 0;
  for (int p = 0; p < count; ++p) {
    BatchedProblemDev& d = s.problems[p];
    d.seg_first = static_cast<int64_t>(s.segments.size());
    const double row_bytes = 8.0 * (d.m + d.k);
    int64_t row = 0;
    do {
      if (cta < sms - 1 && used > 0 && used + row_bytes > per * 1.0000001) {
        ++cta;
        used = 0;
      }
      int64_t take = d.n - row;
      if (cta < sms - 1) {
        const int64_t fit = static_cast<int64_t>((per - used) / row_bytes);
        take = std::max<int64_t>(std::min<int64_t>(take, fit), d.n > 0 ? 1 : 0);
      }
      BatchedSegmentDev seg{};
      seg.problem = p;
      seg.r0 = row;
      seg.r1 = row + take;
      seg.pad = cta;  // owner, used below to build cta_first
      s.segments.push_back(seg);
      row += take;
      used += take * row_bytes;
    } while (row < d.n);
    d.nseg = static_cast<int>(s.segments.size() - d.seg_first);
  }
  s.cta_first.assign(sms + 1, static_cast<int>(s.segments.size()));
  for (int i = static_cast<int>(s.segments.size()) - 1; i >= 0; --i) {
    const int owner = s.segments[i].pad;
    for (int b = owner; b >= 0 && s.cta_first[b] > i; --b) s.cta_first[b] = i;
  }
  size_t off = 0;
  for (auto& seg : s.segments) {
    seg.partial_off = static_cast<int64_t>(off);
    off += static_cast<size_t>(s.problems[seg.problem].m) * s.problems[seg.problem].k;
    seg.pad = 0;
  }
  s.partial_doubles = off;
  *out = std::move(s);
  return TSM_SUCCESS;
}

std::mutex g_mu;
int g_sms[64] = {};
bool g_attr[64] = {};

tsm_status device_sms(int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return TSM_ERROR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_sms[dev] == 0) {
    e = cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(e, "cudaDeviceGetAttribute");
  }
  if (!g_attr[dev]) {
    for (const void* fn : {reinterpret_cast<const void*>(&tsm_tn_batched_kernel<false>),
                           reinterpret_cast<const void*>(&tsm_tn_batched_kernel<true>)}) {
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(batched::kSmemBytes));
      if (e != cudaSuccess) return fail(e, "cudaFuncSetAttribute(batched)");
    }
    g_attr[dev] = true;
  }
  *sms = g_sms[dev];
  return TSM_SUCCESS;
}

}  // namespace
}  // namespace tsm

using namespace tsm;

extern "C" {

size_t tsm_batched_plan_size_f64(int count, const tsm_batched_problem_f64* problems) {
  int sms = 0;
  if (device_sms(&sms) != TSM_SUCCESS) return 0;
  Schedule s;
  if (build_schedule(count, problems, sms, &s) != TSM_SUCCESS) return 0;
  return layout(count, static_cast<int>(s.segments.size()), s.grid, s.partial_doubles).total;
}

tsm_status tsm_batched_plan_init_paths_f64(tsm_stream_t stream, int count, const tsm_batched_problem_f64* problems,
                                           const int* class_paths, void* device_buffer, size_t device_bytes,
                                           tsm_batched_plan* plan) {
  if (plan == nullptr || device_buffer == nullptr || !aligned16(device_buffer)) return TSM_ERROR_INVALID_VALUE;
  if (count < 1 || problems == nullptr) return TSM_ERROR_INVALID_VALUE;
  if (class_paths != nullptr)  // checked before any CUDA call
    for (int c = 0; c < 16; ++c)
      if (class_paths[c] < -1 || class_paths[c] > batched::kPathSimt) return TSM_ERROR_INVALID_VALUE;
  int sms = 0;
  tsm_status st = device_sms(&sms);
  if (st != TSM_SUCCESS) return st;
  Schedule s;
  if ((st = build_schedule(count, problems, sms, &s, class_paths)) != TSM_SUCCESS) return st;
  const int nseg = static_cast<int>(s.segments.size());
  const Layout l = layout(count, nseg, s.grid, s.partial_doubles);
  if (device_bytes < l.total) return TSM_ERROR_WORKSPACE;
  // Everything up to the partials: header (magic, zero error word), tables,
  // zero counters.
  std::vector<unsigned char> img(l.partials, 0);
  std::memcpy(img.data(), &kMagic, sizeof(kMagic));
  std::memcpy(img.data() + l.problems, s.problems.data(), sizeof(BatchedProblemDev) * count);
  std::memcpy(img.data() + l.segments, s.segments.data(), sizeof(BatchedSegmentDev) * nseg);
  std::memcpy(img.data() + l.cta_first, s.cta_first.data(), sizeof(int) * (s.grid + 1));
  // Tensor maps of the problems on the tensor-core path: 16-column x rows-row
  // boxes with the 128-byte swizzle the kernel reads with.
  // (Encoded into an aligned local, then copied: the image's bytes carry no
  // 64-byte alignment on the host.)
  for (int p = 0; p < count; ++p) {
    const BatchedProblemDev& d = s.problems[p];
    if (!batched::uses_dmma(d.m, d.k, d.path) || d.n == 0) continue;
    const int rs = batched::rows_of(d.m, d.k, d.path);
    CUtensorMap mp[2];
    if (!encode_rowmajor_map(&mp[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, d.A, d.n, d.m, d.m, 16, rs,
                             CU_TENSOR_MAP_SWIZZLE_128B, &last_error()) ||
        !encode_rowmajor_map(&mp[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, d.B, d.n, d.k, d.k, 16, rs,
                             CU_TENSOR_MAP_SWIZZLE_128B, &last_error()))
      return TSM_ERROR_CUDA;
    std::memcpy(img.data() + l.maps + sizeof(CUtensorMap) * 2 * p, mp, sizeof(mp));
  }
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(device_buffer, img.data(), img.size(), cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
  if (e != cudaSuccess) return fail(e, "tsm_batched_plan_init_f64");
  std::memset(plan, 0, sizeof(*plan));
  plan->device = device_buffer;
  plan->bytes = l.total;
  plan->count = count;
  plan->segments = nseg;
  plan->grid = s.grid;
  plan->flags = 0;
  for (const BatchedProblemDev& d : s.problems)
    if (batched::dmma_class(d.m, d.k) && d.path == batched::kPathSimt) plan->flags = 1;
  return TSM_SUCCESS;
}

tsm_status tsm_batched_plan_init_f64(tsm_stream_t stream, int count, const tsm_batched_problem_f64* problems,
                                     void* device_buffer, size_t device_bytes, tsm_batched_plan* plan) {
  return tsm_batched_plan_init_paths_f64(stream, count, problems, nullptr, device_buffer, device_bytes, plan);
}

tsm_status tsm_gemm_tn_batched_f64(tsm_stream_t stream, const tsm_batched_plan* plan) {
  if (plan == nullptr || plan->device == nullptr || plan->count < 1 || plan->grid < 1) return TSM_ERROR_INVALID_VALUE;
  int sms = 0;
  tsm_status st = device_sms(&sms);
  if (st != TSM_SUCCESS) return st;
  // The partial area size only matters for the layout's total, which the
  // offsets below do not depend on.
  const Layout l = layout(plan->count, plan->segments, plan->grid, 0);
  unsigned char* base = static_cast<unsigned char*>(plan->device);
  BatchedArgs a{};
  a.problems = reinterpret_cast<const BatchedProblemDev*>(base + l.problems);
  a.maps = reinterpret_cast<const CUtensorMap*>(base + l.maps);
  a.segments = reinterpret_cast<const BatchedSegmentDev*>(base + l.segments);
  a.cta_first = reinterpret_cast<const int*>(base + l.cta_first);
  a.counters = reinterpret_cast<unsigned*>(base + l.counters);
  a.partials = reinterpret_cast<double*>(base + l.partials);
  a.error = reinterpret_cast<unsigned*>(base) + 1;
  void* args[] = {&a};
  const void* fn = plan->flags ? reinterpret_cast<const void*>(&tsm_tn_batched_kernel<true>)
                               : reinterpret_cast<const void*>(&tsm_tn_batched_kernel<false>);
  const cudaError_t e = cudaLaunchKernel(fn, dim3(plan->grid),
                                         dim3(batched::kThreads), args, batched::kSmemBytes,
                                         static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(e, "cudaLaunchKernel(batched)");
  return TSM_SUCCESS;
}

}  // extern "C"
