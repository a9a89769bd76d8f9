// tsm_tmap.h -- host-side construction of 2-D tensor maps (TMA descriptors)
// for row-major operands, through the runtime's driver entry point (no link
// dependency on the driver library).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstdio>
#include <string>

namespace tsm {

inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Tensor map of a row-major operand: `rows` x `width` elements of `type`
// (`esize` bytes), row pitch `ld` elements, boxes of `box_w` columns x
// `box_rows` rows, the given shared-memory swizzle, zero fill out of bounds.
// Returns false and sets *err on failure.  Needs a 16-byte aligned base and
// ld * esize a multiple of 16.
inline bool encode_rowmajor_map(CUtensorMap* map, CUtensorMapDataType type, int esize, const void* base,
                                int64_t rows, int width, int64_t ld, int box_w, int box_rows,
                                CUtensorMapSwizzle swizzle, std::string* err) {
  auto enc = tensor_map_encoder();
  if (enc == nullptr) {
    *err = "cuTensorMapEncodeTiled: entry point not available";
    return false;
  }
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(width), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * static_cast<cuuint64_t>(esize)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_w), static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = enc(map, type, 2, const_cast<void*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[96];
    std::snprintf(buf, sizeof(buf), "cuTensorMapEncodeTiled: CUresult %d", static_cast<int>(r));
    *err = buf;
    return false;
  }
  return true;
}

}  // namespace tsm
