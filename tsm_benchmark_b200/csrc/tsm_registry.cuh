// tsm_registry.cuh -- the table of compiled kernel variants.
//
// The reference picks its launch shape through template parameters and
// generated kernel names (tsmttsm.hh: <M, stride, local_size, tile>;
// sycl_codegen_new.py:153 names tsmttsm_{M}_{N}_{TM}_{TN}{,_lf,_sg,_sg_lf}).
// Here every compiled configuration is one row of a table, written by
// tsm_benchmark_b200/codegen.py into csrc/generated/; the host dispatcher and
// the autotuner choose rows by index.
#pragma once

#include <cstddef>

#include "tsm_dmma.cuh"
#include "tsm_plain.cuh"

namespace tsm {

enum VariantKind : int { kKindBulk = 0, kKindDirect = 1, kKindDmma = 2 };
enum DType : int { kF64 = 0, kF32 = 1 };

template <typename T>
struct DTypeOf;
template <>
struct DTypeOf<double> {
  static constexpr int value = kF64;
};
template <>
struct DTypeOf<float> {
  static constexpr int value = kF32;
};

struct Variant {
  const char* name;
  int kind;     // VariantKind
  int dtype;    // DType of A, B and C
  int wa, wb;   // widths (exact) or capacities
  int ta, tb;   // per-thread tile of C (DMMA: per-warp region of C)
  int exact;    // 1: only m == wa && k == wb; 0: any m <= wa, k <= wb
  int threads;  // CTA size
  int stages;   // bulk: shared-memory ring depth
  int rows;     // bulk: rows per chunk (RS)
  int unroll;   // bulk: row-loop unroll
  size_t smem;  // dynamic shared memory per CTA
  const void* kernel;
  int gram;     // 1: B must be A (m == k, same data): streams A once, C written symmetric
};

struct VariantPart {
  const Variant* rows;
  int count;
};

// Parts written by the generator (csrc/generated/variants_index.cu).
extern const VariantPart kVariantParts[];
extern const int kVariantPartCount;

}  // namespace tsm

#define TSM_BULK_VARIANT(NAME, T, WA, WB, TA, TB, CW, ST, RS, U, EX, GR)                                 \
  ::tsm::Variant {                                                                                       \
    NAME, ::tsm::kKindBulk, ::tsm::DTypeOf<T>::value, WA, WB, TA, TB, EX,                                \
        ::tsm::BulkKernel<T, WA, WB, TA, TB, CW, ST, RS, U, EX, GR>::THREADS, ST, RS, U,                 \
        ::tsm::BulkKernel<T, WA, WB, TA, TB, CW, ST, RS, U, EX, GR>::SMEM_BYTES,                         \
        reinterpret_cast<const void*>(&::tsm::tsm_tn_bulk_kernel<T, WA, WB, TA, TB, CW, ST, RS, U, EX, GR>), GR \
  }

#define TSM_DIRECT_VARIANT(NAME, T, WA, WB, TA, TB, TH, EX)                                        \
  ::tsm::Variant {                                                                                 \
    NAME, ::tsm::kKindDirect, ::tsm::DTypeOf<T>::value, WA, WB, TA, TB, EX, TH, 0, 0, 1,           \
        ::tsm::DirectKernel<T, WA, WB, TA, TB, TH, EX>::SMEM_BYTES,                                \
        reinterpret_cast<const void*>(&::tsm::tsm_tn_direct_kernel<T, WA, WB, TA, TB, TH, EX>), 0  \
  }

#define TSM_DMMA_VARIANT(NAME, WA, WB, MT, NT, CW, ST, RS)                                               \
  ::tsm::Variant {                                                                                       \
    NAME, ::tsm::kKindDmma, ::tsm::kF64, WA, WB, MT * 8, NT * 8, 1,                                        \
        ::tsm::DmmaTn<WA, WB, MT, NT, CW, ST, RS>::THREADS, ST, RS, 1,                                     \
        ::tsm::DmmaTn<WA, WB, MT, NT, CW, ST, RS>::SMEM_BYTES,                                             \
        reinterpret_cast<const void*>(&::tsm::tsm_tn_dmma_kernel<WA, WB, MT, NT, CW, ST, RS>), 0           \
  }

// Gram C = A^T A on the tensor cores, upper-triangle block pairs (tile fields:
// the 16 x 16 block pairs it works in).
#define TSM_GRAM_DMMA_VARIANT(NAME, W, CW, ST, RS)                                                        \
  ::tsm::Variant {                                                                                       \
    NAME, ::tsm::kKindDmma, ::tsm::kF64, W, W, 16, 16, 1, ::tsm::GramDmma<W, CW, ST, RS>::THREADS, ST, RS, 1, \
        ::tsm::GramDmma<W, CW, ST, RS>::SMEM_BYTES,                                                        \
        reinterpret_cast<const void*>(&::tsm::tsm_gram_dmma_kernel<W, CW, ST, RS>), 1                      \
  }
