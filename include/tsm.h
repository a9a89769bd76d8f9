/*
 * tsm.h -- C ABI of the B200 TSMTTSM library (C = A^T * B, tall and skinny).
 *
 * Shapes: A is n x m, B is n x k, both row-major with leading dimensions
 * lda >= m and ldb >= k (in elements); C is m x k row-major with leading
 * dimension ldc >= k.  1 <= m, k <= 64; n >= 0 (int64).  All pointers are
 * device pointers (cudaMalloc / cudaMallocManaged); all calls are
 * asynchronous and ordered on `stream` (a cudaStream_t, NULL = the legacy
 * default stream), like the reference's in-order sycl::queue submits.
 *
 * The reference (nilsfriess/tsm_benchmark) exposes the same operation as
 * C++ templates, `template <typename T, int M, ...> sycl::event
 * tsmttsmN(sycl::queue& q, int K, T* A, T* B, T* C)` for N in
 * {"",2,...,9} (tsmttsm.hh:15-586), and as generated functions
 * `tsmttsm_{M}_{N}_{TM}_{TN}[_lf|_sg|_sg_lf](q, K, const T* A, const T* B,
 * T* C)` (sycl_codegen_new.py:153,159,257,264).  Those always ADD into C
 * (the caller zero-fills C first, main.cc:67-69,93) and have square widths
 * M = N as compile-time parameters; here widths are run-time arguments,
 * rectangular, and `accumulate` selects C += A^T B (reference semantics) or
 * C = A^T B.  The compat header tsm_benchmark_b200/compat/tsmttsm.hh maps the
 * reference's template names onto these entry points.
 *
 * Workspace: callers pass device scratch of at least
 * tsm_gemm_tn_workspace_size(...) bytes, ZERO-FILLED before its first use
 * (e.g. cudaMemsetAsync(ws, 0, bytes, stream)).  Every call leaves it ready
 * for the next one.  Calls that may run concurrently (different streams)
 * need different workspaces.  The library itself never allocates.
 *
 * Results are deterministic: the same inputs, shapes and variant give
 * bit-identical C on every run (no floating-point atomics).
 */
#ifndef TSM_H_
#define TSM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tsm_status {
  TSM_SUCCESS = 0,
  TSM_ERROR_INVALID_VALUE = 1,  /* bad shape, null pointer, bad leading dim  */
  TSM_ERROR_WORKSPACE = 2,      /* workspace missing or too small            */
  TSM_ERROR_CUDA = 3,           /* a CUDA runtime call failed (see below)    */
  TSM_ERROR_UNSUPPORTED = 4,    /* no compiled variant for this request      */
  TSM_ERROR_DEVICE_TIMEOUT = 5  /* a kernel gave up a bounded wait           */
} tsm_status;

typedef void* tsm_stream_t; /* cudaStream_t */

/* Library version, major * 10000 + minor * 100 + patch. */
int tsm_version(void);

/* Static description of a status code. */
const char* tsm_status_string(tsm_status status);

/* Text of the last CUDA error seen by the calling host thread ("" if none). */
const char* tsm_last_cuda_error(void);

/* Bytes of workspace one plain call with these widths needs on the current
 * device (independent of n).  New in this library: the reference kernels
 * need no workspace because they reduce with FP64 atomics into C. */
size_t tsm_gemm_tn_workspace_size(int64_t n, int m, int k);

/* C = A^T B (accumulate = 0) or C += A^T B (accumulate = 1), FP64.
 * Replaces tsmttsm / tsmttsm2 ... tsmttsm9 <double, M, ...> (tsmttsm.hh:15-586)
 * and the generated tsmttsm_{M}_{N}_{TM}_{TN}* kernels (sycl_codegen.py:16-263,
 * sycl_codegen_new.py:142-363); the reference's driver calls are
 * main.cc:103-105,148-150 and sycl_codegen_new.py:484-487.
 * The variant is the autotuned default for (m, k, n). */
tsm_status tsm_gemm_tn_f64(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                           const double* B, int64_t ldb, double* C, int64_t ldc, int accumulate,
                           void* workspace, size_t workspace_bytes);

/* Same, with an explicit variant index (0 <= variant < tsm_variant_count()),
 * or -1 for the default.  Returns TSM_ERROR_UNSUPPORTED if that variant
 * cannot run this request (width, leading dimension or alignment).  Used by
 * the autotuner; replaces choosing a reference kernel by template
 * parameters (main.cc:171-192) or by generated name. */
tsm_status tsm_gemm_tn_f64_variant(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                                   const double* B, int64_t ldb, double* C, int64_t ldc, int accumulate,
                                   void* workspace, size_t workspace_bytes, int variant);

/* Same as tsm_gemm_tn_f64_variant, launching at most max_ctas CTAs (<= 0:
 * the variant's own grid, one or a few CTAs per SM; max_ctas never raises
 * it).  Every kernel deals its rows over whatever grid it gets, so the
 * result is the same product; the last CTA's sum over the per-CTA partials
 * follows the grid, so bits may differ from another grid's.  Replaces the
 * launch-size parameters of the reference: `stride` (the work-item count of
 * tsmttsm.hh:15-439 and of the generated kernels, sycl_codegen.py:466,
 * sycl_codegen_new.py:594) with `local_size` (:468, :596) -- a caller maps
 * stride / local_size work-groups to CTAs, as the generated drop-in header
 * does. */
tsm_status tsm_gemm_tn_f64_launch(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                                  const double* B, int64_t ldb, double* C, int64_t ldc, int accumulate,
                                  void* workspace, size_t workspace_bytes, int variant, int64_t max_ctas);

/* C = A^T B or C += A^T B with FP32 storage (A, B, C float).  Each thread
 * accumulates in FP32 over its rows; every sum across threads and CTAs is
 * FP64, then rounded once to FP32.  The FP32 forward of the autograd form
 * (torch.autograd.Function over the C ABI).  Same workspace as the FP64 call. */
tsm_status tsm_gemm_tn_f32(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                           const float* B, int64_t ldb, float* C, int64_t ldc, int accumulate, void* workspace,
                           size_t workspace_bytes);
tsm_status tsm_gemm_tn_f32_variant(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                                   const float* B, int64_t ldb, float* C, int64_t ldc, int accumulate,
                                   void* workspace, size_t workspace_bytes, int variant);

/* The precision form: C (FP64) = A^T B (accumulate = 0) or C += A^T B for
 * FP32-stored A, B on the tcgen05 tensor cores, 1 <= m, k <= 32, A and B
 * contiguous (lda = m, ldb = k) and 16-byte aligned.  Each FP32 value is
 * split into two TF32 parts, x ~ hi + lo; one tcgen05.mma per 8 rows forms
 * hi.hi + hi.lo + lo.hi + lo.lo with FP32 accumulation, drained to FP64
 * every 256 rows (widths that are multiples of 4) or 128 rows (others);
 * every later sum is FP64 and fixed-order (deterministic).
 * Widths that are multiples of 4 load the raw tile with 2-D TMA and use
 * hi = trunc_tf32(x), lo = rna_tf32(x - hi) (|x - hi - lo| <= 2^-21 |x|);
 * other widths use hi = rna_tf32(x), lo = rna_tf32(x - hi) (<= 2^-22 |x|).
 * Stated error: <= 1e-6 normwise and per entry (of sum_r |a_ri| |b_rj|)
 * against the FP64 oracle; measured at n = 2^25, m = k = 32 on
 * column-scaled data: 4.9e-7 normwise (2.7e-7 with drains every 128 rows,
 * 9 % slower under sustained load).  Reads half the bytes of the FP64
 * path on the same values.  No counterpart in the reference (its kernels are
 * FP64 only).  Workspace: as tsm_gemm_tn_workspace_size(n, m, k). */
tsm_status tsm_gemm_tn_f32_split(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                                 const float* B, int64_t ldb, double* C, int64_t ldc, int accumulate, void* workspace,
                                 size_t workspace_bytes);

/* The precision form with BF16 parts (kind::f16 tensor-core MMAs, K = 16
 * rows per instruction): each FP32 value is split into `parts` BF16 values,
 * h = rn(x) then rn of the remainder -- parts = 2 (hi/lo): |x - h - l| <=
 * 2^-16 |x|, about 1e-5 relative error on C, ABOVE the 1e-6 of the TF32
 * form; parts = 3 (hi/mid/lo): <= 2^-24 |x|.  One MMA per 16 rows forms all
 * parts x parts products, FP32 accumulation per 256 rows, FP64 beyond.  A and
 * B contiguous (lda = m, ldb = k), 16-byte aligned, m and k multiples of 4
 * up to 32 (else TSM_ERROR_UNSUPPORTED).  No counterpart in the reference.
 * Workspace: as tsm_gemm_tn_workspace_size(n, m, k). */
tsm_status tsm_gemm_tn_f32_split_bf16(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                                      const float* B, int64_t ldb, double* C, int64_t ldc, int accumulate, int parts,
                                      void* workspace, size_t workspace_bytes);

/* Element types of the plain entry points. */
#define TSM_F64 0
#define TSM_F32 1

/* Index of the variant tsm_gemm_tn_f64 (dtype TSM_F64) or tsm_gemm_tn_f32
 * (TSM_F32) would run for this request, or -1. */
int tsm_gemm_tn_default_variant(int dtype, int64_t n, int m, int k, const void* A, int64_t lda, const void* B,
                                int64_t ldb);

typedef struct tsm_variant_info {
  char name[64];
  int kind;    /* 0 = TMA bulk pipeline, 1 = direct loads, 2 = FP64 tensor cores (2-D TMA) */
  int dtype;   /* TSM_F64 or TSM_F32 */
  int wa, wb;  /* widths (exact) or width capacities */
  int ta, tb;  /* per-thread tile of C (kind 2: per-warp region of C) */
  int exact;   /* 1: only m == wa, k == wb */
  int threads, stages, rows, unroll;
  size_t smem_bytes;
  int gram;    /* 1: for C = A^T A only (B is A): streams A once, writes C symmetric */
} tsm_variant_info;

/* Number of compiled variants, and the description of one. */
int tsm_variant_count(void);
tsm_status tsm_variant_get_info(int index, tsm_variant_info* info);

/* Reads and clears the workspace's device error word (synchronises
 * `stream`).  *bits != 0 means a kernel gave up a bounded wait and its C is
 * not valid; the call then returns TSM_ERROR_DEVICE_TIMEOUT. */
tsm_status tsm_workspace_check(tsm_stream_t stream, void* workspace, unsigned* bits);

/* Self-test of the device failure path: launches one kernel whose wait on
 * an mbarrier that nothing arrives on runs out after limit_us microseconds
 * (1 .. 2,000,000) -- through the same bounded wait every pipeline uses --
 * and records the timeout in the workspace's error word.  A following
 * tsm_workspace_check returns TSM_ERROR_DEVICE_TIMEOUT and clears the word;
 * the context stays usable.  No fault, no trap.  No counterpart in the
 * reference (it has no failure detection). */
tsm_status tsm_selftest_wait_timeout(tsm_stream_t stream, void* workspace, size_t workspace_bytes,
                                     unsigned limit_us);

/* C = A^T A (accumulate = 0) or C += A^T A, FP64: the Gram matrix of a tall
 * and skinny A (n x m, pitch lda).  Reads A once -- half the bytes of
 * tsm_gemm_tn_f64 on two operands -- and writes C exactly symmetric (each
 * upper-triangle sum is written to both (i, j) and (j, i)).  tsm_gemm_tn_f64
 * takes the same path when B is A (same pointer, pitch and width).  No
 * counterpart in the reference (its drivers always pass distinct A and B,
 * main.cc:63-64).  Workspace: tsm_gemm_tn_workspace_size(n, m, m). */
tsm_status tsm_gram_f64(tsm_stream_t stream, int64_t n, int m, const double* A, int64_t lda, double* C, int64_t ldc,
                        int accumulate, void* workspace, size_t workspace_bytes);

/* C = A^T B (accumulate = 0) or C += A^T B, FP64, for operands in any
 * element layout: A's element (r, i), r < n, i < m, is A[r * a_row + i *
 * a_col] and B's (r, j) is B[r * b_row + j * b_col]; every stride >= 1.
 * Row-major operands (a_col = b_col = 1, a_row >= m, b_row >= k) take the
 * tsm_gemm_tn_f64 path.  Column-major operands (a_row = b_row = 1: A stored
 * as the m x n row-major matrix A^T with pitch a_col >= n, B likewise) stream
 * through tensor maps when the bases are 16-byte aligned, the pitches even and
 * n <= 2^31 - 8193 (values of r contiguous, columns zero-padded to the
 * kernel's capacity);
 * FP64 tensor cores when the widths rounded up to powers of two multiply to
 * more than 64.  Any other layout (mixed, odd pitches, unaligned) runs a
 * register-tile kernel with strided loads: correct, not tuned.  No
 * counterpart in the reference, whose operands are always row-major with
 * pitch M (tsmttsm.hh:15-35; sycl_codegen_new.py:66-67).  Same workspace as
 * tsm_gemm_tn_f64 (tsm_gemm_tn_workspace_size(n, m, k)). */
tsm_status tsm_gemm_tn_strided_f64(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t a_row,
                                   int64_t a_col, const double* B, int64_t b_row, int64_t b_col, double* C,
                                   int64_t ldc, int accumulate, void* workspace, size_t workspace_bytes);

/* C = A^T B (accumulate = 0) or C += A^T B (accumulate = 1), FP64, WITHOUT a
 * workspace.  No counterpart in the reference (its SYCL kernels need no
 * scratch because they add into C with atomics).  For callers that cannot
 * allocate device memory or own a workspace -- a plug-in whose host program
 * owns every device allocation, or a latency-bound loop where cudaMalloc
 * (which may synchronise the device) is not allowed -- this entry point
 * allocates nothing: its scratch is a 4 MiB array inside the library that
 * every GPU loading the library holds until exit.  Same variant choice and
 * result as tsm_gemm_tn_f64.  Limit: the call needs 256 + CTAs * m * k * 8
 * bytes of that array.  On a 148-SM B200 with contiguous, 16-byte aligned
 * operands (one CTA per SM) that admits any n for m * k <= 3542, and 64 x 64
 * up to about 4,000 rows; strided or unaligned operands (up to four CTAs per
 * SM) admit any n for m * k <= 885.  Larger requests return
 * TSM_ERROR_WORKSPACE and launch nothing.  All calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller.  The
 * first call on each device looks up the array's device address; make it
 * before any stream capture.  The address, like all per-device state of the
 * library, does not survive cudaDeviceReset.  A kernel that gives up a
 * bounded wait records it in the array's error word: read it with
 * tsm_noalloc_check. */
tsm_status tsm_gemm_tn_f64_noalloc(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                                   const double* B, int64_t ldb, double* C, int64_t ldc, int accumulate);

/* Reads and clears the error word of tsm_gemm_tn_f64_noalloc's built-in
 * scratch on the current device (synchronises `stream`), as
 * tsm_workspace_check does for a caller's workspace: *bits != 0 means a
 * kernel of an earlier no-allocation call gave up a bounded wait and its C
 * is not valid; the call then returns TSM_ERROR_DEVICE_TIMEOUT.  The word
 * stays set until read.  Allocates nothing.  No counterpart in the reference
 * (it has no failure detection). */
tsm_status tsm_noalloc_check(tsm_stream_t stream, unsigned* bits);

/* Tall-skinny times small (TSMM): Y (n x q) = X (n x p) * W (beta = 0) or
 * Y += X * W (beta = 1), FP64 or FP32, 1 <= p, q <= 64.  W is read as
 * W[a][b] = W[a * w_row + b * w_col], so a row-major p x q matrix is
 * (w_row, w_col) = (q, 1) and the transpose of a row-major q x p matrix is
 * (1, p).  No counterpart in the reference (it has no backward); this is the
 * product the backward of C = A^T B needs, and the second half of block
 * orthogonalisation B - A (A^T B).  Each output is one fixed-order sum over
 * p (deterministic).  Workspace: at least 256 bytes (the device error word);
 * the plain calls' workspace serves. */
tsm_status tsm_tsmm_f64(tsm_stream_t stream, int64_t n, int p, int q, const double* X, int64_t ldx, const double* W,
                        int64_t w_row, int64_t w_col, double* Y, int64_t ldy, int beta, void* workspace,
                        size_t workspace_bytes);
tsm_status tsm_tsmm_f32(tsm_stream_t stream, int64_t n, int p, int q, const float* X, int64_t ldx, const float* W,
                        int64_t w_row, int64_t w_col, float* Y, int64_t ldy, int beta, void* workspace,
                        size_t workspace_bytes);

/* Backward of C = A^T B for a loss L(C): given dC = dL/dC (m x k), writes
 * dA = B * dC^T (n x m) and dB = A * dC (n x k) in ONE launch (either output
 * may be NULL to skip it); beta = 1 adds into dA / dB instead.  Reads A and B
 * once each and writes dA and dB once each: 2x the bytes of the forward.
 * Dense, 16-byte aligned operands run on the FP64 tensor cores (FP32 storage
 * is widened to FP64 in registers: one rounding per output); others on SIMT
 * kernels.  Two launches when the two products need different capacities.
 * No counterpart in the reference (the differentiation form). */
tsm_status tsm_gemm_tn_backward_f64(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda,
                                    const double* B, int64_t ldb, const double* dC, int64_t lddc, double* dA,
                                    int64_t ldda, double* dB, int64_t lddb, int beta, void* workspace,
                                    size_t workspace_bytes);
tsm_status tsm_gemm_tn_backward_f32(tsm_stream_t stream, int64_t n, int m, int k, const float* A, int64_t lda,
                                    const float* B, int64_t ldb, const float* dC, int64_t lddc, float* dA,
                                    int64_t ldda, float* dB, int64_t lddb, int beta, void* workspace,
                                    size_t workspace_bytes);

/* Block orthogonalisation against A: C = A^T B (m x k), then B <- B - A C
 * (in place).  When A has orthonormal columns this removes from B's columns
 * their components in A's span (one block Gram-Schmidt step); C holds the
 * projection coefficients.  Two launches on `stream` -- the product, then a
 * TSMM update (tsm_tsmm_f64 with W = -C, beta = 1) -- reading A twice and B
 * twice and writing B once; a one-kernel form would still read A twice
 * and would need a grid-wide wait for C.  A and B must not overlap.
 * Workspace: tsm_gemm_tn_workspace_size(n, m, k).  No counterpart in the
 * reference (the fused TSMTTSM + TSMM pipeline). */
tsm_status tsm_block_orth_f64(tsm_stream_t stream, int64_t n, int m, int k, const double* A, int64_t lda, double* B,
                             int64_t ldb, double* C, int64_t ldc, void* workspace, size_t workspace_bytes);

/* ---- Batched products: many C_p = A_p^T B_p (+ C_p) in one launch. ----
 * No counterpart in the reference (it submits one kernel per product; the
 * batching form).  Widths m, k in {4, 8, 16, 32}; A_p, B_p contiguous
 * (lda = m, ldb = k) and 16-byte aligned; any n_p >= 0. */
typedef struct tsm_batched_problem_f64 {
  const double* A;
  const double* B;
  double* C;
  int64_t n;
  int m;
  int k;
  int64_t ldc;
  int accumulate;
} tsm_batched_problem_f64;

/* Host handle of a plan whose tables live in caller-owned device memory. */
typedef struct tsm_batched_plan {
  void* device;
  size_t bytes;
  int count;
  int segments;
  int grid;
  int flags;  /* set by the plan init: 1 when a tensor-core class runs its SIMT path */
} tsm_batched_plan;

/* Device bytes the plan for these problems needs on the current device
 * (0 if a problem is invalid or unsupported). */
size_t tsm_batched_plan_size_f64(int count, const tsm_batched_problem_f64* problems);

/* Builds the schedule on the host -- the problems' rows concatenated and cut
 * into one equal byte range per SM, each a list of row segments -- and copies
 * it into `device_buffer` (synchronising `stream`).  Pointers and sizes are
 * baked into the plan: re-initialise it when they change. */
tsm_status tsm_batched_plan_init_f64(tsm_stream_t stream, int count, const tsm_batched_problem_f64* problems,
                                     void* device_buffer, size_t device_bytes, tsm_batched_plan* plan);

/* The same, with the consumer path of each width class chosen by the
 * caller: class_paths[4 log2(m / 4) + log2(k / 4)] is -1 (the autotuned
 * choice, as tsm_batched_plan_init_f64 makes it), 0 (the class's default
 * path: the FP64 tensor cores when m, k >= 16, SIMT register tiles below) or
 * 1 (SIMT 4 x 4 register tiles over 1-D bulk copies; only the tensor-core
 * classes have this second path, the others ignore it).  class_paths may be
 * NULL (all -1).  The autotuner times both paths of each tensor-core class
 * inside the batched launch through this call.  No counterpart in the
 * reference. */
tsm_status tsm_batched_plan_init_paths_f64(tsm_stream_t stream, int count, const tsm_batched_problem_f64* problems,
                                           const int* class_paths, void* device_buffer, size_t device_bytes,
                                           tsm_batched_plan* plan);

/* Runs every product of the plan in ONE persistent launch (capturable in a
 * CUDA graph; the plan's first execution, or any other call, must happen
 * before capture so that the kernel is loaded).  Deterministic for a given
 * plan.  Concurrent executions of one plan race on its counters. */
tsm_status tsm_gemm_tn_batched_f64(tsm_stream_t stream, const tsm_batched_plan* plan);

/* Benchmark-input generator: x[i] = 2u - 1 in [-1, 1), u the top 53 bits of
 * SplitMix64 at counter (stream_id * 2^40 + i + 1) under `seed`.  The same
 * values as the oracle's host generator, bit for bit, independent of the
 * launch shape.  Mirrors the reference drivers' input fill (main.cc:71-86,
 * sycl_codegen_new.py:436-439) with a reproducible generator. */
tsm_status tsm_fill_uniform_f64(tsm_stream_t stream, double* x, int64_t count, uint64_t seed, uint64_t stream_id);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* TSM_H_ */
