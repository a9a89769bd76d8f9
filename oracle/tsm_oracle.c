/*
 * tsm_oracle.c -- CPU oracle for TSMTTSM, C = A^T * B.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker.  Only tests/, the
 * smoke entry point and bench.py's CPU-baseline leg load it; the library in
 * tsm_benchmark_b200/ never links, loads or calls it, and has no CPU path.
 *
 * Conventions (rectangular generalisation of the reference's square case):
 *   A is n x m, B is n x k, both row-major with leading dimensions lda >= m
 *   and ldb >= k;  C is m x k row-major with leading dimension ldc >= k.
 * The reference (nilsfriess/tsm_benchmark) calls the long dimension K and the
 * square width M (tsmttsm.hh:5-10); every function here takes n, m, k.
 *
 * Built with -ffp-contract=off so that a*b+c is never fused: the naive
 * restatement then rounds exactly like the reference's compute_naive compiled
 * with the same flag, which the CPU tests check bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* Plain FP64 product in the reference oracle's summation order.             */
/* ------------------------------------------------------------------------ */

/* Restates compute_naive (main.cc:14-27): for each output (i, j), one running
 * FP64 sum over the rows r = 0, 1, ..., n-1 of A[r][i] * B[r][j], starting
 * from zero.  Same loop nest (i outer, j, then r) and the same operation
 * order, with 64-bit indices instead of the reference's int (which overflows
 * once n * width reaches 2^31).  Overwrites C. */
EXPORT void tsm_oracle_naive_f64(int64_t n, int m, int k, const double* A,
                                 int64_t lda, const double* B, int64_t ldb,
                                 double* C, int64_t ldc) {
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < k; ++j) {
      double acc = 0.0;
      for (int64_t r = 0; r < n; ++r) acc += A[r * lda + i] * B[r * ldb + j];
      C[(int64_t)i * ldc + j] = acc;
    }
  }
}

/* FP32-input variant used to check the split-precision forms: every product
 * and sum is done in FP64 on the FP32 values (exact products), in the same
 * order as tsm_oracle_naive_f64. */
EXPORT void tsm_oracle_naive_f32in(int64_t n, int m, int k, const float* A,
                                   int64_t lda, const float* B, int64_t ldb,
                                   double* C, int64_t ldc) {
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < k; ++j) {
      double acc = 0.0;
      for (int64_t r = 0; r < n; ++r)
        acc += (double)A[r * lda + i] * (double)B[r * ldb + j];
      C[(int64_t)i * ldc + j] = acc;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Compensated (double-double) product: a near-exact reference used to say    */
/* which side of a comparison carries the rounding error.                    */
/* ------------------------------------------------------------------------ */

/* Error-free transformations (Dekker/Knuth TwoSum, FMA-based TwoProduct;
 * Ogita, Rump and Oishi, "Accurate sum and dot product", SIAM J. Sci.
 * Comput. 26(6), 2005, algorithm Dot2).  C_hi receives the double nearest the
 * compensated sum, C_lo (optional) the remainder. */
EXPORT void tsm_oracle_dot2_f64(int64_t n, int m, int k, const double* A,
                                int64_t lda, const double* B, int64_t ldb,
                                double* C_hi, double* C_lo, int64_t ldc) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < k; ++j) {
      double s = 0.0, c = 0.0;
      for (int64_t r = 0; r < n; ++r) {
        double a = A[r * lda + i], b = B[r * ldb + j];
        double p = a * b;
        double ep = fma(a, b, -p);
        double t = s + p;
        double z = t - s;
        double es = (s - (t - z)) + (p - z);
        s = t;
        c += es + ep;
      }
      double hi = s + c;
      C_hi[(int64_t)i * ldc + j] = hi;
      if (C_lo) C_lo[(int64_t)i * ldc + j] = c - (hi - s);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Checkers.                                                                 */
/* ------------------------------------------------------------------------ */

/* Element-wise acceptance rule of is_correct (main.cc:29-41): an entry fails
 * when |ref - got| exceeds abs_tol AND rel_tol * max(|ref|, |got|).  Returns
 * the row-major index i*k+j of the first failing entry, or -1.  The reference
 * uses rel 1e-6 / abs 1e-10 (main.cc:30); its generated drivers use abs 1e-4
 * with rel 1e-8 (sycl_codegen.py:305) or rel 1e-6 (sycl_codegen_new.py:403).
 * A NaN in either operand fails. */
EXPORT int64_t tsm_oracle_check_f64(const double* ref, const double* got,
                                    int m, int k, int64_t ldc, double rel_tol,
                                    double abs_tol) {
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < k; ++j) {
      double r = ref[(int64_t)i * ldc + j], g = got[(int64_t)i * ldc + j];
      double diff = fabs(r - g);
      double mag = fmax(fabs(r), fabs(g));
      if (!(diff <= abs_tol) && !(diff <= rel_tol * mag))
        return (int64_t)i * k + j;
    }
  return -1;
}

/* Normwise comparison: out[0] = ||got - ref||_F, out[1] = ||A||_F,
 * out[2] = ||B||_F, out[3] = 4 * sqrt(n) * 2^-53 * ||A||_F * ||B||_F (the
 * acceptance bound for the plain FP64 path).  Frobenius norms are
 * accumulated in long double. */
EXPORT void tsm_oracle_normwise_f64(int64_t n, int m, int k, const double* A,
                                    int64_t lda, const double* B, int64_t ldb,
                                    const double* ref, const double* got,
                                    int64_t ldc, double* out) {
  long double d2 = 0, a2 = 0, b2 = 0;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < k; ++j) {
      long double d = (long double)got[(int64_t)i * ldc + j] -
                      (long double)ref[(int64_t)i * ldc + j];
      d2 += d * d;
    }
  for (int64_t r = 0; r < n; ++r) {
    for (int i = 0; i < m; ++i) a2 += (long double)A[r * lda + i] * A[r * lda + i];
    for (int j = 0; j < k; ++j) b2 += (long double)B[r * ldb + j] * B[r * ldb + j];
  }
  out[0] = (double)sqrtl(d2);
  out[1] = (double)sqrtl(a2);
  out[2] = (double)sqrtl(b2);
  out[3] = 4.0 * sqrt((double)n) * ldexp(1.0, -53) * out[1] * out[2];
}

/* ------------------------------------------------------------------------ */
/* Input generators.                                                         */
/* ------------------------------------------------------------------------ */

/* Counter-based uniform[-1, 1) generator: element i of stream s under seed
 * is 2*u - 1 with u the top 53 bits of SplitMix64 (Steele, Lea and Flood,
 * "Fast splittable pseudorandom number generators", OOPSLA 2014) applied to
 * seed + (s * 2^40 + i + 1) * golden-gamma, scaled by 2^-53.  2*u - 1 is
 * exact in FP64, so the device generator in the library produces the same
 * bits.  Values do not depend on the thread count (unlike main.cc:72-86). */
static inline uint64_t splitmix64_at(uint64_t seed, uint64_t stream,
                                     uint64_t i) {
  uint64_t z = seed + ((stream << 40) + i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

EXPORT void tsm_oracle_fill_uniform_f64(double* x, int64_t count,
                                        uint64_t seed, uint64_t stream) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < count; ++i) {
    double u = (double)(splitmix64_at(seed, stream, (uint64_t)i) >> 11) *
               0x1.0p-53;
    x[i] = 2.0 * u - 1.0;
  }
}

/* The single-threaded input generator of main.cc:71-86 (the build without
 * OpenMP seeds one engine with 123): a minimal-standard Lehmer engine
 * (Park and Miller 1988, multiplier 16807, modulus 2^31 - 1, i.e.
 * std::minstd_rand0) feeding a uniform real distribution on [lo, hi), with
 * A[i] and B[i] drawn alternately from the one engine.  The canonical
 * [0, 1) variate follows the C++ standard's generate_canonical
 * ([rand.util.canonical]) for 53 bits from an engine of range
 * R = 2^31 - 2: two draws, S = (g0 - 1) + (g1 - 1) * R, u = S / R^2 (in
 * double arithmetic, u clamped below 1), then x = u * (hi - lo) + lo. */
EXPORT void tsm_oracle_fill_minstd_f64(double* A, double* B, int64_t count,
                                       uint32_t seed, double lo, double hi) {
  const uint64_t mod = 2147483647u;
  uint64_t state = seed % mod;
  if (state == 0) state = 1;
  const double R = 2147483646.0;
  for (int64_t i = 0; i < 2 * count; ++i) {
    double sum = 0.0, scale = 1.0;
    for (int d = 0; d < 2; ++d) {
      state = (state * 16807u) % mod;
      sum += (double)(state - 1) * scale;
      scale *= R;
    }
    double u = sum / scale;
    if (u >= 1.0) u = nextafter(1.0, 0.0);
    double x = u * (hi - lo) + lo;
    if (i % 2 == 0)
      A[i / 2] = x;
    else
      B[i / 2] = x;
  }
}

/* ------------------------------------------------------------------------ */
/* OpenMP restatements of the reference kernels (CPU baseline, kind "port"). */
/* ------------------------------------------------------------------------ */

static inline void atomic_add_f64(double* p, double v) {
  uint64_t old_bits, new_bits;
  __atomic_load(( uint64_t*)p, &old_bits, __ATOMIC_RELAXED);
  do {
    double old_v;
    memcpy(&old_v, &old_bits, 8);
    double nv = old_v + v;
    memcpy(&new_bits, &nv, 8);
  } while (!__atomic_compare_exchange((uint64_t*)p, &old_bits, &new_bits, 0,
                                      __ATOMIC_RELAXED, __ATOMIC_RELAXED));
}

/* Variant 4 of tsmttsm.hh:125-166 (the variant main.cc times) restated for
 * host threads: `stride` work-items; work-item t owns the interleaved tile
 * (r0, c0) = (t % tiles % tpd, t % tiles / tpd) whose columns are
 * r0 + i*tpd and c0 + j*tpd (tpd = m / tile), walks the rows t / tiles,
 * t / tiles + stride / tiles, ... accumulating a tile x tile register block,
 * then adds the block into C with relaxed atomics.  Widths must be square
 * (m == k) and divisible by `tile`, as the reference's static_assert
 * requires.  Accumulates into C (the caller zeroes it, main.cc:67-69). */
EXPORT int tsm_oracle_v4_omp(int64_t n, int m, int stride, int tile,
                             const double* A, const double* B, double* C) {
  if (tile > m) tile = m;
  if (tile <= 0 || m % tile || tile > 8) return -1;
  const int tiles = (m / tile) * (m / tile), tpd = m / tile;
  if (stride % tiles) return -1;
  const int64_t kstride = stride / tiles;
#pragma omp parallel for schedule(static)
  for (int t = 0; t < stride; ++t) {
    double acc[8][8] = {{0}};
    double av[8], bv[8];
    const int tile_idx = t % tiles;
    const int r0 = tile_idx % tpd, c0 = tile_idx / tpd;
    for (int64_t r = t / tiles; r < n; r += kstride) {
      const double* ar = A + r * m;
      const double* br = B + r * m;
      for (int i = 0; i < tile; ++i) {
        av[i] = ar[r0 + i * tpd];
        bv[i] = br[c0 + i * tpd];
      }
      for (int i = 0; i < tile; ++i)
        for (int j = 0; j < tile; ++j) acc[i][j] += av[i] * bv[j];
    }
    for (int i = 0; i < tile; ++i)
      for (int j = 0; j < tile; ++j)
        atomic_add_f64(&C[(int64_t)(r0 + i * tpd) * m + (c0 + j * tpd)],
                       acc[i][j]);
  }
  return 0;
}

/* Number of host threads an OpenMP region would use. */
EXPORT int tsm_oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Oracles for the derived forms (backward TSMM, batched products).          */
/* ------------------------------------------------------------------------ */

/* Tall-skinny times small: Y (n x q) = X (n x p) * W, with W p x q read as
 * W[a][b] = Wm[a * w_row + b * w_col] so that both W and W^T can be passed
 * without copies.  One FP64 sum per output in the order a = 0..p-1.  With
 * X = B, W = dC^T this is the backward dA = B * dC^T of C = A^T * B; with
 * X = A, W = dC it is dB = A * dC.  beta = 0 overwrites Y, 1 accumulates. */
EXPORT void tsm_oracle_tsmm_f64(int64_t n, int p, int q, const double* X,
                                int64_t ldx, const double* Wm, int64_t w_row,
                                int64_t w_col, double* Y, int64_t ldy,
                                int beta) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; ++r)
    for (int b = 0; b < q; ++b) {
      double acc = 0.0;
      for (int a = 0; a < p; ++a) acc += X[r * ldx + a] * Wm[a * w_row + b * w_col];
      Y[r * ldy + b] = beta ? Y[r * ldy + b] + acc : acc;
    }
}

/* ------------------------------------------------------------------------ */
/* Streaming compensated product for the full-size checks.                   */
/* ------------------------------------------------------------------------ */

/* The full-size configurations (up to 2^26 rows, 32 GiB per operand) are
 * checked against a compensated product (Dot2, Ogita, Rump and Oishi 2005,
 * as tsm_oracle_dot2_f64 above) computed over row blocks, so that the host
 * never holds a whole operand.  Its result is within about one rounding of
 * the exact A^T B, so the comparison measures the tested kernel's own error
 * against the normwise bound 4 sqrt(n) 2^-53 ||A||_F ||B||_F.
 *
 * State carried across calls (the caller zero-fills it first):
 *   S[m*k], E[m*k]  -- the double-double sum, value S + E;
 *   nrm[2]          -- sum of A's squares, sum of B's squares;
 *   absC[m*k]       -- optional (NULL to skip): sum_r |a_ri| |b_rj|, the
 *                      entries' own condition scale.
 * Each call splits its rows over the OpenMP threads (contiguous ranges), each
 * thread keeps its own double-double sums, and the threads' sums are merged
 * in thread order with the same error-free additions. */

#define DOT2_BLOCK 256

static inline void dot2_merge(double* s, double* e, double hi, double lo) {
  const double t = *s + hi;
  const double z = t - *s;
  const double es = (*s - (t - z)) + (hi - z);
  *s = t;
  *e += es + lo;
}

/* One block of rows, both operands as doubles with pitches m and k.  The
 * product's rounding error comes from an FMA where the host has one; the
 * other body splits the factors (Veltkamp/Dekker) -- both exact, since the
 * file is compiled with -ffp-contract=off. */
__attribute__((target("avx2,fma"))) static void dot2_rows_fma(
    int64_t rows, int m, int k, const double* a, const double* b, double* s, double* c) {
  for (int64_t r = 0; r < rows; ++r) {
    const double* ar = a + r * m;
    const double* br = b + r * k;
    for (int i = 0; i < m; ++i) {
      const double ai = ar[i];
      double* si = s + (int64_t)i * k;
      double* ci = c + (int64_t)i * k;
#pragma omp simd
      for (int j = 0; j < k; ++j) {
        const double p = ai * br[j];
        const double ep = __builtin_fma(ai, br[j], -p);
        const double t = si[j] + p;
        const double z = t - si[j];
        const double es = (si[j] - (t - z)) + (p - z);
        si[j] = t;
        ci[j] += es + ep;
      }
    }
  }
}

static void dot2_rows_split(int64_t rows, int m, int k, const double* a, const double* b, double* s,
                            double* c) {
  const double kSplit = 134217729.0; /* 2^27 + 1 */
  for (int64_t r = 0; r < rows; ++r) {
    const double* ar = a + r * m;
    const double* br = b + r * k;
    for (int i = 0; i < m; ++i) {
      const double ai = ar[i];
      const double ga = kSplit * ai, ah = ga - (ga - ai), al = ai - ah;
      double* si = s + (int64_t)i * k;
      double* ci = c + (int64_t)i * k;
#pragma omp simd
      for (int j = 0; j < k; ++j) {
        const double bj = br[j];
        const double gb = kSplit * bj, bh = gb - (gb - bj), bl = bj - bh;
        const double p = ai * bj;
        const double ep = ((ah * bh - p) + ah * bl + al * bh) + al * bl;
        const double t = si[j] + p;
        const double z = t - si[j];
        const double es = (si[j] - (t - z)) + (p - z);
        si[j] = t;
        ci[j] += es + ep;
      }
    }
  }
}

static int g_force_split = 0;

static int host_has_fma(void) {
  static int cached = -1;
  if (cached < 0) cached = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
  return cached && !g_force_split;
}

/* Makes the streaming product use the factor-splitting body even where the
 * host has an FMA (the CPU tests check both bodies against each other). */
EXPORT void tsm_oracle_force_split(int on) { g_force_split = on; }

/* Where a block's values come from: host arrays (FP64 or FP32, row pitches
 * lda, ldb), or the counter-based uniform generator (A from stream sa, B
 * from stream sb under `seed`; row-major: element (r, i) of A is value
 * r*m + i of its stream; column-major, the layout of A^T stored row-major
 * with pitch n_total: value i*n_total + r). */
typedef struct {
  const void* A;
  const void* B;
  int64_t lda, ldb;
  int f32;
  int generate;
  uint64_t seed;
  int64_t row0; /* global index of row 0 of this call (generator) */
  uint64_t sa, sb;
  int col_major;
  int64_t n_total;
} dot2_source;

static inline double uniform_at(uint64_t seed, uint64_t stream, uint64_t idx) {
  return 2.0 * ((double)(splitmix64_at(seed, stream, idx) >> 11) * 0x1.0p-53) - 1.0;
}

static void gen_block(const dot2_source* src, uint64_t stream, int w, int64_t r, int64_t rows, double* x) {
  const int64_t g = src->row0 + r; /* global first row of the block */
  if (!src->col_major) {
    for (int64_t q = 0; q < rows * w; ++q) x[q] = uniform_at(src->seed, stream, (uint64_t)(g * w + q));
    return;
  }
  for (int i = 0; i < w; ++i)
    for (int64_t q = 0; q < rows; ++q)
      x[q * w + i] = uniform_at(src->seed, stream, (uint64_t)((int64_t)i * src->n_total + g + q));
}

static void dot2_load(const dot2_source* src, int m, int k, int64_t r, int64_t rows, double* a,
                      double* b) {
  if (src->generate) {
    gen_block(src, src->sa, m, r, rows, a);
    gen_block(src, src->sb, k, r, rows, b);
    return;
  }
  for (int64_t q = 0; q < rows; ++q) {
    for (int i = 0; i < m; ++i)
      a[q * m + i] = src->f32 ? (double)((const float*)src->A)[(r + q) * src->lda + i]
                              : ((const double*)src->A)[(r + q) * src->lda + i];
    for (int j = 0; j < k; ++j)
      b[q * k + j] = src->f32 ? (double)((const float*)src->B)[(r + q) * src->ldb + j]
                              : ((const double*)src->B)[(r + q) * src->ldb + j];
  }
}

static int dot2_stream(const dot2_source* src, int64_t rows, int m, int k, double* S, double* E,
                       double* nrm, double* absC) {
  const int64_t mk = (int64_t)m * k;
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  /* per thread: s, c (and abs) sums, two norms */
  const int64_t stride = 3 * mk + 2;
  double* part = (double*)calloc((size_t)nt * (size_t)stride, sizeof(double));
  if (!part) return -1;
  int failed = 0;
  const int fma_ok = host_has_fma();
#pragma omp parallel num_threads(nt)
  {
    int t = 0, T = 1;
#ifdef _OPENMP
    t = omp_get_thread_num();
    T = omp_get_num_threads();
#endif
    const int64_t r0 = rows * t / T, r1 = rows * (t + 1) / T;
    double* s = part + (int64_t)t * stride;
    double* c = s + mk;
    double* ab = c + mk;
    double* nr = ab + mk;
    double* a = (double*)malloc(sizeof(double) * DOT2_BLOCK * (size_t)m);
    double* b = (double*)malloc(sizeof(double) * DOT2_BLOCK * (size_t)k);
    if (!a || !b) {
#pragma omp atomic write
      failed = 1;
    } else {
      for (int64_t r = r0; r < r1; r += DOT2_BLOCK) {
        const int64_t nb = (r1 - r < DOT2_BLOCK) ? r1 - r : DOT2_BLOCK;
        dot2_load(src, m, k, r, nb, a, b);
        if (fma_ok)
          dot2_rows_fma(nb, m, k, a, b, s, c);
        else
          dot2_rows_split(nb, m, k, a, b, s, c);
        for (int64_t q = 0; q < nb * m; ++q) nr[0] += a[q] * a[q];
        for (int64_t q = 0; q < nb * k; ++q) nr[1] += b[q] * b[q];
        if (absC) {
          for (int64_t q = 0; q < nb; ++q)
            for (int i = 0; i < m; ++i) {
              const double ai = fabs(a[q * m + i]);
              for (int j = 0; j < k; ++j) ab[(int64_t)i * k + j] += ai * fabs(b[q * k + j]);
            }
        }
      }
    }
    free(a);
    free(b);
  }
  if (!failed) {
    for (int t = 0; t < nt; ++t) {
      const double* s = part + (int64_t)t * stride;
      const double* c = s + mk;
      const double* ab = c + mk;
      const double* nr = ab + mk;
      for (int64_t q = 0; q < mk; ++q) {
        dot2_merge(&S[q], &E[q], s[q], c[q]);
        if (absC) absC[q] += ab[q];
      }
      nrm[0] += nr[0];
      nrm[1] += nr[1];
    }
  }
  free(part);
  return failed ? -1 : 0;
}

/* Adds one chunk of host rows (A: rows x m, pitch lda; B: rows x k, pitch
 * ldb; FP64, or FP32 widened exactly when f32 != 0) into the state.
 * Returns 0, or -1 when a buffer could not be allocated. */
EXPORT int tsm_oracle_dot2_acc(int64_t rows, int m, int k, const void* A, int64_t lda, const void* B,
                               int64_t ldb, int f32, double* S, double* E, double* nrm, double* absC) {
  if (rows <= 0) return 0;
  dot2_source src = {A, B, lda, ldb, f32, 0, 0, 0, 0, 0, 0, 0};
  return dot2_stream(&src, rows, m, k, S, E, nrm, absC);
}

/* The same over counter-based uniform operands of `seed`: A from stream sa,
 * B from stream sb (sb == sa with k == m: B is A, the Gram product), rows
 * [row0, row0 + rows) of an n_total-row operand pair, row-major (contiguous)
 * or column-major (A^T stored row-major with pitch n_total): the values the
 * library's device fill writes into those buffers, generated block by block
 * on the host. */
EXPORT int tsm_oracle_dot2_uniform_ex(int64_t row0, int64_t rows, int64_t n_total, int m, int k,
                                      uint64_t seed, uint64_t sa, uint64_t sb, int col_major, double* S,
                                      double* E, double* nrm, double* absC) {
  if (rows <= 0) return 0;
  dot2_source src = {NULL, NULL, 0, 0, 0, 1, seed, row0, sa, sb, col_major, n_total};
  return dot2_stream(&src, rows, m, k, S, E, nrm, absC);
}

/* Row-major operands, A = stream 0, B = stream 1: oracle.operands' values. */
EXPORT int tsm_oracle_dot2_uniform(int64_t row0, int64_t rows, int m, int k, uint64_t seed, double* S,
                                   double* E, double* nrm, double* absC) {
  return tsm_oracle_dot2_uniform_ex(row0, rows, row0 + rows, m, k, seed, 0, 1, 0, S, E, nrm, absC);
}
