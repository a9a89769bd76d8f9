// Generated by tsm_benchmark_b200/codegen.py -- do not edit.
// Regenerate with: python -m tsm_benchmark_b200.codegen
//
// Drop-in for the header `sycl_codegen_new.py` emits, on libtsm_b200.so.
// Kernel names and signatures are the reference generator's; every kernel adds
// A^T B into C through tsm_gemm_tn_f64_launch on the queue's stream, with a
// compiled variant of this library (named above each kernel) on at most
// stride / local_size CTAs.
//   widths 4 8 16; tiles 2 4; stride=524288 local_size=256 sg_size=32 unroll=1
#pragma once

#include <sycl/sycl.hpp>

#include <vector>

#include "tsm_compat_bench.hh"
#include "tsmttsm.hh"

// ============================================================
// M = 4
// ============================================================

// runs bulk_4x4_t2x2_w8_s6_r512_u1: deepest ring
template <typename T>
sycl::event tsmttsm_4_4_2_2(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_4x4_t2x2_w8_s6_r512_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 4, 4, A, B, C, variant, 2048);
}

// runs bulk_4x4_t2x2_w8_s6_r512_u1: shallowest ring (double buffer) (the same kernel as tsmttsm_4_4_2_2: no other ring compiled for this tile)
template <typename T>
sycl::event tsmttsm_4_4_2_2_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_4x4_t2x2_w8_s6_r512_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 4, 4, A, B, C, variant, 2048);
}

// runs the autotuned default: chosen per (M, M, K) at run time; every kernel reduces with the two-level sum
template <typename T>
sycl::event tsmttsm_4_4_2_2_sg(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = -1;
  return tsm_compat::accumulate_tn<T>(q, K, 4, 4, A, B, C, variant, 2048);
}

// runs bulk_4x4_t2x2_w8_s6_r512_u1: SIMT tile, middle ring depth (the same kernel as tsmttsm_4_4_2_2: no other ring compiled for this tile)
template <typename T>
sycl::event tsmttsm_4_4_2_2_sg_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_4x4_t2x2_w8_s6_r512_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 4, 4, A, B, C, variant, 2048);
}

// runs bulk_4x4_t4x4_w8_s6_r512_u1: deepest ring
template <typename T>
sycl::event tsmttsm_4_4_4_4(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_4x4_t4x4_w8_s6_r512_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 4, 4, A, B, C, variant, 2048);
}

// runs bulk_4x4_t4x4_w8_s2_r1536_u1: shallowest ring (double buffer)
template <typename T>
sycl::event tsmttsm_4_4_4_4_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_4x4_t4x4_w8_s2_r1536_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 4, 4, A, B, C, variant, 2048);
}

// runs the autotuned default: chosen per (M, M, K) at run time; every kernel reduces with the two-level sum
template <typename T>
sycl::event tsmttsm_4_4_4_4_sg(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = -1;
  return tsm_compat::accumulate_tn<T>(q, K, 4, 4, A, B, C, variant, 2048);
}

// runs bulk_4x4_t4x4_w8_s4_r768_u1: SIMT tile, middle ring depth
template <typename T>
sycl::event tsmttsm_4_4_4_4_sg_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_4x4_t4x4_w8_s4_r768_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 4, 4, A, B, C, variant, 2048);
}

// ============================================================
// M = 8
// ============================================================

// runs bulk_8x8_t4x4_w8_s6_r256_u1: deepest ring; no 2x2 tile compiled for width 8: nearest tile 4x4
template <typename T>
sycl::event tsmttsm_8_8_2_2(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_8x8_t4x4_w8_s6_r256_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 8, 8, A, B, C, variant, 2048);
}

// runs bulk_8x8_t4x4_w8_s2_r768_u1: shallowest ring (double buffer); no 2x2 tile compiled for width 8: nearest tile 4x4
template <typename T>
sycl::event tsmttsm_8_8_2_2_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_8x8_t4x4_w8_s2_r768_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 8, 8, A, B, C, variant, 2048);
}

// runs the autotuned default: chosen per (M, M, K) at run time; every kernel reduces with the two-level sum
template <typename T>
sycl::event tsmttsm_8_8_2_2_sg(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = -1;
  return tsm_compat::accumulate_tn<T>(q, K, 8, 8, A, B, C, variant, 2048);
}

// runs bulk_8x8_t4x4_w8_s4_r384_u1: SIMT tile, middle ring depth; no 2x2 tile compiled for width 8: nearest tile 4x4
template <typename T>
sycl::event tsmttsm_8_8_2_2_sg_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_8x8_t4x4_w8_s4_r384_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 8, 8, A, B, C, variant, 2048);
}

// runs bulk_8x8_t4x4_w8_s6_r256_u1: deepest ring
template <typename T>
sycl::event tsmttsm_8_8_4_4(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_8x8_t4x4_w8_s6_r256_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 8, 8, A, B, C, variant, 2048);
}

// runs bulk_8x8_t4x4_w8_s2_r768_u1: shallowest ring (double buffer)
template <typename T>
sycl::event tsmttsm_8_8_4_4_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_8x8_t4x4_w8_s2_r768_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 8, 8, A, B, C, variant, 2048);
}

// runs the autotuned default: chosen per (M, M, K) at run time; every kernel reduces with the two-level sum
template <typename T>
sycl::event tsmttsm_8_8_4_4_sg(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = -1;
  return tsm_compat::accumulate_tn<T>(q, K, 8, 8, A, B, C, variant, 2048);
}

// runs bulk_8x8_t4x4_w8_s4_r384_u1: SIMT tile, middle ring depth
template <typename T>
sycl::event tsmttsm_8_8_4_4_sg_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_8x8_t4x4_w8_s4_r384_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 8, 8, A, B, C, variant, 2048);
}

// ============================================================
// M = 16
// ============================================================

// runs bulk_16x16_t4x4_w8_s6_r128_u1: deepest ring; no 2x2 tile compiled for width 16: nearest tile 4x4
template <typename T>
sycl::event tsmttsm_16_16_2_2(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_16x16_t4x4_w8_s6_r128_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 16, 16, A, B, C, variant, 2048);
}

// runs bulk_16x16_t4x4_w8_s6_r128_u1: shallowest ring (double buffer); no 2x2 tile compiled for width 16: nearest tile 4x4 (the same kernel as tsmttsm_16_16_2_2: no other ring compiled for this tile)
template <typename T>
sycl::event tsmttsm_16_16_2_2_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_16x16_t4x4_w8_s6_r128_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 16, 16, A, B, C, variant, 2048);
}

// runs the autotuned default: chosen per (M, M, K) at run time; every kernel reduces with the two-level sum
template <typename T>
sycl::event tsmttsm_16_16_2_2_sg(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = -1;
  return tsm_compat::accumulate_tn<T>(q, K, 16, 16, A, B, C, variant, 2048);
}

// runs dmma_16x16_t16x16_w12_s2_r384: FP64 tensor cores, shallowest ring other than the autotuned choice
template <typename T>
sycl::event tsmttsm_16_16_2_2_sg_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("dmma_16x16_t16x16_w12_s2_r384");
  return tsm_compat::accumulate_tn<T>(q, K, 16, 16, A, B, C, variant, 2048);
}

// runs bulk_16x16_t4x4_w8_s6_r128_u1: deepest ring
template <typename T>
sycl::event tsmttsm_16_16_4_4(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_16x16_t4x4_w8_s6_r128_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 16, 16, A, B, C, variant, 2048);
}

// runs bulk_16x16_t4x4_w8_s6_r128_u1: shallowest ring (double buffer) (the same kernel as tsmttsm_16_16_4_4: no other ring compiled for this tile)
template <typename T>
sycl::event tsmttsm_16_16_4_4_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("bulk_16x16_t4x4_w8_s6_r128_u1");
  return tsm_compat::accumulate_tn<T>(q, K, 16, 16, A, B, C, variant, 2048);
}

// runs the autotuned default: chosen per (M, M, K) at run time; every kernel reduces with the two-level sum
template <typename T>
sycl::event tsmttsm_16_16_4_4_sg(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = -1;
  return tsm_compat::accumulate_tn<T>(q, K, 16, 16, A, B, C, variant, 2048);
}

// runs dmma_16x16_t16x16_w12_s2_r384: FP64 tensor cores, shallowest ring other than the autotuned choice
template <typename T>
sycl::event tsmttsm_16_16_4_4_sg_lf(sycl::queue& q, int K, const T* A, const T* B, T* C) {
  static const int variant = tsm_compat::variant_by_name("dmma_16x16_t16x16_w12_s2_r384");
  return tsm_compat::accumulate_tn<T>(q, K, 16, 16, A, B, C, variant, 2048);
}

template <typename T>
void run_all_benchmarks(sycl::queue& q, int K = 1 << 20, int warmup = 10, int runs = 30) {
  std::cout << "Device: " << q.get_device().get_info<sycl::info::device::name>() << "\n\n";
  std::vector<tsm_compat::BenchResult> results;
  {
    tsm_compat::Problem<T> p(q, K, 4, 123, 1e-6);
    results.push_back(p.bench("M4_T2_basic", [&](int k) { return tsmttsm_4_4_2_2<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M4_T2_lf", [&](int k) { return tsmttsm_4_4_2_2_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M4_T2_sg", [&](int k) { return tsmttsm_4_4_2_2_sg<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M4_T2_sg_lf", [&](int k) { return tsmttsm_4_4_2_2_sg_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M4_T4_basic", [&](int k) { return tsmttsm_4_4_4_4<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M4_T4_lf", [&](int k) { return tsmttsm_4_4_4_4_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M4_T4_sg", [&](int k) { return tsmttsm_4_4_4_4_sg<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M4_T4_sg_lf", [&](int k) { return tsmttsm_4_4_4_4_sg_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
  }
  {
    tsm_compat::Problem<T> p(q, K, 8, 123, 1e-6);
    results.push_back(p.bench("M8_T2_basic", [&](int k) { return tsmttsm_8_8_2_2<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M8_T2_lf", [&](int k) { return tsmttsm_8_8_2_2_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M8_T2_sg", [&](int k) { return tsmttsm_8_8_2_2_sg<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M8_T2_sg_lf", [&](int k) { return tsmttsm_8_8_2_2_sg_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M8_T4_basic", [&](int k) { return tsmttsm_8_8_4_4<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M8_T4_lf", [&](int k) { return tsmttsm_8_8_4_4_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M8_T4_sg", [&](int k) { return tsmttsm_8_8_4_4_sg<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M8_T4_sg_lf", [&](int k) { return tsmttsm_8_8_4_4_sg_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
  }
  {
    tsm_compat::Problem<T> p(q, K, 16, 123, 1e-6);
    results.push_back(p.bench("M16_T2_basic", [&](int k) { return tsmttsm_16_16_2_2<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M16_T2_lf", [&](int k) { return tsmttsm_16_16_2_2_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M16_T2_sg", [&](int k) { return tsmttsm_16_16_2_2_sg<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M16_T2_sg_lf", [&](int k) { return tsmttsm_16_16_2_2_sg_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M16_T4_basic", [&](int k) { return tsmttsm_16_16_4_4<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M16_T4_lf", [&](int k) { return tsmttsm_16_16_4_4_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M16_T4_sg", [&](int k) { return tsmttsm_16_16_4_4_sg<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
    results.push_back(p.bench("M16_T4_sg_lf", [&](int k) { return tsmttsm_16_16_4_4_sg_lf<T>(q, k, p.A, p.B, p.C); }, warmup, runs));
  }
  tsm_compat::print_results(results);
}

// End of generated code
