// compat_templates.cc -- instantiates every reference entry point of the
// compat headers against libtsm_b200.so and prints each one's C, for
// tests/test_dropin_gpu.py to compare with the reference's own outputs
// (tests/golden/ref_variants.npz).
//
//   the nine templates of tsmttsm.hh (tsmttsm.hh:15-586), with the launch
//   parameters the golden outputs were made with (M = 8, stride 4096,
//   local_size 32, tile 4; tsmttsm8 with its default worker_mult), and the
//   kernels the two generators emit by default for M = 8 (v2:
//   tsmttsm_8_8_{2,4}_{2,4}{,_lf,_sg,_sg_lf}; v1:
//   tsmttsm_gen_8_8_4_4{,_lf}{,_2l}_tr), from headers the generator wrote
//   without their benchmark harness.
//
// Inputs: n = 4099 rows, A and B from the library's counter-based generator
// under seed 7 (streams 0 and 1), the values the golden outputs used.
// Output: one line per entry point, "name c_00 c_01 ... c_77" (%.17g).
#include <sycl/sycl.hpp>

#include <cstdio>
#include <vector>

#include "tsmttsm.hh"
#include "v1_kernels.hh"
#include "v2_kernels.hh"

namespace {

constexpr int kM = 8;
constexpr int kRows = 4099;
constexpr int kStride = 4096, kLocal = 32, kTile = 4;

template <class F>
void run(sycl::queue& q, const char* name, double* C, F&& f) {
  q.fill(C, 0.0, kM * kM).wait();
  f().wait();
  std::vector<double> h(kM * kM);
  q.memcpy(h.data(), C, h.size() * sizeof(double)).wait();
  std::printf("%s", name);
  for (double x : h) std::printf(" %.17g", x);
  std::printf("\n");
}

}  // namespace

int main() {
  sycl::queue q{{sycl::property::queue::in_order{}, sycl::property::queue::enable_profiling{}}};
  double* A = sycl::malloc_device<double>(kRows * kM, q);
  double* B = sycl::malloc_device<double>(kRows * kM, q);
  double* C = sycl::malloc_device<double>(kM * kM, q);
  if (tsm_fill_uniform_f64(q.native_stream(), A, kRows * kM, 7, 0) != TSM_SUCCESS ||
      tsm_fill_uniform_f64(q.native_stream(), B, kRows * kM, 7, 1) != TSM_SUCCESS)
    return 2;
  const int K = kRows;
  run(q, "tsmttsm", C, [&] { return tsmttsm<double, kM, kStride>(q, K, A, B, C); });
  run(q, "tsmttsm2", C, [&] { return tsmttsm2<double, kM, kStride, kTile>(q, K, A, B, C); });
  run(q, "tsmttsm3", C, [&] { return tsmttsm3<double, kM, kStride, kTile>(q, K, A, B, C); });
  run(q, "tsmttsm4", C, [&] { return tsmttsm4<double, kM, kStride, kTile>(q, K, A, B, C); });
  run(q, "tsmttsm5", C, [&] { return tsmttsm5<double, kM, kStride, kTile>(q, K, A, B, C); });
  run(q, "tsmttsm6", C, [&] { return tsmttsm6<double, kM, kStride, kLocal, kTile>(q, K, A, B, C); });
  run(q, "tsmttsm7", C, [&] { return tsmttsm7<double, kM, kStride, kTile>(q, K, A, B, C); });
  run(q, "tsmttsm8", C, [&] { return tsmttsm8<double, kM>(q, K, A, B, C); });
  run(q, "tsmttsm9", C, [&] { return tsmttsm9<double, kM, kStride, kLocal, kTile>(q, K, A, B, C); });
#define GEN(name) run(q, #name, C, [&] { return name<double>(q, K, A, B, C); })
  GEN(tsmttsm_8_8_4_4);
  GEN(tsmttsm_8_8_4_4_lf);
  GEN(tsmttsm_8_8_4_4_sg);
  GEN(tsmttsm_8_8_4_4_sg_lf);
  GEN(tsmttsm_8_8_2_2);
  GEN(tsmttsm_8_8_2_2_lf);
  GEN(tsmttsm_8_8_2_2_sg);
  GEN(tsmttsm_8_8_2_2_sg_lf);
  GEN(tsmttsm_gen_8_8_4_4_tr);
  GEN(tsmttsm_gen_8_8_4_4_lf_tr);
  GEN(tsmttsm_gen_8_8_4_4_2l_tr);
  GEN(tsmttsm_gen_8_8_4_4_lf_2l_tr);
#undef GEN
  sycl::free(A, q);
  sycl::free(B, q);
  sycl::free(C, q);
  return 0;
}
