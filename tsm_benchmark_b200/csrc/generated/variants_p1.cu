// Generated by tsm_benchmark_b200/codegen.py -- do not edit.
// Regenerate with: python -m tsm_benchmark_b200.codegen

#include "../tsm_registry.cuh"

namespace tsm {

extern const Variant kGenPart1[];
const Variant kGenPart1[] = {
    TSM_DMMA_VARIANT("dmma_16x32_t16x32_w8_s3_r160", 16, 32, 2, 4, 8, 3, 160),
    TSM_DMMA_VARIANT("dmma_48x32_t48x16_w8_s3_r96", 48, 32, 6, 2, 8, 3, 96),
    TSM_BULK_VARIANT("bulk_1x1_t1x1_w8_s6_r2048_u2", double, 1, 1, 1, 1, 8, 6, 2048, 2, true, false),
    TSM_BULK_VARIANT("bulk_1x64_t1x8_w8_s2_r96_u1", double, 1, 64, 1, 8, 8, 2, 96, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x4_t4x4_w8_s6_r512_u2", double, 4, 4, 4, 4, 8, 6, 512, 2, true, false),
    TSM_BULK_VARIANT("bulk_4x16_t4x8_w8_s6_r128_u1", double, 4, 16, 4, 8, 8, 6, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x4_t4x4_w8_s6_r256_u1", double, 8, 4, 4, 4, 8, 6, 256, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x8_t2x8_w8_s3_r512_u1", double, 8, 8, 2, 8, 8, 3, 512, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x16_t4x8_w8_s3_r256_u1", double, 8, 16, 4, 8, 8, 3, 256, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x4_t8x4_w8_s3_r256_u1", double, 16, 4, 8, 4, 8, 3, 256, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x16_t4x4_w8_s6_r128_u1", double, 16, 16, 4, 4, 8, 6, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x32_t8x8_w8_s2_r192_u1", double, 16, 32, 8, 8, 8, 2, 192, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x8_t8x4_w8_s2_r288_u1", double, 32, 8, 8, 4, 8, 2, 288, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x32_t8x8_w8_s3_r128_u1", double, 32, 32, 8, 8, 8, 3, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_64x64_t8x8_w8_s2_r96_u1", double, 64, 64, 8, 8, 8, 2, 96, 1, true, false),
    TSM_BULK_VARIANT("bulk_2x1_t2x1_w8_s6_r1280_u1_cap", double, 2, 1, 2, 1, 8, 6, 1280, 1, false, false),
    TSM_BULK_VARIANT("bulk_4x2_t4x2_w8_s6_r512_u1_cap", double, 4, 2, 4, 2, 8, 6, 512, 1, false, false),
    TSM_BULK_VARIANT("bulk_8x4_t4x4_w8_s6_r256_u1_cap", double, 8, 4, 4, 4, 8, 6, 256, 1, false, false),
    TSM_BULK_VARIANT("bulk_16x8_t8x4_w8_s6_r128_u1_cap", double, 16, 8, 8, 4, 8, 6, 128, 1, false, false),
    TSM_BULK_VARIANT("bulk_32x16_t8x8_w8_s6_r64_u1_cap", double, 32, 16, 8, 8, 8, 6, 64, 1, false, false),
    TSM_BULK_VARIANT("bulk_64x32_t8x8_w8_s6_r40_u1_cap", double, 64, 32, 8, 8, 8, 6, 40, 1, false, false),
    TSM_DIRECT_VARIANT("direct_1x64_t1x8_th256_cap", double, 1, 64, 1, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_4x1_t4x1_th256_cap", double, 4, 1, 4, 1, 256, false),
    TSM_DIRECT_VARIANT("direct_8x2_t4x2_th256_cap", double, 8, 2, 4, 2, 256, false),
    TSM_DIRECT_VARIANT("direct_16x4_t8x4_th256_cap", double, 16, 4, 8, 4, 256, false),
    TSM_DIRECT_VARIANT("direct_32x8_t8x4_th256_cap", double, 32, 8, 8, 4, 256, false),
    TSM_DIRECT_VARIANT("direct_64x16_t8x8_th256_cap", double, 64, 16, 8, 8, 256, false),
    TSM_BULK_VARIANT("bulkf32_32x32_t8x8_w8_s2_r384_u1", float, 32, 32, 8, 8, 8, 2, 384, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_64x64_t8x8_w8_s3_r128_u1", float, 64, 64, 8, 8, 8, 3, 128, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_1x1_t1x1_w8_s6_r4096_u1_cap", float, 1, 1, 1, 1, 8, 6, 4096, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_2x2_t2x2_w8_s6_r2048_u1_cap", float, 2, 2, 2, 2, 8, 6, 2048, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_4x4_t4x4_w8_s6_r1024_u1_cap", float, 4, 4, 4, 4, 8, 6, 1024, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_8x8_t4x4_w8_s6_r512_u1_cap", float, 8, 8, 4, 4, 8, 6, 512, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_16x16_t8x8_w8_s6_r256_u1_cap", float, 16, 16, 8, 8, 8, 6, 256, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_32x32_t8x8_w8_s6_r128_u1_cap", float, 32, 32, 8, 8, 8, 6, 128, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_64x64_t8x8_w8_s6_r64_u1_cap", float, 64, 64, 8, 8, 8, 6, 64, 1, false, false),
    TSM_DIRECT_VARIANT("directf32_2x1_t2x1_th256_cap", float, 2, 1, 2, 1, 256, false),
    TSM_DIRECT_VARIANT("directf32_4x2_t4x2_th256_cap", float, 4, 2, 4, 2, 256, false),
    TSM_DIRECT_VARIANT("directf32_8x4_t4x4_th256_cap", float, 8, 4, 4, 4, 256, false),
    TSM_DIRECT_VARIANT("directf32_16x8_t8x4_th256_cap", float, 16, 8, 8, 4, 256, false),
    TSM_DIRECT_VARIANT("directf32_32x16_t8x8_th256_cap", float, 32, 16, 8, 8, 256, false),
    TSM_DIRECT_VARIANT("directf32_64x32_t8x8_th256_cap", float, 64, 32, 8, 8, 256, false),
    TSM_BULK_VARIANT("bulk_4x4_t4x4_w8_s2_r3072_u1_gram", double, 4, 4, 4, 4, 8, 2, 3072, 1, true, true),
    TSM_BULK_VARIANT("bulk_4x4_t4x4_w8_s6_r1024_u1_gram", double, 4, 4, 4, 4, 8, 6, 1024, 1, true, true),
    TSM_DMMA_VARIANT("dmma_16x16_t16x16_w8_s3_r288", 16, 16, 2, 2, 8, 3, 288),
    TSM_GRAM_DMMA_VARIANT("dmma_32x32_gram_w12_s2_r384", 32, 12, 2, 384),
};
extern const int kGenPart1Count;
const int kGenPart1Count = 46;

}  // namespace tsm
