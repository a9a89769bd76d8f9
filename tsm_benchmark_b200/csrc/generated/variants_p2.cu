// Generated by tsm_benchmark_b200/codegen.py -- do not edit.
// Regenerate with: python -m tsm_benchmark_b200.codegen

#include "../tsm_registry.cuh"

namespace tsm {

extern const Variant kGenPart2[];
const Variant kGenPart2[] = {
    TSM_DMMA_VARIANT("dmma_16x48_t16x48_w8_s3_r128", 16, 48, 2, 6, 8, 3, 128),
    TSM_DMMA_VARIANT("dmma_48x48_t48x16_w9_s4_r72", 48, 48, 6, 2, 9, 4, 72),
    TSM_BULK_VARIANT("bulk_1x1_t1x1_w8_s6_r2048_u4", double, 1, 1, 1, 1, 8, 6, 2048, 4, true, false),
    TSM_BULK_VARIANT("bulk_2x2_t2x2_w8_s6_r1024_u1", double, 2, 2, 2, 2, 8, 6, 1024, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x4_t4x4_w8_s3_r1024_u1", double, 4, 4, 4, 4, 8, 3, 1024, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x16_t4x8_w8_s3_r256_u1", double, 4, 16, 4, 8, 8, 3, 256, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x4_t4x4_w8_s3_r512_u1", double, 8, 4, 4, 4, 8, 3, 512, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x8_t2x8_w8_s4_r384_u1", double, 8, 8, 2, 8, 8, 4, 384, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x16_t4x8_w8_s4_r192_u1", double, 8, 16, 4, 8, 8, 4, 192, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x4_t8x4_w8_s4_r128_u1", double, 16, 4, 8, 4, 8, 4, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x16_t4x8_w8_s6_r128_u1", double, 16, 16, 4, 8, 8, 6, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x4_t8x4_w8_s6_r64_u1", double, 32, 4, 8, 4, 8, 6, 64, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x16_t8x8_w8_s6_r64_u1", double, 32, 16, 8, 8, 8, 6, 64, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x32_t8x8_w8_s4_r96_u1", double, 32, 32, 8, 8, 8, 4, 96, 1, true, false),
    TSM_BULK_VARIANT("bulk_1x1_t1x1_w8_s6_r2048_u1_cap", double, 1, 1, 1, 1, 8, 6, 2048, 1, false, false),
    TSM_BULK_VARIANT("bulk_2x2_t2x2_w8_s6_r1024_u1_cap", double, 2, 2, 2, 2, 8, 6, 1024, 1, false, false),
    TSM_BULK_VARIANT("bulk_4x4_t4x4_w8_s6_r512_u1_cap", double, 4, 4, 4, 4, 8, 6, 512, 1, false, false),
    TSM_BULK_VARIANT("bulk_8x8_t4x4_w8_s6_r256_u1_cap", double, 8, 8, 4, 4, 8, 6, 256, 1, false, false),
    TSM_BULK_VARIANT("bulk_16x16_t8x8_w8_s6_r128_u1_cap", double, 16, 16, 8, 8, 8, 6, 128, 1, false, false),
    TSM_BULK_VARIANT("bulk_32x32_t8x8_w8_s6_r64_u1_cap", double, 32, 32, 8, 8, 8, 6, 64, 1, false, false),
    TSM_BULK_VARIANT("bulk_64x64_t8x8_w8_s6_r32_u1_cap", double, 64, 64, 8, 8, 8, 6, 32, 1, false, false),
    TSM_DIRECT_VARIANT("direct_2x1_t2x1_th256_cap", double, 2, 1, 2, 1, 256, false),
    TSM_DIRECT_VARIANT("direct_4x2_t4x2_th256_cap", double, 4, 2, 4, 2, 256, false),
    TSM_DIRECT_VARIANT("direct_8x4_t4x4_th256_cap", double, 8, 4, 4, 4, 256, false),
    TSM_DIRECT_VARIANT("direct_16x8_t8x4_th256_cap", double, 16, 8, 8, 4, 256, false),
    TSM_DIRECT_VARIANT("direct_32x16_t8x8_th256_cap", double, 32, 16, 8, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_64x32_t8x8_th256_cap", double, 64, 32, 8, 8, 256, false),
    TSM_BULK_VARIANT("bulkf32_64x64_t8x8_w8_s2_r192_u1", float, 64, 64, 8, 8, 8, 2, 192, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_1x1_t1x1_w8_s6_r4096_u1", float, 1, 1, 1, 1, 8, 6, 4096, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_1x2_t1x2_w8_s6_r2560_u1_cap", float, 1, 2, 1, 2, 8, 6, 2560, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_2x4_t2x4_w8_s6_r1280_u1_cap", float, 2, 4, 2, 4, 8, 6, 1280, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_4x8_t4x4_w8_s6_r640_u1_cap", float, 4, 8, 4, 4, 8, 6, 640, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_8x16_t4x8_w8_s6_r320_u1_cap", float, 8, 16, 4, 8, 8, 6, 320, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_16x32_t8x8_w8_s6_r160_u1_cap", float, 16, 32, 8, 8, 8, 6, 160, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_32x64_t8x8_w8_s6_r80_u1_cap", float, 32, 64, 8, 8, 8, 6, 80, 1, false, false),
    TSM_DIRECT_VARIANT("directf32_1x1_t1x1_th256_cap", float, 1, 1, 1, 1, 256, false),
    TSM_DIRECT_VARIANT("directf32_2x2_t2x2_th256_cap", float, 2, 2, 2, 2, 256, false),
    TSM_DIRECT_VARIANT("directf32_4x4_t4x4_th256_cap", float, 4, 4, 4, 4, 256, false),
    TSM_DIRECT_VARIANT("directf32_8x8_t4x4_th256_cap", float, 8, 8, 4, 4, 256, false),
    TSM_DIRECT_VARIANT("directf32_16x16_t8x8_th256_cap", float, 16, 16, 8, 8, 256, false),
    TSM_DIRECT_VARIANT("directf32_32x32_t8x8_th256_cap", float, 32, 32, 8, 8, 256, false),
    TSM_DIRECT_VARIANT("directf32_64x64_t8x8_th256_cap", float, 64, 64, 8, 8, 256, false),
    TSM_BULK_VARIANT("bulk_8x8_t4x4_w8_s2_r1536_u1_gram", double, 8, 8, 4, 4, 8, 2, 1536, 1, true, true),
    TSM_BULK_VARIANT("bulk_8x8_t4x4_w8_s6_r512_u1_gram", double, 8, 8, 4, 4, 8, 6, 512, 1, true, true),
    TSM_GRAM_DMMA_VARIANT("dmma_16x16_gram_w8_s2_r768", 16, 8, 2, 768),
    TSM_GRAM_DMMA_VARIANT("dmma_48x48_gram_w8_s2_r256", 48, 8, 2, 256),
};
extern const int kGenPart2Count;
const int kGenPart2Count = 46;

}  // namespace tsm
