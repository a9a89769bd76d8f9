// Generated by tsm_benchmark_b200/codegen.py -- do not edit.
// Regenerate with: python -m tsm_benchmark_b200.codegen

#include "../tsm_registry.cuh"

namespace tsm {

extern const Variant kGenPart6[];
const Variant kGenPart6[] = {
    TSM_DMMA_VARIANT("dmma_32x48_t16x48_w8_s3_r96", 32, 48, 2, 6, 8, 3, 96),
    TSM_DMMA_VARIANT("dmma_64x48_t64x16_w9_s3_r72", 64, 48, 8, 2, 9, 3, 72),
    TSM_BULK_VARIANT("bulk_1x64_t1x8_w8_s3_r64_u1", double, 1, 64, 1, 8, 8, 3, 64, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x4_t4x4_w8_s6_r512_u2", double, 4, 4, 4, 4, 8, 6, 512, 2, true, false),
    TSM_BULK_VARIANT("bulk_4x16_t4x8_w8_s4_r128_u1", double, 4, 16, 4, 8, 8, 4, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x8_t8x8_w8_s6_r256_u1", double, 8, 8, 8, 8, 8, 6, 256, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x16_t4x8_w8_s6_r128_u1", double, 8, 16, 4, 8, 8, 6, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x4_t8x4_w8_s4_r128_u1", double, 16, 4, 8, 4, 8, 4, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x16_t8x8_w8_s4_r192_u1", double, 16, 16, 8, 8, 8, 4, 192, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x8_t8x4_w8_s3_r192_u1", double, 32, 8, 8, 4, 8, 3, 192, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x32_t8x8_w8_s3_r128_u1", double, 32, 32, 8, 8, 8, 3, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_1x2_t1x2_w8_s6_r1280_u1_cap", double, 1, 2, 1, 2, 8, 6, 1280, 1, false, false),
    TSM_BULK_VARIANT("bulk_2x4_t2x4_w8_s6_r512_u1_cap", double, 2, 4, 2, 4, 8, 6, 512, 1, false, false),
    TSM_BULK_VARIANT("bulk_4x8_t4x4_w8_s6_r256_u1_cap", double, 4, 8, 4, 4, 8, 6, 256, 1, false, false),
    TSM_BULK_VARIANT("bulk_8x16_t4x8_w8_s6_r128_u1_cap", double, 8, 16, 4, 8, 8, 6, 128, 1, false, false),
    TSM_BULK_VARIANT("bulk_16x32_t8x8_w8_s6_r64_u1_cap", double, 16, 32, 8, 8, 8, 6, 64, 1, false, false),
    TSM_BULK_VARIANT("bulk_32x64_t8x8_w8_s6_r40_u1_cap", double, 32, 64, 8, 8, 8, 6, 40, 1, false, false),
    TSM_DIRECT_VARIANT("direct_1x1_t1x1_th256_cap", double, 1, 1, 1, 1, 256, false),
    TSM_DIRECT_VARIANT("direct_2x2_t2x2_th256_cap", double, 2, 2, 2, 2, 256, false),
    TSM_DIRECT_VARIANT("direct_4x4_t4x4_th256_cap", double, 4, 4, 4, 4, 256, false),
    TSM_DIRECT_VARIANT("direct_8x8_t4x4_th256_cap", double, 8, 8, 4, 4, 256, false),
    TSM_DIRECT_VARIANT("direct_16x16_t8x8_th256_cap", double, 16, 16, 8, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_32x32_t8x8_th256_cap", double, 32, 32, 8, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_64x64_t8x8_th256_cap", double, 64, 64, 8, 8, 256, false),
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
    TSM_BULK_VARIANT("bulk_8x8_t4x4_w8_s3_r1024_u1_gram", double, 8, 8, 4, 4, 8, 3, 1024, 1, true, true),
    TSM_DMMA_VARIANT("dmma_32x32_t32x32_w8_s2_r192", 32, 32, 4, 4, 8, 2, 192),
};
extern const int kGenPart6Count;
const int kGenPart6Count = 40;

}  // namespace tsm
