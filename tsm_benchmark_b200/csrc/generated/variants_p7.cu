// Generated by tsm_benchmark_b200/codegen.py -- do not edit.
// Regenerate with: python -m tsm_benchmark_b200.codegen

#include "../tsm_registry.cuh"

namespace tsm {

extern const Variant kGenPart7[];
const Variant kGenPart7[] = {
    TSM_DMMA_VARIANT("dmma_32x64_t32x32_w8_s3_r80", 32, 64, 4, 4, 8, 3, 80),
    TSM_DMMA_VARIANT("dmma_64x64_t32x32_w8_s3_r64", 64, 64, 4, 4, 8, 3, 64),
    TSM_BULK_VARIANT("bulk_1x64_t1x8_w8_s3_r64_u1", double, 1, 64, 1, 8, 8, 3, 64, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x4_t4x4_w8_s6_r512_u1", double, 4, 4, 4, 4, 8, 6, 512, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x8_t4x4_w8_s4_r384_u1", double, 4, 8, 4, 4, 8, 4, 384, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x32_t4x8_w8_s4_r64_u1", double, 4, 32, 4, 8, 8, 4, 64, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x8_t4x4_w8_s6_r256_u2", double, 8, 8, 4, 4, 8, 6, 256, 2, true, false),
    TSM_BULK_VARIANT("bulk_8x8_t4x4_w8_s2_r768_u1", double, 8, 8, 4, 4, 8, 2, 768, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x32_t4x8_w8_s2_r288_u1", double, 8, 32, 4, 8, 8, 2, 288, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x8_t8x4_w8_s2_r384_u1", double, 16, 8, 8, 4, 8, 2, 384, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x32_t8x8_w8_s3_r128_u1", double, 16, 32, 8, 8, 8, 3, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x8_t8x4_w8_s3_r192_u1", double, 32, 8, 8, 4, 8, 3, 192, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x32_t8x4_w8_s6_r64_u1", double, 32, 32, 8, 4, 8, 6, 64, 1, true, false),
    TSM_BULK_VARIANT("bulk_64x64_t8x8_w8_s3_r64_u1", double, 64, 64, 8, 8, 8, 3, 64, 1, true, false),
    TSM_BULK_VARIANT("bulk_1x32_t1x8_w8_s6_r64_u1_cap", double, 1, 32, 1, 8, 8, 6, 64, 1, false, false),
    TSM_BULK_VARIANT("bulk_2x64_t2x8_w8_s6_r32_u1_cap", double, 2, 64, 2, 8, 8, 6, 32, 1, false, false),
    TSM_BULK_VARIANT("bulk_8x1_t4x1_w8_s6_r384_u1_cap", double, 8, 1, 4, 1, 8, 6, 384, 1, false, false),
    TSM_BULK_VARIANT("bulk_16x2_t8x2_w8_s6_r128_u1_cap", double, 16, 2, 8, 2, 8, 6, 128, 1, false, false),
    TSM_BULK_VARIANT("bulk_32x4_t8x4_w8_s6_r64_u1_cap", double, 32, 4, 8, 4, 8, 6, 64, 1, false, false),
    TSM_BULK_VARIANT("bulk_64x8_t8x4_w8_s6_r48_u1_cap", double, 64, 8, 8, 4, 8, 6, 48, 1, false, false),
    TSM_DIRECT_VARIANT("direct_1x16_t1x8_th256_cap", double, 1, 16, 1, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_2x32_t2x8_th256_cap", double, 2, 32, 2, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_4x64_t4x8_th256_cap", double, 4, 64, 4, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_16x1_t8x1_th256_cap", double, 16, 1, 8, 1, 256, false),
    TSM_DIRECT_VARIANT("direct_32x2_t8x2_th256_cap", double, 32, 2, 8, 2, 256, false),
    TSM_DIRECT_VARIANT("direct_64x4_t8x4_th256_cap", double, 64, 4, 8, 4, 256, false),
    TSM_BULK_VARIANT("bulkf32_8x8_t4x4_w8_s2_r1536_u1", float, 8, 8, 4, 4, 8, 2, 1536, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_16x16_t8x8_w8_s3_r512_u1", float, 16, 16, 8, 8, 8, 3, 512, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_32x32_t8x8_w8_s6_r128_u1", float, 32, 32, 8, 8, 8, 6, 128, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_1x64_t1x8_w8_s6_r96_u1_cap", float, 1, 64, 1, 8, 8, 6, 96, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_4x1_t4x1_w8_s6_r1536_u1_cap", float, 4, 1, 4, 1, 8, 6, 1536, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_8x2_t4x2_w8_s6_r768_u1_cap", float, 8, 2, 4, 2, 8, 6, 768, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_16x4_t8x4_w8_s6_r384_u1_cap", float, 16, 4, 8, 4, 8, 6, 384, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_32x8_t8x4_w8_s6_r192_u1_cap", float, 32, 8, 8, 4, 8, 6, 192, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_64x16_t8x8_w8_s6_r96_u1_cap", float, 64, 16, 8, 8, 8, 6, 96, 1, false, false),
    TSM_DIRECT_VARIANT("directf32_1x32_t1x8_th256_cap", float, 1, 32, 1, 8, 256, false),
    TSM_DIRECT_VARIANT("directf32_2x64_t2x8_th256_cap", float, 2, 64, 2, 8, 256, false),
    TSM_DIRECT_VARIANT("directf32_8x1_t4x1_th256_cap", float, 8, 1, 4, 1, 256, false),
    TSM_DIRECT_VARIANT("directf32_16x2_t8x2_th256_cap", float, 16, 2, 8, 2, 256, false),
    TSM_DIRECT_VARIANT("directf32_32x4_t8x4_th256_cap", float, 32, 4, 8, 4, 256, false),
    TSM_DIRECT_VARIANT("directf32_64x8_t8x4_th256_cap", float, 64, 8, 8, 4, 256, false),
    TSM_BULK_VARIANT("bulk_1x1_t1x1_w8_s2_r12288_u1_gram", double, 1, 1, 1, 1, 8, 2, 12288, 1, true, true),
    TSM_BULK_VARIANT("bulk_1x1_t1x1_w8_s6_r4096_u1_gram", double, 1, 1, 1, 1, 8, 6, 4096, 1, true, true),
    TSM_DMMA_VARIANT("dmma_32x32_t32x32_w8_s6_r64", 32, 32, 4, 4, 8, 6, 64),
    TSM_DMMA_VARIANT("dmma_64x64_t32x32_w12_s2_r96", 64, 64, 4, 4, 12, 2, 96),
};
extern const int kGenPart7Count;
const int kGenPart7Count = 45;

}  // namespace tsm
