// Generated by tsm_benchmark_b200/codegen.py -- do not edit.
// Regenerate with: python -m tsm_benchmark_b200.codegen

#include "../tsm_registry.cuh"

namespace tsm {

extern const Variant kGenPart4[];
const Variant kGenPart4[] = {
    TSM_DMMA_VARIANT("dmma_32x16_t32x16_w8_s3_r160", 32, 16, 4, 2, 8, 3, 160),
    TSM_DMMA_VARIANT("dmma_64x16_t64x16_w8_s3_r96", 64, 16, 8, 2, 8, 3, 96),
    TSM_BULK_VARIANT("bulk_1x1_t1x1_w8_s4_r3072_u1", double, 1, 1, 1, 1, 8, 4, 3072, 1, true, false),
    TSM_BULK_VARIANT("bulk_2x2_t2x2_w8_s3_r2048_u1", double, 2, 2, 2, 2, 8, 3, 2048, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x4_t4x4_w8_s2_r1536_u1", double, 4, 4, 4, 4, 8, 2, 1536, 1, true, false),
    TSM_BULK_VARIANT("bulk_4x16_t4x8_w8_s2_r384_u1", double, 4, 16, 4, 8, 8, 2, 384, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x4_t4x4_w8_s2_r768_u1", double, 8, 4, 4, 4, 8, 2, 768, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x8_t2x8_w8_s2_r768_u1", double, 8, 8, 2, 8, 8, 2, 768, 1, true, false),
    TSM_BULK_VARIANT("bulk_8x32_t4x8_w8_s6_r96_u1", double, 8, 32, 4, 8, 8, 6, 96, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x8_t8x4_w8_s6_r128_u1", double, 16, 8, 8, 4, 8, 6, 128, 1, true, false),
    TSM_BULK_VARIANT("bulk_16x16_t8x8_w8_s4_r192_u1", double, 16, 16, 8, 8, 8, 4, 192, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x4_t8x4_w8_s4_r64_u1", double, 32, 4, 8, 4, 8, 4, 64, 1, true, false),
    TSM_BULK_VARIANT("bulk_32x16_t8x8_w8_s4_r96_u1", double, 32, 16, 8, 8, 8, 4, 96, 1, true, false),
    TSM_BULK_VARIANT("bulk_64x64_t8x8_w8_s6_r32_u1", double, 64, 64, 8, 8, 8, 6, 32, 1, true, false),
    TSM_BULK_VARIANT("bulk_1x4_t1x4_w8_s6_r768_u1_cap", double, 1, 4, 1, 4, 8, 6, 768, 1, false, false),
    TSM_BULK_VARIANT("bulk_2x8_t2x4_w8_s6_r384_u1_cap", double, 2, 8, 2, 4, 8, 6, 384, 1, false, false),
    TSM_BULK_VARIANT("bulk_4x16_t4x8_w8_s6_r128_u1_cap", double, 4, 16, 4, 8, 8, 6, 128, 1, false, false),
    TSM_BULK_VARIANT("bulk_8x32_t4x8_w8_s6_r96_u1_cap", double, 8, 32, 4, 8, 8, 6, 96, 1, false, false),
    TSM_BULK_VARIANT("bulk_16x64_t8x8_w8_s6_r48_u1_cap", double, 16, 64, 8, 8, 8, 6, 48, 1, false, false),
    TSM_BULK_VARIANT("bulk_64x1_t8x1_w8_s6_r32_u1_cap", double, 64, 1, 8, 1, 8, 6, 32, 1, false, false),
    TSM_DIRECT_VARIANT("direct_1x2_t1x2_th256_cap", double, 1, 2, 1, 2, 256, false),
    TSM_DIRECT_VARIANT("direct_2x4_t2x4_th256_cap", double, 2, 4, 2, 4, 256, false),
    TSM_DIRECT_VARIANT("direct_4x8_t4x4_th256_cap", double, 4, 8, 4, 4, 256, false),
    TSM_DIRECT_VARIANT("direct_8x16_t4x8_th256_cap", double, 8, 16, 4, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_16x32_t8x8_th256_cap", double, 16, 32, 8, 8, 256, false),
    TSM_DIRECT_VARIANT("direct_32x64_t8x8_th256_cap", double, 32, 64, 8, 8, 256, false),
    TSM_BULK_VARIANT("bulkf32_1x1_t1x1_w8_s2_r12288_u1", float, 1, 1, 1, 1, 8, 2, 12288, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_2x2_t2x2_w8_s3_r4096_u1", float, 2, 2, 2, 2, 8, 3, 4096, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_4x4_t4x4_w8_s6_r1024_u1", float, 4, 4, 4, 4, 8, 6, 1024, 1, true, false),
    TSM_BULK_VARIANT("bulkf32_1x8_t1x4_w8_s6_r896_u1_cap", float, 1, 8, 1, 4, 8, 6, 896, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_2x16_t2x8_w8_s6_r384_u1_cap", float, 2, 16, 2, 8, 8, 6, 384, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_4x32_t4x8_w8_s6_r192_u1_cap", float, 4, 32, 4, 8, 8, 6, 192, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_8x64_t4x8_w8_s6_r112_u1_cap", float, 8, 64, 4, 8, 8, 6, 112, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_32x1_t8x1_w8_s6_r192_u1_cap", float, 32, 1, 8, 1, 8, 6, 192, 1, false, false),
    TSM_BULK_VARIANT("bulkf32_64x2_t8x2_w8_s6_r96_u1_cap", float, 64, 2, 8, 2, 8, 6, 96, 1, false, false),
    TSM_DIRECT_VARIANT("directf32_1x4_t1x4_th256_cap", float, 1, 4, 1, 4, 256, false),
    TSM_DIRECT_VARIANT("directf32_2x8_t2x4_th256_cap", float, 2, 8, 2, 4, 256, false),
    TSM_DIRECT_VARIANT("directf32_4x16_t4x8_th256_cap", float, 4, 16, 4, 8, 256, false),
    TSM_DIRECT_VARIANT("directf32_8x32_t4x8_th256_cap", float, 8, 32, 4, 8, 256, false),
    TSM_DIRECT_VARIANT("directf32_16x64_t8x8_th256_cap", float, 16, 64, 8, 8, 256, false),
    TSM_DIRECT_VARIANT("directf32_64x1_t8x1_th256_cap", float, 64, 1, 8, 1, 256, false),
    TSM_GRAM_DMMA_VARIANT("dmma_32x32_gram_w8_s3_r256", 32, 8, 3, 256),
    TSM_BULK_VARIANT("bulk_2x2_t2x2_w8_s3_r4096_u1_gram", double, 2, 2, 2, 2, 8, 3, 4096, 1, true, true),
    TSM_DMMA_VARIANT("dmma_16x16_t16x16_w8_s6_r128", 16, 16, 2, 2, 8, 6, 128),
    TSM_DMMA_VARIANT("dmma_64x64_t32x32_w8_s2_r96", 64, 64, 4, 4, 8, 2, 96),
    TSM_GRAM_DMMA_VARIANT("dmma_48x48_gram_w12_s2_r240", 48, 12, 2, 240),
};
extern const int kGenPart4Count;
const int kGenPart4Count = 46;

}  // namespace tsm
