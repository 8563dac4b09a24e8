/*
 * swehr_batch16_f32.cu -- the batched kernels of the mixed form built for
 * 16 x 16-cell tiles (see swehr_batch16_f64.cu).  The mixed form allows
 * fused multiply-adds, whose placement the compiler may choose differently
 * in this translation unit, so a mixed-form scenario can differ in the last
 * FP32 bits between the two shapes (the FP64 form cannot).
 */
#define SWEHR_TILE_I 16
#define SWEHR_TILE_J 16
#define SWEHR_TILE_NS t16x16
#include "swehr_launch.cuh"

namespace swehr {

int configure_batch_f32_t16(int max_classes, bool budget, BatchConfig &cfg)
{
    return FormLauncher<PolicyF32, float>::configure_batch(max_classes, budget, cfg);
}

}  // namespace swehr
