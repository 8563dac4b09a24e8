/*
 * swehr_batch16_f64.cu -- the batched kernels of the plain FP64 form built
 * for 16 x 16-cell tiles (the default build, swehr_step_f64.cu, uses 8 x 32).
 * The pool's tuner times both shapes on its own scenarios: square tiles
 * carry less halo per cell (18 x 18 staged for 256 cells against 10 x 34)
 * and waste fewer lanes at the j edge of narrow scenarios.  Compiled with
 * --fmad=false like every FP64 kernel, so results do not depend on the shape.
 */
#define SWEHR_TILE_I 16
#define SWEHR_TILE_J 16
#define SWEHR_TILE_NS t16x16
#include "swehr_launch.cuh"

namespace swehr {

int configure_batch_f64_t16(int max_classes, bool budget, BatchConfig &cfg)
{
    return FormLauncher<PolicyF64, double>::configure_batch(max_classes, budget, cfg);
}

}  // namespace swehr
