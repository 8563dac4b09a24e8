/*
 * swehr_faces.cuh -- warp reductions shared by the step kernels, and the
 * block size of the allocation-free CFL kernel.
 */
#pragma once
#include "swehr_device.cuh"

namespace swehr {

#define NB_THREADS 256

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_down_sync(0xffffffffu, v, o);
        v = (w > v) ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace swehr
