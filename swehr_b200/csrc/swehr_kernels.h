/* swehr_kernels.h -- host-visible launch entry points of the step kernels. */
#pragma once
#include <cuda_runtime.h>

#include "swehr_device.cuh"

namespace swehr {

/* device buffers of one simulation: two state sets (9 + 2S planes each),
 * three topography planes, optional per-cell Ks */
struct Bufs {
    double *set[2];
    double *z[3];
    const double *ks;
};

/* launch geometry of the step kernels of one simulation */
struct StepConfig {
    int grid_wave = 1, grid_update = 1;
    size_t smem_wave = 0, smem_update = 0;
    void *fn_update = nullptr;
};

/* Pick the kernel instantiation, set its shared-memory limit and size the
 * persistent grids from the occupancy (returns a cudaError_t). */
int configure_step_f64(const DevParams &P, int num_sms, StepConfig &cfg);

/* Enqueue one full step (wave pass + update pass) of the FP64 form.
 * ev0/ev1 (optional) are recorded around the update kernel. */
int launch_step_f64(const DevParams &P, const Bufs &B, Ctl *ctl, const double *rain, double *partials,
                    double *stage, double *saveflow, const StepConfig &cfg, cudaStream_t s, cudaEvent_t ev0,
                    cudaEvent_t ev1);

}  // namespace swehr
