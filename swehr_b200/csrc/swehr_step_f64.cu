/*
 * swehr_step_f64.cu -- the plain FP64 form of one SWEHR time step on sm_100a.
 * Compiled with --fmad=false: no contraction, so every cell is bit-identical
 * to the CPU restatement built with the project's math.
 *
 * A step is two stream-ordered launches and needs no grid barrier:
 *   k_wave_tile   largest wave speed over every face (SWEHR.c:1092-1230's
 *                 Smax); the last block to finish computes dt and the Courant
 *                 check (SWEHR.c:1409-1413) and arms the update;
 *   k_update_tile fluxes, sources and the update of every cell (SWEHR.c:
 *                 1233-1588), reading state set n%2 and writing set (n+1)%2;
 *                 the last block sums the budget partials, advances t and the
 *                 step counter, records a stage row when one is due
 *                 (SWEHR.c:1593-1676) and disarms stepping at t >= tend,
 *                 t_stop, the step limit or a CFL error.
 * Both kernels read the step counter from the control block to pick their
 * buffers, so every step is the same pair of launches and a chunk of steps
 * is captured once as a CUDA graph.  Nothing spins or waits on the device.
 */
#include <cuda_runtime.h>

#include "swehr_kernels.h"
#include "swehr_tile.cuh"

namespace swehr {

static size_t update_smem(int S) { return (size_t)TileLayout::make(S).total * sizeof(double); }
static size_t wave_smem() { return (size_t)5 * N_H * sizeof(double); }

template <int MAXS, bool BUDGET>
static void *update_fn() { return (void *)k_update_tile<MAXS, BUDGET>; }

static void *pick_update(int S, bool budget)
{
    if (S <= 4) return budget ? update_fn<4, true>() : update_fn<4, false>();
    if (S <= 8) return budget ? update_fn<8, true>() : update_fn<8, false>();
    return budget ? update_fn<16, true>() : update_fn<16, false>();
}

int configure_step_f64(const DevParams &P, int num_sms, StepConfig &cfg)
{
    const int64_t ntiles = (int64_t)((P.nx + T_I - 1) / T_I) * ((P.ny + T_J - 1) / T_J);
    void *fu = pick_update(P.S, P.budget != 0);
    const size_t su = update_smem(P.S);
    cudaError_t e = cudaFuncSetAttribute(fu, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)su);
    if (e != cudaSuccess) return (int)e;
    int occ_u = 0, occ_w = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_u, fu, TILE_THREADS, su);
    if (e != cudaSuccess) return (int)e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_w, (void *)k_wave_tile, TILE_THREADS, wave_smem());
    if (e != cudaSuccess) return (int)e;
    if (occ_u < 1) occ_u = 1;
    if (occ_w < 1) occ_w = 1;
    cfg.grid_update = (int)(ntiles < (int64_t)num_sms * occ_u ? ntiles : (int64_t)num_sms * occ_u);
    cfg.grid_wave = (int)(ntiles < (int64_t)num_sms * occ_w ? ntiles : (int64_t)num_sms * occ_w);
    cfg.smem_update = su;
    cfg.smem_wave = wave_smem();
    cfg.fn_update = fu;
    return 0;
}

int launch_step_f64(const DevParams &P, const Bufs &B, Ctl *ctl, const double *rain, double *partials,
                    double *stage, double *saveflow, const StepConfig &cfg, cudaStream_t s, cudaEvent_t ev0,
                    cudaEvent_t ev1)
{
    k_wave_tile<<<cfg.grid_wave, TILE_THREADS, cfg.smem_wave, s>>>(P, B, ctl);
    if (ev0) cudaEventRecord(ev0, s);
    void *args[] = {(void *)&P, (void *)&B, (void *)&ctl, (void *)&rain, (void *)&partials, (void *)&stage,
                    (void *)&saveflow};
    cudaLaunchKernel(cfg.fn_update, dim3(cfg.grid_update), dim3(TILE_THREADS), args, cfg.smem_update, s);
    if (ev1) cudaEventRecord(ev1, s);
    return (int)cudaGetLastError();
}

}  // namespace swehr
