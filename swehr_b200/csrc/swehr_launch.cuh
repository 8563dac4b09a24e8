/*
 * swehr_launch.cuh -- launch geometry and enqueueing of the two step kernels
 * of one form (included once per form, by swehr_step_f64.cu and
 * swehr_step_f32.cu, which are compiled with different contraction flags).
 */
#pragma once
#include <cuda_runtime.h>

#include "swehr_kernels.h"
#include "swehr_tile.cuh"

namespace swehr {

template <class PP, class RS>
struct FormLauncher {
    typedef typename PP::R R;

    static size_t update_smem(int S) { return StagedLayout::make(S, sizeof(R), 1).total; }
    static size_t wave_smem() { return StagedLayout::make(0, sizeof(R), 0).total; }

    template <int MAXS, bool BUDGET>
    static void *update_fn() { return (void *)k_update_tile<PP, RS, MAXS, BUDGET>; }

    static void *pick_update(int S, bool budget)
    {
        if (S <= 4) return budget ? update_fn<4, true>() : update_fn<4, false>();
        if (S <= 8) return budget ? update_fn<8, true>() : update_fn<8, false>();
        return budget ? update_fn<16, true>() : update_fn<16, false>();
    }

    static int configure(const DevParams &P, int num_sms, StepConfig &cfg)
    {
        const int64_t ntiles = (int64_t)((P.nx + T_I - 1) / T_I) * ((P.ny + T_J - 1) / T_J);
        void *fu = pick_update(P.S, P.budget != 0);
        void *fw = (void *)k_wave_tile<PP, RS>;
        const size_t su = update_smem(P.S), sw = wave_smem();
        cudaError_t e = cudaFuncSetAttribute(fu, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)su);
        if (e != cudaSuccess) return (int)e;
        e = cudaFuncSetAttribute(fw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw);
        if (e != cudaSuccess) return (int)e;
        int occ_u = 0, occ_w = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_u, fu, TILE_THREADS, su);
        if (e != cudaSuccess) return (int)e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_w, fw, TILE_THREADS, sw);
        if (e != cudaSuccess) return (int)e;
        if (occ_u < 1) occ_u = 1;
        if (occ_w < 1) occ_w = 1;
        cfg.grid_update = (int)(ntiles < (int64_t)num_sms * occ_u ? ntiles : (int64_t)num_sms * occ_u);
        cfg.grid_wave = (int)(ntiles < (int64_t)num_sms * occ_w ? ntiles : (int64_t)num_sms * occ_w);
        cfg.smem_update = su;
        cfg.smem_wave = sw;
        cfg.fn_update = fu;
        cfg.fn_wave = fw;
        return 0;
    }

    template <int MAXS, bool BUDGET>
    static void *ubatch_fn() { return (void *)k_update_batch<PP, RS, MAXS, BUDGET>; }

    static int configure_batch(int max_classes, bool budget, BatchConfig &cfg)
    {
        void *fu;
        if (max_classes <= 4) fu = budget ? ubatch_fn<4, true>() : ubatch_fn<4, false>();
        else if (max_classes <= 8) fu = budget ? ubatch_fn<8, true>() : ubatch_fn<8, false>();
        else fu = budget ? ubatch_fn<16, true>() : ubatch_fn<16, false>();
        void *fw = (void *)k_wave_batch<PP, RS>;
        const size_t su = update_smem(max_classes), sw = wave_smem();
        cudaError_t e = cudaFuncSetAttribute(fu, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)su);
        if (e != cudaSuccess) return (int)e;
        e = cudaFuncSetAttribute(fw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw);
        if (e != cudaSuccess) return (int)e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cfg.occ_update, fu, TILE_THREADS, su);
        if (e != cudaSuccess) return (int)e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cfg.occ_wave, fw, TILE_THREADS, sw);
        if (e != cudaSuccess) return (int)e;
        if (cfg.occ_update < 1) cfg.occ_update = 1;
        if (cfg.occ_wave < 1) cfg.occ_wave = 1;
        for (int S = 0; S <= 16; S++) {
            const int Sc = S < 1 ? 1 : (S > max_classes ? max_classes : S);
            cfg.smem_update_s[S] = update_smem(Sc);
            int o = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fu, TILE_THREADS, cfg.smem_update_s[S]);
            if (e != cudaSuccess) return (int)e;
            cfg.occ_update_s[S] = o < 1 ? 1 : o;
        }
        cfg.fn_update = fu;
        cfg.fn_wave = fw;
        cfg.smem_update = su;
        cfg.smem_wave = sw;
        cfg.threads = TILE_THREADS;
        cfg.tile_i = T_I;
        cfg.tile_j = T_J;
        return 0;
    }

    static int launch(const DevParams &P, const BufsT<RS> &B, Ctl *ctl, const double *rain, double *partials,
                      double *stage, double *saveflow, const StepConfig &cfg, cudaStream_t s, cudaEvent_t ev0,
                      cudaEvent_t ev1)
    {
        void *wargs[] = {(void *)&P, (void *)&B, (void *)&ctl};
        cudaLaunchKernel(cfg.fn_wave, dim3(cfg.grid_wave), dim3(TILE_THREADS), wargs, cfg.smem_wave, s);
        if (ev0) cudaEventRecord(ev0, s);
        void *args[] = {(void *)&P, (void *)&B, (void *)&ctl, (void *)&rain, (void *)&partials, (void *)&stage,
                        (void *)&saveflow};
        cudaLaunchKernel(cfg.fn_update, dim3(cfg.grid_update), dim3(TILE_THREADS), args, cfg.smem_update, s);
        if (ev1) cudaEventRecord(ev1, s);
        return (int)cudaGetLastError();
    }
};

}  // namespace swehr
