/*
 * swehr_launch.cuh -- launch geometry and enqueueing of the two step kernels
 * of one form (included once per form, by swehr_step_f64.cu and
 * swehr_step_f32.cu, which are compiled with different contraction flags).
 */
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <type_traits>

#include "swehr_kernels.h"
#include "swehr_tile.cuh"

namespace swehr {

typedef CUresult (*TensorMapEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                      const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

/* cuTensorMapEncodeTiled through the runtime's driver entry point (no link
 * against libcuda); null when the driver does not offer it */
static inline TensorMapEncodeFn tensor_map_encoder()
{
    static TensorMapEncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (TensorMapEncodeFn)p;
    }
    return fn;
}

/* A 3-D tensor (ny, nx, planes) of T planes at base with the domain's pitch
 * and plane stride, copied in boxes of box_x x box_y x 1.  The driver checks
 * the base (16-byte aligned), the strides (multiples of 16 bytes) and the
 * box's inner extent (a multiple of 16 bytes). */
template <class T>
static inline bool encode_planes(TensorMapEncodeFn enc, CUtensorMap *m, const void *base, const DevParams &P,
                                 int planes, unsigned box_x, unsigned box_y)
{
    const cuuint64_t dims[3] = {(cuuint64_t)P.ny, (cuuint64_t)P.nx, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)P.pitch * sizeof(T), (cuuint64_t)P.plane * sizeof(T)};
    const cuuint32_t box[3] = {box_x, box_y, 1};
    const cuuint32_t elem[3] = {1, 1, 1};
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    return enc(m, dt, 3, const_cast<void *>(base), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

inline namespace SWEHR_TILE_NS {

template <class PP, class RS>
struct FormLauncher {
    typedef typename PP::R R;

    static size_t update_smem(int S, int stage_m = 1) { return StagedLayout::make(S, sizeof(R), stage_m).total; }

    /* The update kernel and shared memory for S classes: M_k staged unless
     * leaving it in global memory fits more blocks per SM (measured: staging
     * is 2-5 % faster at equal occupancy; at 10 FP64 classes dropping it
     * doubles the resident blocks and the update runs ~27 % faster).  Sets
     * both kernels' shared-memory limits. */
    static cudaError_t pick_staging(void *f_with, void *f_without, int S, size_t &smem, int &occ, int &stage_m,
                                    void *&fn, size_t extra = 0)
    {
        const size_t with = update_smem(S, 1) + extra, without = update_smem(S, 0) + extra;
        int ow = 0, oo = 0;
        cudaError_t e = cudaFuncSetAttribute(f_with, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)with);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(f_without, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)without);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ow, f_with, TILE_THREADS, with);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oo, f_without, TILE_THREADS, without);
        if (e != cudaSuccess) return e;
        stage_m = ow >= oo;
        smem = stage_m ? with : without;
        occ = stage_m ? ow : oo;
        fn = stage_m ? f_with : f_without;
        if (occ < 1) occ = 1;
        return cudaSuccess;
    }
    static size_t wave_smem() { return 0; }   /* the wave pass stages nothing */

    static int init_gz(const DevParams &P, const BufsT<RS> &B, int64_t n, cudaStream_t s)
    {
        k_init_gz<PP, RS><<<4 * 148, TILE_THREADS, 0, s>>>(P, B, n);
        return (int)cudaGetLastError();
    }

    /* tile loads through tensor maps (both forms: every staged window starts
     * on a 16-byte column, see Cols) */
    static constexpr bool kHasTma = true;

    /* Tensor maps for the update kernel's tile loads (planes of one domain):
     * each state set's planes of the storage type with the halo box and the
     * cell box, its FP64 planes with the cell box, the three topography
     * planes with the z_prev and z window boxes, and the Ks plane.  Returns 0
     * when every map was encoded. */
    static int encode_tma(const DevParams &P, const BufsT<RS> &B, TmaMaps &tm)
    {
        TensorMapEncodeFn enc = tensor_map_encoder();
        if (!enc) return 1;
        memset(&tm, 0, sizeof tm);
        const bool mixed = !std::is_same<RS, double>::value;
        const int planes = mixed ? 9 + P.S : P_FIXED + 2 * P.S;     /* the storage-type block of a set */
        bool ok = true;
        for (int s = 0; s < 2; s++) {
            ok = ok && encode_planes<RS>(enc, &tm.m[TM_HALO0 + s], B.set[s].h, P, planes, Cols<RS>::rj, HALO_ROWS);
            ok = ok && encode_planes<RS>(enc, &tm.m[TM_CELL0 + s], B.set[s].h, P, planes, T_J, T_I);
            if (mixed)
                ok = ok && encode_planes<double>(enc, &tm.m[TM_CELLD0 + s], B.set[s].vinf, P, 1 + P.S, T_J, T_I);
            else
                ok = ok && encode_planes<double>(enc, &tm.m[TM_CELLD0 + s], B.set[s].h, P, planes, T_J, T_I);
        }
        ok = ok && encode_planes<double>(enc, &tm.m[TM_ZP], B.z[0], P, 3, R_J, ZP_ROWS);
        ok = ok && encode_planes<double>(enc, &tm.m[TM_ZC], B.z[0], P, 3, R_J, ZC_ROWS);
        if (B.ks) ok = ok && encode_planes<RS>(enc, &tm.m[TM_KS], B.ks, P, 1, T_J, T_I);
        return ok ? 0 : 2;
    }

    template <int MAXS, bool BUDGET, bool SM, bool TMA, int NS = 0>
    static void *update_fn() { return (void *)k_update_tile<PP, RS, MAXS, BUDGET, SM, TMA, NS>; }

    template <bool BUDGET, bool SM, bool TMA>
    static void *pick_u(int S)
    {
        /* the class counts of the benchmark configurations get kernels
         * built for exactly that many classes: their class loops have no
         * exit tests, so the compiler interleaves the classes' independent
         * division chains (mixed form -7 %) */
        if (S == 7) return update_fn<8, BUDGET, SM, TMA, 7>();
        if (S == 10) return update_fn<16, BUDGET, SM, TMA, 10>();
        if (S <= 4) return update_fn<4, BUDGET, SM, TMA>();
        if (S <= 8) return update_fn<8, BUDGET, SM, TMA>();
        return update_fn<16, BUDGET, SM, TMA>();
    }

    template <bool TMA>
    static void *pick_update_t(int S, bool budget, bool sm)
    {
        if (budget) return sm ? pick_u<true, true, TMA>(S) : pick_u<true, false, TMA>(S);
        return sm ? pick_u<false, true, TMA>(S) : pick_u<false, false, TMA>(S);
    }

    static void *pick_update(int S, bool budget, bool sm, bool tma = false)
    {
        if constexpr (kHasTma) {
            if (tma) return pick_update_t<true>(S, budget, sm);
        }
        return pick_update_t<false>(S, budget, sm);
    }

    static int configure(const DevParams &P, int num_sms, StepConfig &cfg)
    {
        const int64_t ntiles = (int64_t)((P.nx + T_I - 1) / T_I) * ((P.ny + T_J - 1) / T_J);
        void *fu = nullptr;
        void *fw = (void *)k_wave_cells<PP, RS>;
        size_t su = 0;
        const size_t sw = wave_smem();
        int occ_u = 0, occ_w = 0, stage_m = 1;
        const bool tma = kHasTma && cfg.tma;
        cfg.tma = tma ? 1 : 0;
        cudaError_t e = pick_staging(pick_update(P.S, P.budget != 0, true, tma),
                                     pick_update(P.S, P.budget != 0, false, tma), P.S, su, occ_u, stage_m, fu,
                                     tma ? 128 : 0);
        if (e != cudaSuccess) return (int)e;
        e = cudaFuncSetAttribute(fw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw);
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
        cfg.stage_m = stage_m;
        return 0;
    }

    template <int MAXS, bool BUDGET, bool SM, int NS = 0>
    static void *ubatch_fn() { return (void *)k_update_batch<PP, RS, MAXS, BUDGET, SM, NS>; }

    /* batched kernels for exactly NS classes (every running scenario has NS) */
    template <int MAXS, int NS>
    static cudaError_t exact_batch(bool budget, BatchConfig &cfg)
    {
        void *fw = budget ? ubatch_fn<MAXS, true, true, NS>() : ubatch_fn<MAXS, false, true, NS>();
        void *fo = budget ? ubatch_fn<MAXS, true, false, NS>() : ubatch_fn<MAXS, false, false, NS>();
        int sm = 1;
        return pick_staging(fw, fo, NS, cfg.smem_update_x[NS], cfg.occ_update_x[NS], sm, cfg.fn_update_x[NS]);
    }

    template <bool SM>
    static void *pick_ub(int max_classes, bool budget)
    {
        if (max_classes <= 4) return budget ? ubatch_fn<4, true, SM>() : ubatch_fn<4, false, SM>();
        if (max_classes <= 8) return budget ? ubatch_fn<8, true, SM>() : ubatch_fn<8, false, SM>();
        return budget ? ubatch_fn<16, true, SM>() : ubatch_fn<16, false, SM>();
    }

    static int configure_batch(int max_classes, bool budget, BatchConfig &cfg)
    {
        void *fu_with = pick_ub<true>(max_classes, budget), *fu_without = pick_ub<false>(max_classes, budget);
        void *fw = (void *)k_wave_batch<PP, RS>;
        const size_t su = update_smem(max_classes), sw = wave_smem();
        cudaError_t e = cudaFuncSetAttribute(fw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw);
        if (e != cudaSuccess) return (int)e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cfg.occ_wave, fw, TILE_THREADS, sw);
        if (e != cudaSuccess) return (int)e;
        if (cfg.occ_wave < 1) cfg.occ_wave = 1;
        cfg.occ_update = 1;
        for (int S = 0; S <= 16; S++) {
            const int Sc = S < 1 ? 1 : (S > max_classes ? max_classes : S);
            e = pick_staging(fu_with, fu_without, Sc, cfg.smem_update_s[S], cfg.occ_update_s[S], cfg.stage_m_s[S],
                             cfg.fn_update_s[S]);
            if (e != cudaSuccess) return (int)e;
            if (cfg.occ_update_s[S] > cfg.occ_update) cfg.occ_update = cfg.occ_update_s[S];
        }
        if (max_classes >= 7) {
            e = exact_batch<8, 7>(budget, cfg);
            if (e != cudaSuccess) return (int)e;
        }
        if (max_classes >= 10) {
            e = exact_batch<16, 10>(budget, cfg);
            if (e != cudaSuccess) return (int)e;
        }
        /* limits for the largest shape either kernel is launched with */
        e = cudaFuncSetAttribute(fu_with, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)su);
        if (e != cudaSuccess) return (int)e;
        e = cudaFuncSetAttribute(fu_without, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)update_smem(max_classes, 0));
        if (e != cudaSuccess) return (int)e;
        cfg.fn_update = cfg.fn_update_s[max_classes];
        cfg.fn_wave = fw;
        cfg.smem_update = su;
        cfg.smem_wave = sw;
        cfg.threads = TILE_THREADS;
        cfg.tile_i = T_I;
        cfg.tile_j = T_J;
        return 0;
    }

    static int launch(const DevParams &P, const BufsT<RS> &B, Ctl *ctl, const double *rain, double *partials,
                      double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s,
                      cudaEvent_t ev0, cudaEvent_t ev1)
    {
        void *wargs[] = {(void *)&P, (void *)&B, (void *)&ctl};
        cudaLaunchKernel(cfg.fn_wave, dim3(cfg.grid_wave), dim3(TILE_THREADS), wargs, cfg.smem_wave, s);
        if (ev0) cudaEventRecord(ev0, s);
        void *args[] = {(void *)&P, (void *)&B, (void *)&ctl, (void *)&rain, (void *)&partials, (void *)&stage,
                        (void *)&saveflow, (void *)&tm};
        cudaLaunchKernel(cfg.fn_update, dim3(cfg.grid_update), dim3(TILE_THREADS), args, cfg.smem_update, s);
        if (ev1) cudaEventRecord(ev1, s);
        return (int)cudaGetLastError();
    }

    /* the two passes of a step one at a time (a slab of a split domain takes
     * the largest wave speed over every slab between them) */
    static int launch_wave(const DevParams &P, const BufsT<RS> &B, Ctl *ctl, const StepConfig &cfg, cudaStream_t s)
    {
        void *wargs[] = {(void *)&P, (void *)&B, (void *)&ctl};
        cudaLaunchKernel(cfg.fn_wave, dim3(cfg.grid_wave), dim3(TILE_THREADS), wargs, cfg.smem_wave, s);
        return (int)cudaGetLastError();
    }

    static int launch_update(const DevParams &P, const BufsT<RS> &B, Ctl *ctl, const double *rain, double *partials,
                             double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s)
    {
        void *args[] = {(void *)&P, (void *)&B, (void *)&ctl, (void *)&rain, (void *)&partials, (void *)&stage,
                        (void *)&saveflow, (void *)&tm};
        cudaLaunchKernel(cfg.fn_update, dim3(cfg.grid_update), dim3(TILE_THREADS), args, cfg.smem_update, s);
        return (int)cudaGetLastError();
    }
};

}  // inline namespace SWEHR_TILE_NS
}  // namespace swehr
