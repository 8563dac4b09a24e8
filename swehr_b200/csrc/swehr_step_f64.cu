/*
 * swehr_step_f64.cu -- the plain FP64 form of one SWEHR time step on sm_100a.
 * Compiled with --fmad=false: no contraction, so every cell is bit-identical
 * to the CPU restatement built with the project's math.
 *
 * A step is two stream-ordered launches and needs no grid barrier:
 *   k_wave_cells  largest wave speed over every face (SWEHR.c:1092-1230's
 *                 Smax), one cell's faces per thread straight from global
 *                 memory; the last block to finish computes dt and the
 *                 Courant check (SWEHR.c:1409-1413) and arms the update;
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
#include <cstring>

#include "swehr_launch.cuh"

namespace swehr {

int configure_step_f64(const DevParams &P, int num_sms, StepConfig &cfg)
{
    return FormLauncher<PolicyF64, double>::configure(P, num_sms, cfg);
}

int init_gz_f64(const DevParams &P, const BufsT<double> &B, int64_t n, cudaStream_t s)
{
    return FormLauncher<PolicyF64, double>::init_gz(P, B, n, s);
}

int launch_step_f64(const DevParams &P, const BufsT<double> &B, Ctl *ctl, const double *rain, double *partials,
                    double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s,
                    cudaEvent_t ev0, cudaEvent_t ev1)
{
    return FormLauncher<PolicyF64, double>::launch(P, B, ctl, rain, partials, stage, saveflow, tm, cfg, s, ev0, ev1);
}

/* Tensor maps for the update kernel's tile loads (FP64 planes of one
 * domain): each state set as a 3-D tensor (ny, nx, planes), once with the
 * halo box and once with the cell box, the three topography planes with the
 * z_prev and z window boxes, and the Ks plane.  Returns 0 when every map was
 * encoded (the driver checks bases, strides and boxes). */
typedef CUresult (*TensorMapEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                      const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static TensorMapEncodeFn tensor_map_encoder()
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

static bool encode_planes(TensorMapEncodeFn enc, CUtensorMap *m, const void *base, const DevParams &P, int planes,
                          unsigned box_x, unsigned box_y)
{
    const cuuint64_t dims[3] = {(cuuint64_t)P.ny, (cuuint64_t)P.nx, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)P.pitch * sizeof(double), (cuuint64_t)P.plane * sizeof(double)};
    const cuuint32_t box[3] = {box_x, box_y, 1};
    const cuuint32_t elem[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), dims, strides, box, elem,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int tma_available_f64() { return tensor_map_encoder() != nullptr; }

int encode_tma_f64(const DevParams &P, const BufsT<double> &B, TmaMaps &tm)
{
    TensorMapEncodeFn enc = tensor_map_encoder();
    if (!enc) return 1;
    memset(&tm, 0, sizeof tm);
    const int planes = P_FIXED + 2 * P.S;
    bool ok = true;
    for (int s = 0; s < 2; s++) {
        ok = ok && encode_planes(enc, &tm.m[TM_HALO0 + s], B.set[s].h, P, planes, R_J, HALO_ROWS);
        ok = ok && encode_planes(enc, &tm.m[TM_CELL0 + s], B.set[s].h, P, planes, T_J, T_I);
    }
    ok = ok && encode_planes(enc, &tm.m[TM_ZP], B.z[0], P, 3, R_J, ZP_ROWS);
    ok = ok && encode_planes(enc, &tm.m[TM_ZC], B.z[0], P, 3, R_J, ZC_ROWS);
    if (B.ks) ok = ok && encode_planes(enc, &tm.m[TM_KS], B.ks, P, 1, T_J, T_I);
    return ok ? 0 : 2;
}

int configure_batch_f64(int max_classes, bool budget, BatchConfig &cfg)
{
    return FormLauncher<PolicyF64, double>::configure_batch(max_classes, budget, cfg);
}

}  // namespace swehr
