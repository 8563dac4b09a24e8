/*
 * swehr_step_f32.cu -- the mixed form of one SWEHR time step on sm_100a:
 * h, hu, hv, U_k, the maxima, TOTM, DEP, TOTSED and Ks in FP32 (SFU
 * intrinsics, fused multiply-add allowed); z, cumulative infiltration and its
 * Green-Ampt update, deposited mass M_k, t/dt and the budgets in FP64.
 * Same two-launch step as the FP64 form (swehr_step_f64.cu).
 */
#include "swehr_launch.cuh"

namespace swehr {

int configure_step_f32(const DevParams &P, int num_sms, StepConfig &cfg)
{
    return FormLauncher<PolicyF32, float>::configure(P, num_sms, cfg);
}

int launch_wave_f32(const DevParams &P, const BufsT<float> &B, Ctl *ctl, const StepConfig &cfg, cudaStream_t s)
{
    return FormLauncher<PolicyF32, float>::launch_wave(P, B, ctl, cfg, s);
}

int launch_update_f32(const DevParams &P, const BufsT<float> &B, Ctl *ctl, const double *rain, double *partials,
                      double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s)
{
    return FormLauncher<PolicyF32, float>::launch_update(P, B, ctl, rain, partials, stage, saveflow, tm, cfg, s);
}

int init_gz_f32(const DevParams &P, const BufsT<float> &B, int64_t n, cudaStream_t s)
{
    return FormLauncher<PolicyF32, float>::init_gz(P, B, n, s);
}

int launch_step_f32(const DevParams &P, const BufsT<float> &B, Ctl *ctl, const double *rain, double *partials,
                    double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s,
                    cudaEvent_t ev0, cudaEvent_t ev1)
{
    return FormLauncher<PolicyF32, float>::launch(P, B, ctl, rain, partials, stage, saveflow, tm, cfg, s, ev0, ev1);
}

int encode_tma_f32(const DevParams &P, const BufsT<float> &B, TmaMaps &tm)
{
    return FormLauncher<PolicyF32, float>::encode_tma(P, B, tm);
}

int configure_batch_f32(int max_classes, bool budget, BatchConfig &cfg)
{
    return FormLauncher<PolicyF32, float>::configure_batch(max_classes, budget, cfg);
}

}  // namespace swehr
