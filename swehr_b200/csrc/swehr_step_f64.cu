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
#include "swehr_launch.cuh"

namespace swehr {

int configure_step_f64(const DevParams &P, int num_sms, StepConfig &cfg)
{
    return FormLauncher<PolicyF64, double>::configure(P, num_sms, cfg);
}

int launch_wave_f64(const DevParams &P, const BufsT<double> &B, Ctl *ctl, const StepConfig &cfg, cudaStream_t s)
{
    return FormLauncher<PolicyF64, double>::launch_wave(P, B, ctl, cfg, s);
}

int launch_update_f64(const DevParams &P, const BufsT<double> &B, Ctl *ctl, const double *rain, double *partials,
                      double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s)
{
    return FormLauncher<PolicyF64, double>::launch_update(P, B, ctl, rain, partials, stage, saveflow, tm, cfg, s);
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

int tma_available() { return tensor_map_encoder() != nullptr; }

int encode_tma_f64(const DevParams &P, const BufsT<double> &B, TmaMaps &tm)
{
    return FormLauncher<PolicyF64, double>::encode_tma(P, B, tm);
}

int configure_batch_f64(int max_classes, bool budget, BatchConfig &cfg)
{
    return FormLauncher<PolicyF64, double>::configure_batch(max_classes, budget, cfg);
}

}  // namespace swehr
