/* swehr_kernels.h -- host-visible launch entry points of the step kernels. */
#pragma once
#include <cuda_runtime.h>

#include "swehr_device.cuh"
#include "swehr_tma.cuh"

namespace swehr {

/* one state set as seen by a kernel: RS = storage type of the bulk fields
 * (double in the plain form, float in the mixed form) */
template <class RS>
struct SetV {
    RS *h, *hu, *hv, *maxvel, *maxdep, *totm, *dep, *totsed, *U;   /* U: S planes */
    RS *gz;            /* GZ from this step's previous-step topography, for the wave pass */
    double *vinf, *M;                                                /* M: S planes */
};

/* device buffers of one simulation: two state sets, the topography of the
 * previous, current and next step, optional per-cell Ks, and -- with
 * interior solid cells -- the solid mask (one byte per cell, same pitch)
 * and the topography at set-up, from which the slopes a solid cell keeps
 * are taken (a solid cell never recomputes them, SWEHR.c:1233) */
template <class RS>
struct BufsT {
    SetV<RS> set[2];
    double *z[3];
    const RS *ks;
    const uint8_t *solid;
    const double *z0;
};

/* one scenario of a batch: everything its tiles need */
template <class RS>
struct ScenDesc {
    DevParams P;
    BufsT<RS> B;
    Ctl *ctl;
    const double *rain;
    double *stage, *saveflow;
    ScenSummary *sum;                /* this scenario's progress slot */
    int64_t tile0, ntiles;           /* its range in the batch's tile list */
};

/* what a batched launch walks; lives in device memory so that a captured
 * graph stays valid while scenarios join and leave */
template <class RS>
struct BatchHdr {
    const ScenDesc<RS> *tab;
    int32_t nscen, pad;
    int64_t total_tiles;
    const int32_t *tile_scen;        /* scenario of each tile of the list */
    /* tile counters the blocks take work from: [0] wave pass, [1] update
     * pass.  Each pass resets the other's counter (the other pass is not
     * running then, by stream order), so both are 0 when their pass starts. */
    unsigned long long *grab;
};

/* the batched kernels of one form (both take one argument: the header) */
struct BatchConfig {
    void *fn_wave = nullptr, *fn_update = nullptr;
    size_t smem_wave = 0, smem_update = 0;
    int occ_wave = 1, occ_update = 1;   /* resident blocks per SM */
    int threads = 0;                    /* threads per block */
    int tile_i = 0, tile_j = 0;         /* cells per tile */
    /* update kernel: dynamic shared memory and resident blocks per SM when
     * the largest class count among the scenarios is S (index S = 0..16) */
    size_t smem_update_s[17] = {};
    int occ_update_s[17] = {};
    int stage_m_s[17] = {};             /* stage M_k in shared memory at this class count */
    void *fn_update_s[17] = {};         /* the update kernel for that choice */
    /* kernels built for exactly S classes (S = 7, 10; null elsewhere), used
     * when every running scenario has S classes */
    void *fn_update_x[17] = {};
    size_t smem_update_x[17] = {};
    int occ_update_x[17] = {};
};

int configure_batch_f64(int max_classes, bool budget, BatchConfig &cfg);
int configure_batch_f32(int max_classes, bool budget, BatchConfig &cfg);
/* the same kernels built for 16 x 16-cell tiles (cfg.tile_i = cfg.tile_j = 16) */
int configure_batch_f64_t16(int max_classes, bool budget, BatchConfig &cfg);
int configure_batch_f32_t16(int max_classes, bool budget, BatchConfig &cfg);

/* launch geometry of the step kernels of one simulation */
struct StepConfig {
    int grid_wave = 1, grid_update = 1;
    size_t smem_wave = 0, smem_update = 0;
    void *fn_update = nullptr, *fn_wave = nullptr;
    int stage_m = 1;                    /* the update stages M_k in shared memory */
    int tma = 0;                        /* in: tensor maps can be encoded; out: the update loads tiles through them */
};

/* Pick the kernel instantiations, set their shared-memory limit and size the
 * persistent grids from the occupancy (return a cudaError_t). */
int configure_step_f64(const DevParams &P, int num_sms, StepConfig &cfg);
int configure_step_f32(const DevParams &P, int num_sms, StepConfig &cfg);

/* Enqueue one full step (wave pass + update pass); ev0/ev1 (optional) are
 * recorded around the update kernel. */
int launch_step_f64(const DevParams &P, const BufsT<double> &B, Ctl *ctl, const double *rain, double *partials,
                    double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s,
                    cudaEvent_t ev0, cudaEvent_t ev1);
/* the two passes of a step separately (slabs of a split domain) */
int launch_wave_f64(const DevParams &P, const BufsT<double> &B, Ctl *ctl, const StepConfig &cfg, cudaStream_t s);
int launch_wave_f32(const DevParams &P, const BufsT<float> &B, Ctl *ctl, const StepConfig &cfg, cudaStream_t s);
int launch_update_f64(const DevParams &P, const BufsT<double> &B, Ctl *ctl, const double *rain, double *partials,
                      double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s);
int launch_update_f32(const DevParams &P, const BufsT<float> &B, Ctl *ctl, const double *rain, double *partials,
                      double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s);
/* the update kernel's tile loads through tensor maps (one domain): whether
 * the driver offers the encoder, and the maps of a simulation's planes (0
 * when all were encoded) */
int tma_available();
int encode_tma_f64(const DevParams &P, const BufsT<double> &B, TmaMaps &tm);
int encode_tma_f32(const DevParams &P, const BufsT<float> &B, TmaMaps &tm);

/* the gz plane of the set step n reads, from its previous-step topography
 * (at creation and after the topography is written) */
int init_gz_f64(const DevParams &P, const BufsT<double> &B, int64_t n, cudaStream_t s);
int init_gz_f32(const DevParams &P, const BufsT<float> &B, int64_t n, cudaStream_t s);
int launch_step_f32(const DevParams &P, const BufsT<float> &B, Ctl *ctl, const double *rain, double *partials,
                    double *stage, double *saveflow, const TmaMaps &tm, const StepConfig &cfg, cudaStream_t s,
                    cudaEvent_t ev0, cudaEvent_t ev1);

}  // namespace swehr
