/*
 * swehr_ctx.h -- host-side state of one simulation (internal to the library;
 * shared by the single-domain entry points and the scenario pool).
 */
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/swehr.h"
#include "swehr_kernels.h"

static const int GRAPH_STEPS = 32;
static const int TIMING_RING = 64;

/* What a pool lends the contexts it creates: its stream and a device-memory
 * allocator (a cache of released allocations), so that admitting and
 * releasing a scenario needs no cudaMalloc / cudaFree (which synchronises
 * the device), no stream and no pinned allocation. */
struct CtxHost {
    cudaStream_t stream;
    void *self;
    void *(*alloc)(void *self, size_t bytes);
    void (*release)(void *self, void *ptr);
};

struct swehr_ctx {
    swehr_params p;
    int precision = SWEHR_FP64;
    int device = 0, num_sms = 148;
    int pooled = 0;         /* stepped by a swehr_pool, not by swehr_advance */
    const CtxHost *host = nullptr;   /* the pool's stream and allocator (pooled contexts) */
    swehr::DevParams P;
    swehr::BufsT<double> B64;      /* plain form */
    swehr::BufsT<float> B32;       /* mixed form */
    size_t rsize = 8;       /* bytes of a bulk (RS) element */
    char *mem = nullptr;    /* the one device allocation */
    size_t mem_bytes = 0;
    double *d_rain = nullptr, *d_partials = nullptr, *d_stage = nullptr, *d_saveflow = nullptr;
    swehr::Ctl *d_ctl = nullptr;
    swehr::Ctl *h_ctl = nullptr;   /* pinned mirror */
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    cudaEvent_t ev_k[2 * TIMING_RING] = {};
    void *h_stage = nullptr;           /* the process's two pinned download buffers (set on the first large read) */
    cudaEvent_t ev_stage[2] = {};
    swehr::StepConfig cfg;
    swehr::TmaMaps tm;      /* tensor maps of the update's tile loads (when cfg.tma) */
    int timing = 0;
    int64_t stagecap = 0;
    double water_init = 0;
    double sed_init[SWEHR_MAX_CLASSES] = {};
    /* a slab of a split domain (swehr_slab_create): halo rows held on each
     * side, and the device buffers send[2] then recv[2], halo_bytes each */
    int slab = 0, halo_lo = 0, halo_hi = 0;
    char *d_halo = nullptr;
    size_t halo_bytes = 0;
};

/* record an error message for swehr_last_error() and return code */
int swehr_err(int code, const std::string &msg);

/* Create a context.  With a host (a pool): stream and device memory come
 * from it, the control-block mirror is pageable, and the single-domain
 * kernels are neither configured nor timed. */
int swehr_ctx_create(const swehr_params *p, const swehr_inputs *in, int precision, const CtxHost *host,
                     swehr_ctx **out);

/* device bytes swehr_ctx_create() allocates for these inputs (upper bound);
 * num_sms 0 for a pooled context */
size_t swehr_ctx_footprint(const swehr_params *p, int has_ks, int has_solid, int precision, int num_sms);

/* free a context (pools use this for their scenarios) */
void swehr_ctx_destroy(swehr_ctx *c);
