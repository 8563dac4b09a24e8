/*
 * swehr.h -- C ABI of the B200-native SWEHR time step.
 *
 * The reference (SWEHR.c of csdms-contrib/swehr) is one C program whose
 * solver is the body of `while (t<tend)` inside main() (SWEHR.c:808-1699).
 * It has no library interface; the entry points below are the seam a
 * maintainer would cut at, each one citing the region of SWEHR.c it
 * replaces.  All pointers are plain host pointers; the library copies what
 * it is given and never keeps a caller buffer.  No torch or CUDA types
 * appear in the signatures.
 *
 * Grid orientation follows the reference: i = 1..nx is the first index,
 * j = 1..ny the second, and every nx*ny host array is i-major with j
 * contiguous, element (i,j) at [(i-1)*ny + (j-1)] -- the order topoin.txt is
 * read in (SWEHR.c:223-227).
 */
#ifndef SWEHR_H
#define SWEHR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWEHR_ABI_VERSION 2
#define SWEHR_MAX_CLASSES 16

typedef enum swehr_status {
    SWEHR_OK = 0,
    SWEHR_CFL_ERROR = 1,    /* Courant number > 1 (SWEHR.c:1412-1413); the step completes, then stepping stops */
    SWEHR_NAN = 2,          /* non-finite water depth detected (only when params.stop_on_nan) */
    SWEHR_TIMEOUT = 3,      /* host wall-clock limit of swehr_advance reached */
    SWEHR_CUDA_ERROR = 4,   /* a CUDA runtime call failed; see swehr_last_error() */
    SWEHR_INVALID = 5,      /* bad argument (sizes, NULL pointers, class count, ...) */
    SWEHR_OOM = 6,          /* device allocation failed / pool budget exceeded */
    SWEHR_NO_DEVICE = 7,    /* no CUDA device visible */
    SWEHR_BUSY = 8          /* pool: no slot or memory free right now */
} swehr_status;

typedef enum swehr_precision {
    SWEHR_FP64 = 0,         /* plain form: every operation in FP64, bit-identical to the CPU restatement */
    SWEHR_MIXED = 1         /* FP32 bulk; FP64 for z, cumulative infiltration, deposited mass and budgets */
} swehr_precision;

/* Run parameters.  The first block is input.txt in file order
 * (SWEHR.c:474-504); everything after it is hard-coded in the reference and
 * exposed here with the reference's values as defaults (swehr_params_default). */
typedef struct swehr_params {
    /* input.txt: nx ny dx F manning0 tend a ad h0 mtstar0 rnum rint sclass J */
    int32_t nx, ny;
    double  dx;
    double  F;              /* effective fraction of stream power in entrainment */
    double  manning0;       /* read but unused by the reference (roughness is hard-coded) */
    double  tend;           /* total simulated time [s] */
    double  a, ad;          /* detachability of original / deposited soil */
    double  h0;             /* critical depth in rain-splash depth dependence */
    double  mtstar0;        /* deposited mass that fully shields the soil */
    int32_t rnum;           /* number of hyetograph entries */
    int32_t sclass;         /* number of sediment size classes S */
    double  rint;           /* seconds per hyetograph entry */
    double  J;              /* energy to entrain a unit mass */
    /* SWEHR.c:490-494 */
    double  hcfriction, depthdependentexponent, b, af, afr;
    /* SWEHR.c:632-633 */
    double  cstable, maxstep;
    /* SWEHR.c:638-650 */
    double  g, hfilm, phi, rhos, rhow, nu, frictionangle, cohesion, lambda, cthreshold, betabedload;
    /* per-cell soil defaults, SWEHR.c:236-246 (uniform unless a per-cell array is given) */
    double  roughness, ks, theta0, thetas, hf, vinf0, uc, uc2;
    /* boundary types BNDRY[1..4] = {i=1, j=1, i=nx, j=ny} (SWEHR.c:617-621): 0 transmissive, 1 solid */
    int32_t bndry[4];
    int32_t inflow;         /* 1: hard-wired sediment-laden inflow ghost at j=ny (SWEHR.c:1010-1035) */
    int32_t stop_on_nan;    /* 1: stop with SWEHR_NAN when a non-finite depth appears */
    /* stage / point series (SWEHR.c:1593-1676): stageint [s], outlet row, six sample points (1-based) */
    double  stageint;
    int32_t outlet_row;
    int32_t npoints;
    int32_t xpoint[6], ypoint[6];
    /* moving Gaussian storm (an extension; the reference only has a uniform hyetograph).
     * When storm_peak > 0 the rain at cell centre (x,y) = ((i-0.5)dx, (j-0.5)dx) is
     * storm_peak*exp(-0.5*((x-x0-vx t)^2+(y-y0-vy t)^2)/storm_radius^2) and the hyetograph is ignored. */
    double  storm_peak, storm_radius, storm_x0, storm_y0, storm_vx, storm_vy;
    int32_t budget;         /* 1: accumulate compensated water / sediment budget terms every step */
    int32_t reserved_i[7];
    double  reserved_d[8];
} swehr_params;

/* Host inputs (copied by swehr_create). */
typedef struct swehr_inputs {
    const double *topo;     /* nx*ny elevations, i-major (topoin.txt) */
    const double *rain;     /* rnum rates [m/s] (rain.txt) */
    const double *ds;       /* sclass diameters [m] (particlesizein.txt) */
    const double *pfrac;    /* sclass mass fractions of the original soil (particlepercentin.txt) */
    const double *ks;       /* optional nx*ny saturated conductivity [m/s]; NULL -> params.ks everywhere */
    /* optional nx*ny interior solid mask, i-major (SOLID[i][j], SWEHR.c:597; the
     * stock program leaves it all zero): a nonzero cell is outside the flow
     * domain.  swehr_create fills its topography from its neighbours as
     * initialcondition does (SWEHR.c:288-322), faces between a solid and a flow
     * cell reflect the flow cell's state (SWEHR.c:1137-1146, 1205-1214), and a
     * solid cell takes no sources and holds no water or suspended sediment
     * (SWEHR.c:1233, 1421, 1566-1574).  NULL -> no solid cells.  (Added in ABI 2.) */
    const int32_t *solid;
} swehr_inputs;

/* Fields readable with swehr_read_field; all are nx*ny, i-major. */
typedef enum swehr_field {
    SWEHR_FIELD_H = 0,        /* U[1]  depth            (depth.txt) */
    SWEHR_FIELD_HU = 1,       /* U[2]                   (uh.txt) */
    SWEHR_FIELD_HV = 2,       /* U[3]                   (vh.txt) */
    SWEHR_FIELD_Z = 3,        /* TOPO                   (topoout.txt) */
    SWEHR_FIELD_VINF = 4,     /* cumulative infiltration */
    SWEHR_FIELD_U = 5,        /* U[3+k] suspended mass per area, class k (ch.txt for k=1) */
    SWEHR_FIELD_M = 6,        /* M[k] deposited mass per area, class k */
    SWEHR_FIELD_TOTM = 7,     /* TOTM                   (m.txt) */
    SWEHR_FIELD_TOTSED = 8,   /* TOTSED                 (c.txt) */
    SWEHR_FIELD_VEL = 9,      /* |v|                    (vel.txt) */
    SWEHR_FIELD_MAXVEL = 10,  /*                        (maxvel.txt) */
    SWEHR_FIELD_MAXDEPTH = 11,/*                        (maxdepth.txt) */
    SWEHR_FIELD_DEP = 12,     /* DEP deposited thickness */
    SWEHR_FIELD_SED = 13      /* SED[k] suspended concentration, class k */
} swehr_field;

/* Progress of one swehr_advance call. */
typedef struct swehr_progress {
    double  t;              /* simulated time after the last completed step */
    double  dt;             /* last time step */
    double  courant;        /* last Courant number */
    double  rain;           /* uniform rain rate of the last step (0 with a moving storm) */
    int64_t steps;          /* steps completed since swehr_create */
    int64_t steps_this_call;
    double  device_ms;      /* device time of this call, CUDA events on the context stream */
    double  kernel_ms;      /* summed device time of the update kernel (only with swehr_set_timing(ctx,1)) */
    int64_t kernel_launches;/* kernels this call launched */
    int32_t status;
    int32_t done;           /* 1 when t >= tend */
    double  t_step;         /* start time of the last completed step (the time a CFL error is reported at) */
} swehr_progress;

/* Water / sediment budget (an addition; the reference keeps none).  All sums
 * are over the interior cells in depth units [m] (water) or mass per area
 * [kg/m^2] (sediment, per class), accumulated in compensated FP64.
 * water:  sum(h+VINF)_now - sum(h+VINF)_0 == rain_in - outflow + clamp_gain + bulking + rounding
 * sed k:  sum(U_k+M_k)_now - sum(U_k+M_k)_0 == detach_k - sed_outflow_k + sed_rounding_k */
typedef struct swehr_budget {
    double water_now, water_init;
    double rain_in, outflow, clamp_gain, bulking, infiltration;
    double water_residual;                /* (now - init) - (rain_in - outflow + clamp_gain + bulking) */
    double sed_now[SWEHR_MAX_CLASSES], sed_init[SWEHR_MAX_CLASSES];
    double detach[SWEHR_MAX_CLASSES], sed_outflow[SWEHR_MAX_CLASSES];
    double sed_residual[SWEHR_MAX_CLASSES];
    int32_t sclass;
    int32_t valid;
    /* rounding of the stored state: what the arithmetic and the storage format
     * (FP32 in the mixed form) added to sum(h) and sum(U_k+M_k); ~1e-17
     * relative in the plain form */
    double rounding;
    double sed_rounding[SWEHR_MAX_CLASSES];
} swehr_budget;

typedef struct swehr_ctx swehr_ctx;

/* Reference defaults for every parameter (SWEHR.c:490-494, 617-650, 236-246);
 * input.txt values are zeroed and must be filled by the caller. */
void swehr_params_default(swehr_params *p);
size_t swehr_params_size(void);
int swehr_abi_version(void);
const char *swehr_status_str(int status);
const char *swehr_last_error(void);

/* Replaces SWEHR.c:540-803 (allocation, initialcondition, masks, neighbour
 * tables, initial slopes and gravity).  Copies inputs to the device. */
int swehr_create(const swehr_params *p, const swehr_inputs *in, int precision, swehr_ctx **out);

/* Replaces the body of `while (t<tend)` (SWEHR.c:808-1591): steps until
 * t >= min(t_stop, tend) or max_steps steps (max_steps < 0: unbounded) were
 * taken.  dt is clamped against tend only (SWEHR.c:1411), so pausing at
 * t_stop never changes the trajectory.  progress may be NULL. */
int swehr_advance(swehr_ctx *ctx, double t_stop, int64_t max_steps, swehr_progress *progress);

/* Replaces the final writers (SWEHR.c:1718-1747): copies one field (class k,
 * 1-based, for the per-class fields) into dst[nx*ny], i-major, FP64. */
int swehr_read_field(swehr_ctx *ctx, int field, int k, double *dst);

/* Replaces STAGE / SAVEFLOW (SWEHR.c:1593-1676, written at 1749-1761).
 * Copies up to max_rows rows of the stage series (24 doubles per row) and the
 * point series (18 doubles per row, three per point) recorded so far;
 * returns the row count through *rows. */
int swehr_read_series(swehr_ctx *ctx, double *stage, double *saveflow, int64_t max_rows, int64_t *rows);

/* Budget sums accumulated so far (requires params.budget = 1). */
int swehr_get_budget(swehr_ctx *ctx, swehr_budget *b);

/* 1: time the update kernel with CUDA events around every launch. */
int swehr_set_timing(swehr_ctx *ctx, int on);

/* Replaces nothing in the reference: uploads a whole state (one field) to
 * continue from a snapshot; same layout as swehr_read_field. */
int swehr_write_field(swehr_ctx *ctx, int field, int k, const double *src);

/* Device bytes held by a context for the given sizes (admission control). */
size_t swehr_footprint_bytes(int nx, int ny, int sclass, int precision);

void swehr_destroy(swehr_ctx *ctx);

/* No counterpart in the reference (SWEHR.c computes dt on the host inside
 * main, SWEHR.c:1409-1411, and has no device).  The CFL time step of one
 * state, for callers that cannot allocate device memory -- a framework that
 * owns every allocation through its own pool, or code running where the
 * allocator is locked: nothing is allocated; the kernel's scratch is a fixed
 * file-scope device array of 128.25 KiB held by every GPU that loads the
 * library.  d_h, d_hu, d_hv, d_zprev are caller-owned device planes of nx rows
 * by `pitch` doubles (cell (i,j) at [(i-1)*pitch + (j-1)]; d_zprev is the
 * topography of the previous step, or the current one at the first step);
 * d_result (device, 2 doubles) receives {Smax, dt} exactly as the update
 * path's wave pass computes them.  Asynchronous on `stream` (a cudaStream_t,
 * NULL for the legacy default stream).  Domains above SWEHR_NOALLOC_MAX_CELLS
 * cells are rejected with SWEHR_INVALID.  The first call on a device looks up
 * the scratch address there (make it before any stream capture); calls that
 * overlap on the GPU share the scratch and race -- serialise them. */
#define SWEHR_NOALLOC_MAX_CELLS 16777216
#define SWEHR_NOALLOC_MAX_BLOCKS 16384
int swehr_cfl_noalloc(const swehr_params *p, const double *d_h, const double *d_hu, const double *d_hv,
                      const double *d_zprev, int64_t pitch, double t, double *d_result, void *stream);

/* ---- scenario pool: many independent simulations stepped together ------
 * No reference counterpart (SWEHR.c runs one catchment per process).  Every
 * resident scenario advances one of its own time steps per pool step; one
 * pool step is two persistent launches over the tiles of all unfinished
 * scenarios (CUDA graphs of 32 steps), so scenarios of any mix of sizes share
 * the GPU.  Each scenario keeps its own dt, time, stage rows and budgets and
 * computes exactly what it computes alone.  A scenario is admitted only when
 * its device footprint fits the pool's HBM limit and a slot is free, stays
 * resident until its event ends (t >= tend), its step limit or an error, and
 * is read through the single-domain calls on the handle swehr_pool_scenario
 * returns.  All pool calls are synchronous and not thread-safe. */
typedef struct swehr_pool swehr_pool;

typedef struct {
    int32_t resident;        /* scenarios holding device memory */
    int32_t running;         /* resident and not yet finished */
    int32_t finished_now;    /* scenarios that finished during this call */
    int32_t tuned;           /* 1 once the launch shape has been chosen */
    int64_t pool_steps;      /* pool steps launched by this call */
    int64_t cell_steps;      /* cells x steps advanced by this call */
    double device_ms;        /* GPU time of this call */
    size_t hbm_used, hbm_limit;
    int32_t grid_wave, grid_update;   /* launch shape in use (blocks) */
    int32_t tile_i, tile_j;           /* tile shape in use (cells; 8 x 32 or 16 x 16) */
} swehr_pool_stats;

/* precision: SWEHR_FP64 or SWEHR_MIXED for every scenario; max_classes:
 * largest sclass admitted; budget: accumulate mass budgets for scenarios
 * that ask for them; hbm_limit: admission limit in bytes for scenario state
 * (0 = 90% of the device memory free now); max_scenarios: resident slots. */
int swehr_pool_create(int precision, int max_classes, int budget, size_t hbm_limit, int max_scenarios,
                      swehr_pool **out);

/* Upload a scenario (t = 0, initial state as swehr_create) and add it to the
 * batch; max_steps < 0 for no step limit.  SWEHR_BUSY when its footprint or
 * a slot is not free now (nothing allocated: retry after a release);
 * SWEHR_INVALID when it can never fit. */
int swehr_pool_submit(swehr_pool *pool, const swehr_params *p, const swehr_inputs *in, int64_t max_steps,
                      int *id);

/* Advance every running scenario by up to `steps` pool steps (< 0: until all
 * finish); returns after one synchronisation. */
int swehr_pool_run(swehr_pool *pool, int64_t steps, swehr_pool_stats *stats);

/* Launch-shape autotuner: times `steps_per_trial` real pool steps for each
 * candidate -- tile shape (8 x 32 or 16 x 16 cells) and persistent grid
 * (1..occupancy blocks per SM for each kernel) -- in three round-robin
 * passes, and keeps the shape and grids with the least time per running
 * cell; the scenarios advance meanwhile, with results that do not depend on
 * the candidate (bit for bit in the FP64 form). */
int swehr_pool_tune(swehr_pool *pool, int64_t steps_per_trial, swehr_pool_stats *stats);

/* progress of one scenario (status, done, t, steps) */
int swehr_pool_poll(swehr_pool *pool, int id, swehr_progress *pr);

/* The scenario's context for swehr_read_field / swehr_read_series /
 * swehr_get_budget / swehr_write_field (not for swehr_advance or
 * swehr_destroy). */
int swehr_pool_scenario(swehr_pool *pool, int id, swehr_ctx **ctx);

/* Free a scenario's device memory and slot (running or finished). */
int swehr_pool_release(swehr_pool *pool, int id);

int swehr_pool_stats_get(swehr_pool *pool, swehr_pool_stats *stats);

void swehr_pool_destroy(swehr_pool *pool);

/* ---- One domain split into row slabs (several devices, or several slabs of
 * one device).  No counterpart in the reference, whose loop body
 * (SWEHR.c:808-1591) runs serially over the whole grid; these replace the
 * same loop body for the rows row_lo..row_hi of the domain.  A step of row i
 * reads rows i-1..i+1 of the previous state and i-2..i+2 of the topography
 * (SWEHR.c:1135, 1203, 1243-1312), and the time step is one maximum over
 * every face of the grid (SWEHR.c:1408).  So a slab context holds its rows
 * plus up to two rows of each neighbour, updates only its own rows, and one
 * step is:
 *   swehr_slab_wave on every slab          largest wave speed of its faces
 *   maximum of those speeds, written back  (swehr_slab_smax_ptr: 8 bytes of
 *                                           device memory per slab, the bit
 *                                           pattern of a non-negative double,
 *                                           so an unsigned 64-bit max-reduce
 *                                           is the max of the speeds)
 *   swehr_slab_update on every slab        time step and update of its rows
 *   swehr_slab_pack / copy / unpack        its two edge rows of every state
 *                                           plane and of the new topography
 *                                           into the neighbours' halo rows
 * All calls are asynchronous on the slab's stream (swehr_slab_stream).
 * Whole-domain inputs and parameters are passed to swehr_slab_create, which
 * keeps the slab's rows.  Budgets, stage rows, interior solid cells and the
 * pool are not available for slabs (SWEHR_INVALID).  The slab's context
 * works with swehr_read_field (its local rows, halo rows included),
 * swehr_destroy and the calls below, not with swehr_advance. */
int swehr_slab_create(const swehr_params *p, const swehr_inputs *in, int precision, int row_lo, int row_hi,
                      swehr_ctx **out);

/* the slab's local rows: halo_lo rows above its own rows, then row_hi - row_lo + 1
 * own rows, then halo_hi rows (halo_lo, halo_hi in 0..2) */
int swehr_slab_rows(swehr_ctx *ctx, int *halo_lo, int *own, int *halo_hi);

int swehr_slab_wave(swehr_ctx *ctx);
int swehr_slab_smax_ptr(swehr_ctx *ctx, void **dev_ptr);
int swehr_slab_update(swehr_ctx *ctx);

/* Halo exchange buffers, one per side (0: toward row 1, 1: toward row nx),
 * each `bytes` long: pack fills both send buffers from the rows the step
 * just wrote, unpack writes both receive buffers into the halo rows.  A side
 * without a neighbour is neither packed nor unpacked. */
int swehr_slab_buffers(swehr_ctx *ctx, int side, void **send, void **recv, size_t *bytes);
int swehr_slab_pack(swehr_ctx *ctx);
int swehr_slab_unpack(swehr_ctx *ctx);

/* the slab's cudaStream_t */
int swehr_slab_stream(swehr_ctx *ctx, void **stream);

/* wait for the slab's stream and report t, steps, the last dt and Courant
 * number, status and done (no more steps: t >= tend or a CFL error) */
int swehr_slab_progress(swehr_ctx *ctx, swehr_progress *pr);

/* For slabs driven by one host thread: max-reduce the n slabs' wave speeds
 * into every slab, and copy slab a's send buffer of `side` into the
 * neighbour b's receive buffer (peer copy across devices); both order
 * themselves after the slabs' earlier work and before their later work. */
int swehr_slab_reduce_local(swehr_ctx *const *ctxs, int n);
int swehr_slab_copy_halo(swehr_ctx *a, int side, swehr_ctx *b);

#ifdef __cplusplus
}
#endif
#endif /* SWEHR_H */
