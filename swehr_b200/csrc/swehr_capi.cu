/*
 * swehr_capi.cu -- host implementation of the C ABI in include/swehr.h.
 *
 * One context = one simulation on one device with its own stream.  All
 * device memory of a context is one allocation (state sets, topography
 * planes, Ks, rain, control block, reduction partials, stage rows), sized by
 * swehr_footprint_bytes().  Stepping is enqueued as CUDA graphs of whole
 * steps; the device decides when to stop (t >= tend, t_stop, step limit,
 * CFL error), so a bounded advance is one host synchronisation at the end.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/swehr.h"
#include "swehr_ctx.h"

using namespace swehr;

static thread_local std::string g_last_error;

int swehr_err(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

static int set_err(int code, const std::string &msg) { return swehr_err(code, msg); }

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return set_err(SWEHR_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

extern "C" {

void swehr_params_default(swehr_params *p)
{
    if (!p) return;
    memset(p, 0, sizeof *p);
    /* SWEHR.c:490-494 */
    p->hcfriction = 0.003; p->depthdependentexponent = -0.33; p->b = 1; p->af = 1; p->afr = 1;
    /* SWEHR.c:632-633 */
    p->cstable = 0.05; p->maxstep = 0.25;
    /* SWEHR.c:638-650 */
    p->g = 9.81; p->hfilm = 1e-5; p->phi = 0.4; p->rhos = 2600; p->rhow = 1000; p->nu = 1.2e-6;
    p->frictionangle = 0.8693; p->cohesion = 400; p->lambda = 0.65; p->cthreshold = 0.4; p->betabedload = 0.5;
    /* SWEHR.c:236-246 */
    p->roughness = 0.1; p->ks = 0; p->theta0 = 0.05; p->thetas = 0.4; p->hf = 0.001; p->vinf0 = 1e-4;
    p->uc = 0; p->uc2 = 0;
    /* SWEHR.c:617-621 */
    p->bndry[0] = 1; p->bndry[1] = 0; p->bndry[2] = 1; p->bndry[3] = 1;
    p->inflow = 1;
    /* SWEHR.c:629, 685, 709-715 */
    p->stageint = 1; p->outlet_row = 1; p->npoints = 6;
    const int yp[6] = {1, 10, 20, 30, 40, 50};
    for (int m = 0; m < 6; m++) { p->xpoint[m] = 2; p->ypoint[m] = yp[m]; }
    p->storm_radius = 1;
}

size_t swehr_params_size(void) { return sizeof(swehr_params); }
int swehr_abi_version(void) { return SWEHR_ABI_VERSION; }

const char *swehr_status_str(int s)
{
    switch (s) {
    case SWEHR_OK: return "ok";
    case SWEHR_CFL_ERROR: return "CFL error: Courant number > 1";
    case SWEHR_NAN: return "non-finite water depth";
    case SWEHR_TIMEOUT: return "host time limit reached";
    case SWEHR_CUDA_ERROR: return "CUDA error";
    case SWEHR_INVALID: return "invalid argument";
    case SWEHR_OOM: return "out of device memory";
    case SWEHR_NO_DEVICE: return "no CUDA device";
    case SWEHR_BUSY: return "busy";
    default: return "unknown status";
    }
}

const char *swehr_last_error(void) { return g_last_error.c_str(); }

/* lets other translation units of the library report an error message */
void swehr_set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

}  // extern "C"

static int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

/* Device layout of one simulation.  A state set is, in the plain form, 10 + 2S
 * double planes in the order h hu hv vinf maxvel maxdep totm dep totsed gz
 * U_1..U_S M_1..M_S; in the mixed form 9 + S float planes (h hu hv maxvel
 * maxdep totm dep totsed gz U_1..U_S) followed by 1 + S double planes (vinf
 * M_1..M_S).  Then three double z planes, the Ks plane (bulk type), rain,
 * control block, reduction partials and stage rows. */
struct Layout {
    int64_t pitch, plane;
    size_t rsize, set_bytes, off_z, off_ks, off_solid, off_z0, off_rain, off_ctl, off_partials, off_stage,
        off_saveflow, total;
};

/* ... with interior solid cells also the byte mask (one byte per plane
 * element) and the set-up topography plane, after the Ks plane */
static Layout layout_for(int nx, int ny, int S, int rnum, int has_ks, int has_solid, int64_t stagecap, int grid,
                         int precision)
{
    Layout L;
    L.pitch = round_up(ny, 32);
    L.plane = round_up((int64_t)nx * L.pitch, 32);
    L.rsize = precision == SWEHR_MIXED ? sizeof(float) : sizeof(double);
    const size_t pb = (size_t)L.plane * sizeof(double), pr = (size_t)L.plane * L.rsize;
    L.set_bytes = precision == SWEHR_MIXED ? (size_t)(9 + S) * pr + (size_t)(1 + S) * pb : (size_t)(P_FIXED + 2 * S) * pb;
    L.off_z = 2 * L.set_bytes;
    L.off_ks = L.off_z + 3 * pb;
    L.off_solid = (size_t)round_up((int64_t)(L.off_ks + (has_ks ? pr : 0)), 256);
    L.off_z0 = (size_t)round_up((int64_t)(L.off_solid + (has_solid ? (size_t)L.plane : 0)), 256);
    L.off_rain = L.off_z0 + (has_solid ? pb : 0);
    L.off_ctl = (size_t)round_up((int64_t)(L.off_rain + (size_t)rnum * sizeof(double)), 256);
    L.off_partials = (size_t)round_up((int64_t)(L.off_ctl + sizeof(Ctl)), 256);
    L.off_stage = (size_t)round_up((int64_t)(L.off_partials + (size_t)grid * B_NTERMS * sizeof(double)), 256);
    L.off_saveflow = L.off_stage + (size_t)stagecap * 24 * sizeof(double);
    L.total = (size_t)round_up((int64_t)(L.off_saveflow + (size_t)stagecap * 18 * sizeof(double)), 256);
    return L;
}

static int64_t stagecap_for(const swehr_params *p)
{
    double rows = p->stageint > 0 ? p->tend / p->stageint + 4 : 4;
    if (!(rows < 100000)) rows = 100000;
    return (int64_t)rows;
}

extern "C" size_t swehr_footprint_bytes(int nx, int ny, int sclass, int precision)
{
    return layout_for(nx, ny, sclass, 64, 1, 1, 4096, 148 * 4, precision).total;
}

static int validate(const swehr_params *p, const swehr_inputs *in)
{
    if (!p || !in) return set_err(SWEHR_INVALID, "NULL params or inputs");
    if (p->nx < 2 || p->ny < 2) return set_err(SWEHR_INVALID, "nx and ny must be >= 2");
    if (p->sclass < 1 || p->sclass > SWEHR_MAX_CLASSES) return set_err(SWEHR_INVALID, "sclass must be 1..16");
    if (p->rnum < 1) return set_err(SWEHR_INVALID, "rnum must be >= 1");
    if (!(p->dx > 0)) return set_err(SWEHR_INVALID, "dx must be > 0");
    if (!(p->rint > 0) && !(p->storm_peak > 0)) return set_err(SWEHR_INVALID, "rint must be > 0");
    for (int k = 0; k < 4; k++)
        if (p->bndry[k] != 0 && p->bndry[k] != 1) return set_err(SWEHR_INVALID, "bndry values must be 0 or 1");
    if (p->outlet_row < 1 || p->outlet_row > p->ny) return set_err(SWEHR_INVALID, "outlet_row outside 1..ny");
    if (p->storm_peak > 0 && !(p->storm_radius > 0)) return set_err(SWEHR_INVALID, "storm_radius must be > 0");
    if (!in->topo || !in->rain || !in->ds || !in->pfrac) return set_err(SWEHR_INVALID, "NULL input array");
    return SWEHR_OK;
}

/* initialcondition's topography fill around interior solid cells
 * (SWEHR.c:288-322): serial and in place, in the reference's order, so a
 * cell filled early is read by later ones exactly as there.  T and solid
 * are nx*ny, i-major. */
static void solid_fill_topography(int nx, int ny, const int32_t *solid, std::vector<double> &T)
{
    auto S = [&](int i, int j) { return solid[(size_t)(i - 1) * ny + (j - 1)] != 0; };
    auto Z = [&](int i, int j) -> double & { return T[(size_t)(i - 1) * ny + (j - 1)]; };
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            const int iup = std::min(i + 1, nx), idown = std::max(i - 1, 1);
            const int jup = std::min(j + 1, ny), jdown = std::max(j - 1, 1);
            if (S(i, j)) {
                if (!S(iup, j)) Z(i, j) = Z(iup, j);
                if (!S(idown, j)) Z(i, j) = Z(idown, j);
                if (!S(iup, jup)) Z(i, j) = Z(iup, jup);
                if (!S(iup, jdown)) Z(i, j) = Z(iup, jdown);
                if (!S(idown, jup)) Z(i, j) = Z(idown, jup);
                if (!S(idown, jdown)) Z(i, j) = Z(idown, jdown);
                if (!S(i, jup)) Z(i, j) = Z(i, jup);
                if (!S(i, jdown)) Z(i, j) = Z(i, jdown);
            }
            if (S(iup, j) && !S(i, j)) Z(iup, j) = Z(i, j);
            if (S(idown, j) && !S(i, j)) Z(idown, j) = Z(i, j);
            if (S(i, jup) && !S(i, j)) Z(i, jup) = Z(i, j);
            if (S(i, jdown) && !S(i, j)) Z(i, jdown) = Z(i, j);
        }
}

template <class R>
static void fill_realc(const DevParams &P, RealC<R> &K)
{
    K.g = (R)P.g; K.hfilm = (R)P.hfilm; K.hfx10 = (R)P.hfx10; K.rhos = (R)P.rhos; K.rhow = (R)P.rhow;
    K.rho0 = (R)P.rho0; K.porod = (R)P.porod; K.oneoverdx = (R)P.oneoverdx; K.half_odx = (R)P.half_odx;
    K.fa = (R)P.fa; K.cohesion = (R)P.cohesion; K.neg1ml = (R)P.neg1ml; K.cthreshold = (R)P.cthreshold;
    K.one_m_bb = (R)P.one_m_bb; K.hc = (R)P.hc; K.dde = (R)P.dde; K.b = (R)P.b; K.af = (R)P.af; K.afr = (R)P.afr;
    K.h0 = (R)P.h0; K.h0x3 = (R)P.h0x3; K.h0x6 = (R)P.h0x6; K.h0x9 = (R)P.h0x9; K.mtstar0 = (R)P.mtstar0;
    K.a = (R)P.a; K.ad = (R)P.ad; K.F = (R)P.F; K.J = (R)P.J; K.roughness = (R)P.roughness;
    K.uc = (R)P.uc; K.uc2 = (R)P.uc2; K.c109s = (R)P.c109s; K.rhos08 = (R)P.rhos08;
    for (int k = 0; k < 16; k++) {
        K.ds[k] = (R)P.ds[k]; K.pf[k] = (R)P.pf[k]; K.a13[k] = (R)P.a13[k]; K.a13sq[k] = (R)P.a13sq[k];
    }
}

static void make_devparams(const swehr_params *p, const swehr_inputs *in, const Layout &L, DevParams &P)
{
    memset(&P, 0, sizeof P);
    P.nx = p->nx; P.ny = p->ny; P.S = p->sclass; P.pitch = (int32_t)L.pitch;
    P.rnum = p->rnum; P.inflow = p->inflow ? 1 : 0; P.storm = p->storm_peak > 0; P.budget = p->budget ? 1 : 0;
    for (int k = 0; k < 4; k++) P.bndry[k] = p->bndry[k];
    P.outlet_row = p->outlet_row; P.npoints = p->npoints;
    for (int m = 0; m < 6; m++) { P.xpoint[m] = p->xpoint[m]; P.ypoint[m] = p->ypoint[m]; }
    P.has_ks = in->ks != nullptr;
    P.has_solid = in->solid != nullptr;
    P.own_lo = 1;
    P.own_hi = p->nx;
    P.row0 = 0;
    P.slab = 0;
    P.plane = L.plane;
    P.dx = p->dx; P.oneoverdx = 1 / p->dx; P.half_odx = 0.5 * P.oneoverdx; P.tend = p->tend; P.rint = p->rint;
    P.stageint = p->stageint;
    P.g = p->g; P.hfilm = p->hfilm; P.hfx10 = 10 * p->hfilm; P.rhos = p->rhos; P.rhow = p->rhow;
    P.rho0 = p->rhow * p->phi + p->rhos * (1 - p->phi);
    P.porod = p->rhos * (1 - p->phi);
    P.invporo = 1 / (p->rhos * (1 - p->phi));
    P.nu = p->nu; P.fa = p->frictionangle; P.cohesion = p->cohesion; P.neg1ml = -(1 - p->lambda);
    P.cthreshold = p->cthreshold; P.one_m_bb = 1 - p->betabedload; P.hc = p->hcfriction;
    P.dde = p->depthdependentexponent; P.b = p->b; P.af = p->af; P.afr = p->afr;
    P.h0 = p->h0; P.h0x3 = 3 * p->h0; P.h0x6 = 6 * p->h0; P.h0x9 = 9 * p->h0; P.mtstar0 = p->mtstar0;
    P.a = p->a; P.ad = p->ad; P.F = p->F; P.J = p->J;
    P.roughness = p->roughness; P.ks = p->ks; P.theta0 = p->theta0; P.thetas = p->thetas; P.hf = p->hf;
    P.uc = p->uc; P.uc2 = p->uc2; P.cstable = p->cstable; P.maxstep = p->maxstep;
    P.c109s = 1.09 * (p->rhos / p->rhow - 1);
    P.rhos08 = 0.8 * p->rhos;
    P.inv_rhos = 1.0 / p->rhos;
    P.inv_J = 1.0 / p->J;
    P.inv_h0x6 = 1.0 / P.h0x6;
    P.inv_p2 = 1.0 / 0.2;
    P.inv_dtheta = 1.0 / (p->thetas - p->theta0);
    {
        auto in_range = [](double c) { return c >= 0x1p-100 && c <= 0x1p100; };
        P.divk_ok = in_range(P.porod) && in_range(p->rhos) && in_range(p->J) && in_range(P.h0x6) &&
                    in_range(p->thetas - p->theta0);
    }
    P.storm_peak = p->storm_peak; P.storm_r2 = p->storm_radius * p->storm_radius;
    P.storm_x0 = p->storm_x0; P.storm_y0 = p->storm_y0; P.storm_vx = p->storm_vx; P.storm_vy = p->storm_vy;
    for (int k = 0; k < p->sclass; k++) {
        P.ds[k] = in->ds[k];
        P.pf[k] = in->pfrac[k];
        P.a13[k] = 13.95 * p->nu / in->ds[k];
        P.a13sq[k] = P.a13[k] * P.a13[k];
    }
    fill_realc(P, P.kd);
    fill_realc(P, P.kf);
}

/* one device plane: element size 8 (double) or 4 (float) */
struct PlaneRef {
    void *ptr;
    size_t esize;
};

static int upload_plane(swehr_ctx *c, PlaneRef d, const double *host, cudaStream_t s)
{
    const size_t N = (size_t)c->P.nx * c->P.ny;
    if (d.esize == sizeof(double)) {
        CK(cudaMemcpy2DAsync(d.ptr, (size_t)c->P.pitch * sizeof(double), host, (size_t)c->P.ny * sizeof(double),
                             (size_t)c->P.ny * sizeof(double), (size_t)c->P.nx, cudaMemcpyHostToDevice, s));
        return SWEHR_OK;
    }
    std::vector<float> tmp(N);
    for (size_t q = 0; q < N; q++) tmp[q] = (float)host[q];
    CK(cudaMemcpy2DAsync(d.ptr, (size_t)c->P.pitch * sizeof(float), tmp.data(), (size_t)c->P.ny * sizeof(float),
                         (size_t)c->P.ny * sizeof(float), (size_t)c->P.nx, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    return SWEHR_OK;
}

/* Rows of a device array (nrows x ncols elements of esize bytes, spitch
 * bytes apart) into contiguous host doubles.  Planes of 32 MB and more go
 * through two pinned 16 MB buffers, the device copy of one chunk overlapping
 * the host copy of the one before (a pageable destination is otherwise
 * filled at a fraction of the link's speed); smaller reads (a serving
 * request's) and pooled contexts return 0 without copying. */
static const size_t kStageBytes = (size_t)16 << 20;
static const size_t kStageMin = (size_t)32 << 20;

static void stage_part(double *dst, const void *src, size_t n, size_t esize)
{
    if (esize == sizeof(double)) {
        memcpy(dst, src, n * sizeof(double));
        return;
    }
    const float *f = (const float *)src;
    for (size_t q = 0; q < n; q++) dst[q] = (double)f[q];
}

/* the host side of a chunk, split over a few threads: filling fresh pageable
 * pages is bound by page faults, which proceed in parallel (half the host's
 * hardware threads, 2..8) */
static const int kStageThreadsMax = 8;

static int stage_threads()
{
    static const int T = std::max(2, std::min(kStageThreadsMax, (int)std::thread::hardware_concurrency() / 2));
    return T;
}

static void stage_out(double *dst, const void *src, size_t n, size_t esize)
{
    const int T = stage_threads();
    const size_t per = (n + T - 1) / T;
    std::thread th[kStageThreadsMax - 1];
    for (int t = 1; t < T; t++) {
        const size_t a = std::min(n, (size_t)t * per), b = std::min(n, a + per);
        th[t - 1] = std::thread(stage_part, dst + a, (const char *)src + a * esize, b - a, esize);
    }
    stage_part(dst, src, std::min(n, per), esize);
    for (int t = 0; t < T - 1; t++) th[t].join();
}

static int d2h_staged_copy(swehr_ctx *c, double *host, const void *dev, size_t spitch, size_t esize,
                           int64_t nrows, int64_t ncols);

static int d2h_staged(swehr_ctx *c, double *host, const void *dev, size_t spitch, size_t esize, int64_t nrows,
                      int64_t ncols, int *done)
{
    *done = 0;
    const size_t row_in = (size_t)ncols * esize;
    if (c->host || row_in * (size_t)nrows < kStageMin || row_in > kStageBytes) return SWEHR_OK;
    /* one pinned pair per process (pinning takes ~0.1 s), used by one read at a time */
    static std::mutex mu;
    static void *stage = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!stage) CK(cudaHostAlloc(&stage, 2 * kStageBytes, cudaHostAllocPortable));
    if (!c->ev_stage[0])
        for (int e = 0; e < 2; e++) CK(cudaEventCreateWithFlags(&c->ev_stage[e], cudaEventDisableTiming));
    c->h_stage = stage;
    const int rc = d2h_staged_copy(c, host, dev, spitch, esize, nrows, ncols);
    if (rc != SWEHR_OK) {
        /* a copy into the shared pinned pair may still be in flight: let it
         * land before the lock is released and the next reader reuses the pair */
        cudaStreamSynchronize(c->stream);
        return rc;
    }
    *done = 1;
    return SWEHR_OK;
}

/* the chunked copy of d2h_staged (its lock held, the pinned pair set up) */
static int d2h_staged_copy(swehr_ctx *c, double *host, const void *dev, size_t spitch, size_t esize,
                           int64_t nrows, int64_t ncols)
{
    const size_t row_in = (size_t)ncols * esize;
    const int64_t per = (int64_t)(kStageBytes / row_in);
    int64_t prev_r0 = -1, prev_n = 0;
    int prev_b = 0;
    int64_t k = 0;
    for (int64_t r0 = 0; r0 < nrows; r0 += per, k++) {
        const int64_t n = std::min(per, nrows - r0);
        const int b = (int)(k & 1);
        char *buf = (char *)c->h_stage + (size_t)b * kStageBytes;
        CK(cudaMemcpy2DAsync(buf, row_in, (const char *)dev + (size_t)r0 * spitch, spitch, row_in, (size_t)n,
                             cudaMemcpyDeviceToHost, c->stream));
        CK(cudaEventRecord(c->ev_stage[b], c->stream));
        if (prev_r0 >= 0) {
            CK(cudaEventSynchronize(c->ev_stage[prev_b]));
            stage_out(host + (size_t)prev_r0 * ncols, (char *)c->h_stage + (size_t)prev_b * kStageBytes,
                      (size_t)prev_n * ncols, esize);
        }
        prev_r0 = r0;
        prev_n = n;
        prev_b = b;
    }
    if (prev_r0 >= 0) {
        CK(cudaEventSynchronize(c->ev_stage[prev_b]));
        stage_out(host + (size_t)prev_r0 * ncols, (char *)c->h_stage + (size_t)prev_b * kStageBytes,
                  (size_t)prev_n * ncols, esize);
    }
    return SWEHR_OK;
}

/* the lagged GZ the wave pass of step n reads, from z of step n-1 */
static int init_gz(swehr_ctx *c, int64_t n)
{
    const int e = c->precision == SWEHR_MIXED ? init_gz_f32(c->P, c->B32, n, c->stream)
                                              : init_gz_f64(c->P, c->B64, n, c->stream);
    if (e) return set_err(SWEHR_CUDA_ERROR, std::string("init_gz: ") + cudaGetErrorString((cudaError_t)e));
    return SWEHR_OK;
}

static int download_plane(swehr_ctx *c, double *host, PlaneRef d, cudaStream_t s)
{
    const size_t N = (size_t)c->P.nx * c->P.ny;
    int staged = 0;
    int rc = d2h_staged(c, host, d.ptr, (size_t)c->P.pitch * d.esize, d.esize, c->P.nx, c->P.ny, &staged);
    if (rc || staged) return rc;
    if (d.esize == sizeof(double)) {
        CK(cudaMemcpy2DAsync(host, (size_t)c->P.ny * sizeof(double), d.ptr, (size_t)c->P.pitch * sizeof(double),
                             (size_t)c->P.ny * sizeof(double), (size_t)c->P.nx, cudaMemcpyDeviceToHost, s));
        return SWEHR_OK;
    }
    std::vector<float> tmp(N);
    CK(cudaMemcpy2DAsync(tmp.data(), (size_t)c->P.ny * sizeof(float), d.ptr, (size_t)c->P.pitch * sizeof(float),
                         (size_t)c->P.ny * sizeof(float), (size_t)c->P.nx, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (size_t q = 0; q < N; q++) host[q] = (double)tmp[q];
    return SWEHR_OK;
}

template <class RS>
static void set_views(BufsT<RS> &B, char *pool, const Layout &L, int S, int has_ks, int has_solid, int mixed)
{
    for (int s = 0; s < 2; s++) {
        char *base = pool + (size_t)s * L.set_bytes;
        SetV<RS> &v = B.set[s];
        const int64_t pl = L.plane;
        if (!mixed) {
            double *d = (double *)base;
            v.h = (RS *)(d + P_H * pl); v.hu = (RS *)(d + P_HU * pl); v.hv = (RS *)(d + P_HV * pl);
            v.vinf = d + P_VINF * pl;
            v.maxvel = (RS *)(d + P_MAXVEL * pl); v.maxdep = (RS *)(d + P_MAXDEP * pl);
            v.totm = (RS *)(d + P_TOTM * pl); v.dep = (RS *)(d + P_DEP * pl); v.totsed = (RS *)(d + P_TOTSED * pl);
            v.gz = (RS *)(d + P_GZ * pl);
            v.U = (RS *)(d + P_FIXED * pl);
            v.M = d + (P_FIXED + S) * pl;
        } else {
            RS *f = (RS *)base;
            v.h = f; v.hu = f + pl; v.hv = f + 2 * pl; v.maxvel = f + 3 * pl; v.maxdep = f + 4 * pl;
            v.totm = f + 5 * pl; v.dep = f + 6 * pl; v.totsed = f + 7 * pl; v.gz = f + 8 * pl; v.U = f + 9 * pl;
            double *d = (double *)(base + (size_t)(9 + S) * pl * sizeof(RS));
            v.vinf = d;
            v.M = d + pl;
        }
    }
    for (int k = 0; k < 3; k++) B.z[k] = (double *)(pool + L.off_z) + k * L.plane;
    B.ks = has_ks ? (const RS *)(pool + L.off_ks) : nullptr;
    B.solid = has_solid ? (const uint8_t *)(pool + L.off_solid) : nullptr;
    B.z0 = has_solid ? (const double *)(pool + L.off_z0) : nullptr;
}

/* a plane with v in its nx x ny cells and 0 in the row padding */
__global__ void k_fill_cells(double *__restrict__ p, int nx, int ny, int pitch, int64_t plane, double v)
{
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < plane; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q / pitch, j = q - i * pitch;
        p[q] = (i < nx && j < ny) ? v : 0.0;
    }
}

static void destroy_ctx(swehr_ctx *c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->ev_start) cudaEventDestroy(c->ev_start);
    if (c->ev_stop) cudaEventDestroy(c->ev_stop);
    for (int e = 0; e < 2 * TIMING_RING; e++)
        if (c->ev_k[e]) cudaEventDestroy(c->ev_k[e]);
    for (int e = 0; e < 2; e++)
        if (c->ev_stage[e]) cudaEventDestroy(c->ev_stage[e]);
    if (c->host) {
        if (c->mem) c->host->release(c->host->self, c->mem);
        free(c->h_ctl);
    } else {
        if (c->mem) cudaFree(c->mem);
        if (c->d_halo) cudaFree(c->d_halo);
        if (c->h_ctl) cudaFreeHost(c->h_ctl);
        if (c->stream) cudaStreamDestroy(c->stream);
    }
    delete c;
}

extern "C" int swehr_create(const swehr_params *p, const swehr_inputs *in, int precision, swehr_ctx **out)
{
    return swehr_ctx_create(p, in, precision, nullptr, out);
}

size_t swehr_ctx_footprint(const swehr_params *p, int has_ks, int has_solid, int precision, int num_sms)
{
    /* num_sms 0: a pooled context (one reduction slot; pools sum with atomics) */
    const int grid = num_sms > 0 ? num_sms * 4 : 1;
    return layout_for(p->nx, p->ny, p->sclass, p->rnum, has_ks, has_solid, stagecap_for(p), grid, precision).total;
}

int swehr_ctx_create(const swehr_params *p, const swehr_inputs *in, int precision, const CtxHost *host,
                     swehr_ctx **out)
{
    if (!out) return set_err(SWEHR_INVALID, "NULL out");
    *out = nullptr;
    int v = validate(p, in);
    if (v) return v;
    if (precision != SWEHR_FP64 && precision != SWEHR_MIXED) return set_err(SWEHR_INVALID, "unknown precision");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return set_err(SWEHR_NO_DEVICE, "no CUDA device");
    swehr_ctx *c = new swehr_ctx();
    c->p = *p;
    c->precision = precision;
    c->pooled = host != nullptr;
    c->host = host;
    const int pooled = c->pooled;
    int rc;
#define CKC(call)                                                                               \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            rc = set_err(e_ == cudaErrorMemoryAllocation ? SWEHR_OOM : SWEHR_CUDA_ERROR,        \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                   \
            destroy_ctx(c);                                                                     \
            return rc;                                                                          \
        }                                                                                       \
    } while (0)
    CKC(cudaGetDevice(&c->device));
    CKC(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device));
    c->stagecap = stagecap_for(p);
    DevParams tmpP;
    const int has_solid = in->solid != nullptr;
    Layout L0 = layout_for(p->nx, p->ny, p->sclass, p->rnum, in->ks != nullptr, has_solid, c->stagecap, 1, precision);
    make_devparams(p, in, L0, tmpP);
    if (!pooled) {
        /* the update loads its tiles through tensor maps when the driver
         * can encode them (checked again once the planes exist) */
        c->cfg.tma = tma_available();
        int ce = precision == SWEHR_MIXED ? configure_step_f32(tmpP, c->num_sms, c->cfg)
                                          : configure_step_f64(tmpP, c->num_sms, c->cfg);
        if (ce) {
            rc = set_err(SWEHR_CUDA_ERROR, std::string("configure: ") + cudaGetErrorString((cudaError_t)ce));
            destroy_ctx(c);
            return rc;
        }
    }
    Layout L = layout_for(p->nx, p->ny, p->sclass, p->rnum, in->ks != nullptr, has_solid, c->stagecap,
                          c->cfg.grid_update, precision);
    c->rsize = L.rsize;
    make_devparams(p, in, L, c->P);
    if (pooled) {
        c->stream = host->stream;
        c->mem = (char *)host->alloc(host->self, L.total);
        if (!c->mem) {
            rc = set_err(SWEHR_OOM, "scenario allocation failed");
            destroy_ctx(c);
            return rc;
        }
    } else {
        CKC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        CKC(cudaMalloc((void **)&c->mem, L.total));
    }
    c->mem_bytes = L.total;
    CKC(cudaMemsetAsync(c->mem, 0, L.total, c->stream));
    if (precision == SWEHR_MIXED) set_views(c->B32, c->mem, L, p->sclass, in->ks != nullptr, has_solid, 1);
    else set_views(c->B64, c->mem, L, p->sclass, in->ks != nullptr, has_solid, 0);
    if (c->cfg.tma && (precision == SWEHR_MIXED ? encode_tma_f32(c->P, c->B32, c->tm)
                                                : encode_tma_f64(c->P, c->B64, c->tm)) != 0) {
        c->cfg.tma = 0;      /* the maps were refused: stage with per-thread copies instead */
        const int grid = c->cfg.grid_update;    /* the reduction partials are sized for this many blocks */
        int ce = precision == SWEHR_MIXED ? configure_step_f32(c->P, c->num_sms, c->cfg)
                                          : configure_step_f64(c->P, c->num_sms, c->cfg);
        c->cfg.grid_update = std::min(c->cfg.grid_update, grid);
        if (ce) {
            rc = set_err(SWEHR_CUDA_ERROR, std::string("configure: ") + cudaGetErrorString((cudaError_t)ce));
            destroy_ctx(c);
            return rc;
        }
    }
    c->d_rain = (double *)(c->mem + L.off_rain);
    c->d_ctl = (Ctl *)(c->mem + L.off_ctl);
    c->d_partials = (double *)(c->mem + L.off_partials);
    c->d_stage = (double *)(c->mem + L.off_stage);
    c->d_saveflow = (double *)(c->mem + L.off_saveflow);
    if (pooled) {
        c->h_ctl = (Ctl *)calloc(1, sizeof(Ctl));
        if (!c->h_ctl) {
            rc = set_err(SWEHR_OOM, "host allocation failed");
            destroy_ctx(c);
            return rc;
        }
    } else {
        CKC(cudaMallocHost((void **)&c->h_ctl, sizeof(Ctl)));
    }
    if (!pooled) {
        CKC(cudaEventCreate(&c->ev_start));
        CKC(cudaEventCreate(&c->ev_stop));
    }
    if (!pooled)
        for (int e = 0; e < 2 * TIMING_RING; e++) CKC(cudaEventCreate(&c->ev_k[e]));
    /* initial state (initialcondition, SWEHR.c:211-285): dry bed, VINF = vinf0, z = topo;
     * z of the previous step = z (setup slopes, SWEHR.c:721-803) */
    double *const *zpl = precision == SWEHR_MIXED ? c->B32.z : c->B64.z;
    if (has_solid) {
        /* the mask, and the topography filled around solid cells as
         * initialcondition does (SWEHR.c:288-322); that filled topography is
         * also the set-up plane solid cells' slopes come from */
        const size_t N = (size_t)p->nx * p->ny;
        std::vector<double> topo(in->topo, in->topo + N);
        solid_fill_topography(p->nx, p->ny, in->solid, topo);
        rc = upload_plane(c, PlaneRef{zpl[0], sizeof(double)}, topo.data(), c->stream);
        if (rc) { destroy_ctx(c); return rc; }
        std::vector<uint8_t> m(N);
        for (size_t q = 0; q < N; q++) m[q] = in->solid[q] != 0;
        CKC(cudaMemcpy2DAsync(c->mem + L.off_solid, (size_t)c->P.pitch, m.data(), (size_t)p->ny, (size_t)p->ny,
                              (size_t)p->nx, cudaMemcpyHostToDevice, c->stream));
        CKC(cudaMemcpyAsync(c->mem + L.off_z0, zpl[0], (size_t)c->P.plane * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
        CKC(cudaStreamSynchronize(c->stream));      /* the host vectors go out of scope */
    } else {
        rc = upload_plane(c, PlaneRef{zpl[0], sizeof(double)}, in->topo, c->stream);
        if (rc) { destroy_ctx(c); return rc; }
    }
    for (int k = 1; k < 3; k++)     /* the other two z planes from the first, on the device */
        CKC(cudaMemcpyAsync(zpl[k], zpl[0], (size_t)c->P.plane * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    rc = init_gz(c, 0);
    if (rc) { destroy_ctx(c); return rc; }
    if (in->ks) {
        void *kp = precision == SWEHR_MIXED ? (void *)c->B32.ks : (void *)c->B64.ks;
        rc = upload_plane(c, PlaneRef{kp, L.rsize}, in->ks, c->stream);
        if (rc) { destroy_ctx(c); return rc; }
    }
    {
        double *vinf0 = precision == SWEHR_MIXED ? c->B32.set[0].vinf : c->B64.set[0].vinf;
        k_fill_cells<<<4 * 148, 256, 0, c->stream>>>(vinf0, p->nx, p->ny, c->P.pitch, c->P.plane, p->vinf0);
        CKC(cudaGetLastError());
        CKC(cudaMemcpyAsync(c->d_rain, in->rain, (size_t)p->rnum * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        Ctl h;
        memset(&h, 0, sizeof h);
        h.t = 0;
        h.stagecap = c->stagecap;
        h.t_stop = INFINITY;
        *c->h_ctl = h;
        CKC(cudaMemcpyAsync(c->d_ctl, c->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
        CKC(cudaStreamSynchronize(c->stream));
    }
    c->water_init = (double)p->nx * (double)p->ny * p->vinf0;
    *out = c;
    return SWEHR_OK;
#undef CKC
}

extern "C" void swehr_destroy(swehr_ctx *c)
{
    if (c && c->pooled) return;   /* owned by its pool: swehr_pool_release */
    destroy_ctx(c);
}

void swehr_ctx_destroy(swehr_ctx *c) { destroy_ctx(c); }

extern "C" int swehr_set_timing(swehr_ctx *c, int on)
{
    if (!c) return set_err(SWEHR_INVALID, "NULL ctx");
    if (c->pooled) return set_err(SWEHR_INVALID, "a pooled scenario is stepped by its pool");
    c->timing = on ? 1 : 0;
    return SWEHR_OK;
}

static int launch_step(swehr_ctx *c, cudaEvent_t ev0, cudaEvent_t ev1)
{
    if (c->precision == SWEHR_MIXED)
        return launch_step_f32(c->P, c->B32, c->d_ctl, c->d_rain, c->d_partials, c->d_stage, c->d_saveflow, c->tm,
                               c->cfg, c->stream, ev0, ev1);
    return launch_step_f64(c->P, c->B64, c->d_ctl, c->d_rain, c->d_partials, c->d_stage, c->d_saveflow, c->tm,
                           c->cfg, c->stream, ev0, ev1);
}

static int build_graph(swehr_ctx *c)
{
    if (c->graph) return SWEHR_OK;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < GRAPH_STEPS; s++) launch_step(c, nullptr, nullptr);
    CK(cudaStreamEndCapture(c->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&c->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_err(SWEHR_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return SWEHR_OK;
}

extern "C" int swehr_advance(swehr_ctx *c, double t_stop, int64_t max_steps, swehr_progress *pr)
{
    if (!c) return set_err(SWEHR_INVALID, "NULL ctx");
    if (c->pooled) return set_err(SWEHR_INVALID, "a pooled scenario is stepped by its pool");
    if (c->slab) return set_err(SWEHR_INVALID, "a slab is stepped by the swehr_slab_* calls");
    auto wall0 = std::chrono::steady_clock::now();
    /* read the control block, arm it */
    CK(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    Ctl *h = c->h_ctl;
    const int64_t step0 = h->step;
    if (h->status == SWEHR_CFL_ERROR) {
        if (pr) {
            memset(pr, 0, sizeof *pr);
            pr->t = h->t; pr->steps = h->step; pr->status = SWEHR_CFL_ERROR; pr->done = 1;
            pr->dt = h->dt; pr->courant = h->courant; pr->rain = h->rain_now; pr->t_step = h->t_prev;
        }
        return SWEHR_CFL_ERROR;
    }
    double kernel_ms = 0;
    int64_t launched = 0;
    bool run = h->t < c->p.tend && h->t < t_stop && max_steps != 0;
    if (run) {
        h->t_stop = t_stop;
        h->max_step = max_steps < 0 ? INT64_MAX : step0 + max_steps;
        h->active = 1;
        h->pending = 0;
        CK(cudaMemcpyAsync(c->d_ctl, h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
        CK(cudaEventRecord(c->ev_start, c->stream));
        if (c->timing) {
            int64_t left = max_steps;
            for (;;) {
                int n = TIMING_RING;
                if (max_steps >= 0 && left < n) n = (int)left;
                for (int s = 0; s < n; s++) {
                    int e = launch_step(c, c->ev_k[2 * s], c->ev_k[2 * s + 1]);
                    if (e) return set_err(SWEHR_CUDA_ERROR, std::string("launch: ") + cudaGetErrorString((cudaError_t)e));
                }
                launched += 2 * n;
                CK(cudaMemcpyAsync(h, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
                CK(cudaStreamSynchronize(c->stream));
                for (int s = 0; s < n; s++) {
                    float ms = 0;
                    CK(cudaEventElapsedTime(&ms, c->ev_k[2 * s], c->ev_k[2 * s + 1]));
                    kernel_ms += ms;
                }
                if (max_steps >= 0) left -= n;
                if (!h->active || (max_steps >= 0 && left <= 0)) break;
            }
        } else {
            int rcg = build_graph(c);
            if (rcg) return rcg;
            if (max_steps >= 0) {
                int64_t full = max_steps / GRAPH_STEPS, rem = max_steps % GRAPH_STEPS;
                for (int64_t gi = 0; gi < full; gi++) CK(cudaGraphLaunch(c->graph, c->stream));
                for (int64_t s = 0; s < rem; s++) launch_step(c, nullptr, nullptr);
                launched = 2 * max_steps;
                CK(cudaGetLastError());
                CK(cudaMemcpyAsync(h, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
                CK(cudaStreamSynchronize(c->stream));
            } else {
                for (;;) {
                    for (int gi = 0; gi < 4; gi++) CK(cudaGraphLaunch(c->graph, c->stream));
                    launched += 2 * 4 * GRAPH_STEPS;
                    CK(cudaMemcpyAsync(h, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
                    CK(cudaStreamSynchronize(c->stream));
                    if (!h->active) break;
                }
            }
        }
        CK(cudaEventRecord(c->ev_stop, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    float dev_ms = 0;
    if (run) CK(cudaEventElapsedTime(&dev_ms, c->ev_start, c->ev_stop));
    int st = h->status;
    (void)wall0;
    if (pr) {
        memset(pr, 0, sizeof *pr);
        pr->t = h->t; pr->dt = h->dt; pr->courant = h->courant;
        pr->rain = h->rain_now;
        pr->t_step = h->t_prev;
        pr->steps = h->step;
        pr->steps_this_call = h->step - step0;
        pr->device_ms = dev_ms;
        pr->kernel_ms = kernel_ms;
        pr->kernel_launches = launched;
        pr->status = st;
        pr->done = !(h->t < c->p.tend);
    }
    return st;
}

template <class RS>
static PlaneRef field_plane_t(const BufsT<RS> &B, int field, int k, int cur, int64_t pl)
{
    const SetV<RS> &v = B.set[cur];
    const size_t r = sizeof(RS), d = sizeof(double);
    switch (field) {
    case SWEHR_FIELD_H: return PlaneRef{v.h, r};
    case SWEHR_FIELD_HU: return PlaneRef{v.hu, r};
    case SWEHR_FIELD_HV: return PlaneRef{v.hv, r};
    case SWEHR_FIELD_VINF: return PlaneRef{v.vinf, d};
    case SWEHR_FIELD_MAXVEL: return PlaneRef{v.maxvel, r};
    case SWEHR_FIELD_MAXDEPTH: return PlaneRef{v.maxdep, r};
    case SWEHR_FIELD_TOTM: return PlaneRef{v.totm, r};
    case SWEHR_FIELD_DEP: return PlaneRef{v.dep, r};
    case SWEHR_FIELD_TOTSED: return PlaneRef{v.totsed, r};
    case SWEHR_FIELD_U: return PlaneRef{v.U + (k - 1) * pl, r};
    case SWEHR_FIELD_M: return PlaneRef{v.M + (k - 1) * pl, d};
    default: return PlaneRef{nullptr, 0};
    }
}

static PlaneRef field_plane(swehr_ctx *c, int field, int k, int cur)
{
    if (c->precision == SWEHR_MIXED) return field_plane_t(c->B32, field, k, cur, c->P.plane);
    return field_plane_t(c->B64, field, k, cur, c->P.plane);
}

static PlaneRef z_plane(swehr_ctx *c, int64_t m)
{
    double *const *z = c->precision == SWEHR_MIXED ? c->B32.z : c->B64.z;
    return PlaneRef{z[m % 3], sizeof(double)};
}

static int current_step(swehr_ctx *c, int64_t *step)
{
    CK(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *step = c->h_ctl->step;
    return SWEHR_OK;
}

/* |v| (d = hu, e = hv) or SED_k (d = U_k, e unused) of every cell, written
 * contiguously (nx rows of ny) in double: the reference's derived outputs
 * (SWEHR.c:1513-1520 SED_k = U_k/h clamped below -1e-5; vel.txt from hu/h,
 * hv/h).  Explicit round-to-nearest operations, so the values are the ones
 * the same expressions give on the host. */
template <class T>
__global__ void k_derived(const T *__restrict__ h, const T *__restrict__ d, const T *__restrict__ e, int nx, int ny,
                          int pitch, double hfilm, int vel, double *__restrict__ out)
{
    const int64_t N = (int64_t)nx * ny;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q / ny), j = (int)(q - (int64_t)i * ny);
        const int64_t r = (int64_t)i * pitch + j;
        const double hh = (double)h[r];
        double v;
        if (vel) {
            const double v1 = hh > hfilm ? __ddiv_rn((double)d[r], hh) : 0.0;
            const double v2 = hh > hfilm ? __ddiv_rn((double)e[r], hh) : 0.0;
            const double sq = __dsqrt_rn(__dadd_rn(__dmul_rn(v1, v1), __dmul_rn(v2, v2)));
            v = (sq == 0.0) ? 0.0 : sq;
        } else {
            const double sd = hh > hfilm ? __ddiv_rn((double)d[r], hh) : 0.0;
            v = (hh > hfilm && sd < -1e-5) ? 0.0 : sd;
        }
        out[q] = v;
    }
}

/* A derived field computed on the device and copied back once.  Its
 * scratch is the VINF plane (FP64 in both forms, plane >= nx*ny doubles) of
 * the state set the next step writes: between steps that set is dead, and
 * the next update rewrites every cell of it. */
static int read_derived(swehr_ctx *c, int field, int k, int cur, double *dst)
{
    const size_t N = (size_t)c->P.nx * c->P.ny;
    const bool vel = field == SWEHR_FIELD_VEL;
    const PlaneRef h = field_plane(c, SWEHR_FIELD_H, 0, cur);
    const PlaneRef d = field_plane(c, vel ? SWEHR_FIELD_HU : SWEHR_FIELD_U, k, cur);
    const PlaneRef e = vel ? field_plane(c, SWEHR_FIELD_HV, 0, cur) : h;
    const PlaneRef scratch = field_plane(c, SWEHR_FIELD_VINF, 0, cur ^ 1);
    if (scratch.esize != sizeof(double) || (size_t)c->P.plane < N) return set_err(SWEHR_INVALID, "derived-field scratch plane too small");
    double *tmp = (double *)scratch.ptr;
    const int grid = 4 * 148, threads = 256;
    if (h.esize == sizeof(double))
        k_derived<double><<<grid, threads, 0, c->stream>>>((const double *)h.ptr, (const double *)d.ptr,
                                                            (const double *)e.ptr, c->P.nx, c->P.ny, c->P.pitch,
                                                            c->P.hfilm, vel, tmp);
    else
        k_derived<float><<<grid, threads, 0, c->stream>>>((const float *)h.ptr, (const float *)d.ptr,
                                                           (const float *)e.ptr, c->P.nx, c->P.ny, c->P.pitch,
                                                           c->P.hfilm, vel, tmp);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
        int staged = 0;
        const int rc = d2h_staged(c, dst, tmp, (size_t)c->P.ny * sizeof(double), sizeof(double), c->P.nx, c->P.ny,
                                  &staged);
        if (rc) return rc;
        if (!staged) err = cudaMemcpyAsync(dst, tmp, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    }
    if (err != cudaSuccess) return set_err(SWEHR_CUDA_ERROR, std::string("derived field: ") + cudaGetErrorString(err));
    CK(cudaStreamSynchronize(c->stream));
    return SWEHR_OK;
}

extern "C" int swehr_read_field(swehr_ctx *c, int field, int k, double *dst)
{
    if (!c || !dst) return set_err(SWEHR_INVALID, "NULL argument");
    const int S = c->P.S;
    if ((field == SWEHR_FIELD_U || field == SWEHR_FIELD_M || field == SWEHR_FIELD_SED) && (k < 1 || k > S))
        return set_err(SWEHR_INVALID, "class index out of range");
    int64_t step;
    int rc = current_step(c, &step);
    if (rc) return rc;
    const int cur = (int)(step & 1);
    if (field == SWEHR_FIELD_Z) {
        rc = download_plane(c, dst, z_plane(c, step), c->stream);
    } else if (field == SWEHR_FIELD_VEL || field == SWEHR_FIELD_SED) {
        return read_derived(c, field, k, cur, dst);
    } else {
        PlaneRef src = field_plane(c, field, k, cur);
        if (!src.ptr) return set_err(SWEHR_INVALID, "unknown field");
        rc = download_plane(c, dst, src, c->stream);
    }
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return SWEHR_OK;
}

extern "C" int swehr_write_field(swehr_ctx *c, int field, int k, const double *src)
{
    if (!c || !src) return set_err(SWEHR_INVALID, "NULL argument");
    int64_t step;
    int rc = current_step(c, &step);
    if (rc) return rc;
    const int cur = (int)(step & 1);
    if (field == SWEHR_FIELD_Z) {
        rc = upload_plane(c, z_plane(c, step), src, c->stream);
        if (!rc) rc = upload_plane(c, z_plane(c, step + 2), src, c->stream);
        /* a written topography is a new set-up: solid cells take their slopes and GZ from it */
        const double *z0 = c->precision == SWEHR_MIXED ? c->B32.z0 : c->B64.z0;
        if (!rc && z0) rc = upload_plane(c, PlaneRef{const_cast<double *>(z0), sizeof(double)}, src, c->stream);
        if (!rc) rc = init_gz(c, step);
    } else {
        if ((field == SWEHR_FIELD_U || field == SWEHR_FIELD_M) && (k < 1 || k > c->P.S))
            return set_err(SWEHR_INVALID, "class index out of range");
        if (field == SWEHR_FIELD_VEL || field == SWEHR_FIELD_SED) return set_err(SWEHR_INVALID, "derived field");
        PlaneRef dstp = field_plane(c, field, k, cur);
        if (!dstp.ptr) return set_err(SWEHR_INVALID, "unknown field");
        rc = upload_plane(c, dstp, src, c->stream);
    }
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return SWEHR_OK;
}

extern "C" int swehr_read_series(swehr_ctx *c, double *stage, double *saveflow, int64_t max_rows, int64_t *rows)
{
    if (!c) return set_err(SWEHR_INVALID, "NULL ctx");
    int64_t step;
    int rc = current_step(c, &step);
    if (rc) return rc;
    int64_t n = c->h_ctl->stagecnt < max_rows ? c->h_ctl->stagecnt : max_rows;
    if (n > 0 && stage) CK(cudaMemcpyAsync(stage, c->d_stage, (size_t)n * 24 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (n > 0 && saveflow)
        CK(cudaMemcpyAsync(saveflow, c->d_saveflow, (size_t)n * 18 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (rows) *rows = n;
    return SWEHR_OK;
}

/* compensated (Neumaier) sum of a field over the interior */
static double sum_plane(const std::vector<double> &a)
{
    double s = 0, comp = 0;
    for (double v : a) {
        double t = s + v;
        if (std::fabs(s) >= std::fabs(v)) comp += (s - t) + v;
        else comp += (v - t) + s;
        s = t;
    }
    return s + comp;
}

extern "C" int swehr_get_budget(swehr_ctx *c, swehr_budget *b)
{
    if (!c || !b) return set_err(SWEHR_INVALID, "NULL argument");
    memset(b, 0, sizeof *b);
    const size_t N = (size_t)c->P.nx * c->P.ny;
    std::vector<double> h(N), vi(N), tmp(N), tmp2(N);
    int rc = swehr_read_field(c, SWEHR_FIELD_H, 0, h.data());
    if (!rc) rc = swehr_read_field(c, SWEHR_FIELD_VINF, 0, vi.data());
    if (rc) return rc;
    for (size_t q = 0; q < N; q++) tmp[q] = h[q];
    double wsum = sum_plane(tmp) + sum_plane(vi);
    const Ctl *H = c->h_ctl;
    auto term = [&](int m) { return H->budget_hi[m] + H->budget_lo[m]; };
    b->water_now = wsum;
    b->water_init = c->water_init;
    b->rain_in = term(B_RAIN);
    b->outflow = term(B_OUT);
    b->clamp_gain = term(B_CLAMP);
    b->bulking = term(B_BULK);
    b->infiltration = term(B_INF);
    b->rounding = term(B_ROUND);
    b->water_residual = (wsum - c->water_init) - (b->rain_in - b->outflow + b->clamp_gain + b->bulking + b->rounding);
    b->sclass = c->P.S;
    for (int k = 0; k < c->P.S; k++) {
        rc = swehr_read_field(c, SWEHR_FIELD_U, k + 1, tmp.data());
        if (!rc) rc = swehr_read_field(c, SWEHR_FIELD_M, k + 1, tmp2.data());
        if (rc) return rc;
        double s = sum_plane(tmp) + sum_plane(tmp2);
        b->sed_now[k] = s;
        b->sed_init[k] = c->sed_init[k];
        b->detach[k] = term(B_DET + k);
        b->sed_outflow[k] = term(B_SOUT + k);
        b->sed_rounding[k] = term(B_SROUND + k);
        b->sed_residual[k] = (s - c->sed_init[k]) - (b->detach[k] - b->sed_outflow[k] + b->sed_rounding[k]);
    }
    b->valid = c->P.budget;
    return SWEHR_OK;
}
