/*
 * swehr_pool.cu -- many independent scenarios stepped by shared launches
 * (the swehr_pool_* entry points of include/swehr.h).
 *
 * Each scenario is an ordinary context (own device allocation, control block,
 * stage rows, budgets) marked as pooled.  The pool keeps a device table of the
 * running scenarios (ScenDesc: parameters, buffer views, tile range) and a
 * header (table pointer, count, total tiles).  One pool step is
 * k_wave_batch + k_update_batch over the concatenated tile list, each a
 * persistent grid; the block that completes a scenario's last tile of a pass
 * finalizes that scenario (its dt, or its t / step / stage row / stop test),
 * so scenarios of any size mix advance one of their own steps per pool step
 * with no host round trip.  Steps are enqueued as CUDA graphs of GRAPH_STEPS
 * pool steps; the graph only holds the header's address, so it stays valid
 * while scenarios join and leave between calls.  After each call the
 * scenarios' summaries (t, dt, step, status, active) come back in one copy.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <map>
#include <unordered_map>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "swehr_ctx.h"

using namespace swehr;

namespace {

struct PoolScen {
    int id = -1;
    swehr_ctx *ctx = nullptr;
    size_t bytes = 0;
    int64_t ntiles = 0, cells = 0;
    int slot = -1;
    int running = 0;       /* unfinished as of the last synchronisation */
    int64_t step_seen = 0; /* steps completed as of the last synchronisation */
};

int64_t tiles_of(const DevParams &P, const BatchConfig &c)
{
    return (int64_t)((P.nx + c.tile_i - 1) / c.tile_i) * ((P.ny + c.tile_j - 1) / c.tile_j);
}

}  // namespace

struct swehr_pool {
    int device = 0, num_sms = 148, precision = SWEHR_FP64, max_classes = 1, budget = 0, max_scen = 0;
    size_t hbm_limit = 0, hbm_used = 0;
    BatchConfig cfg;                     /* the tile shape in use (a copy of shapes[shape]) */
    BatchConfig shapes[2];               /* 8 x 32 and 16 x 16 tiles */
    int shape = 0;
    int grid_wave = 0, grid_update = 0, tuned = 0;
    int kw_sel = 0, ku_sel = 0;          /* tuned blocks per SM (0: occupancy) */
    int max_s = 1;                       /* largest class count running */
    int min_s = 1;                       /* smallest class count running */
    size_t smem_update = 0;              /* update kernel's dynamic shared memory now */
    void *fn_update = nullptr;           /* update kernel now (staging choice for max_s) */
    cudaStream_t stream = nullptr;
    struct GraphEntry {
        size_t smem;
        int gw, gu;
        void *fn;
        cudaGraphExec_t exec;
    };
    std::vector<GraphEntry> graphs;      /* one per launch shape seen (class count x grids) */
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> ev_ring;   /* tuner: 3 events per step */
    char *d_hdr = nullptr, *h_hdr = nullptr;
    char *d_tab = nullptr, *h_tab = nullptr;
    size_t desc_bytes = 0;
    ScenSummary *d_sum = nullptr, *h_sum = nullptr;
    int32_t *d_map = nullptr, *h_map = nullptr;   /* tile -> scenario */
    int64_t map_cap = 0;
    std::vector<PoolScen> scen;
    std::vector<int> free_slots;
    /* device memory of scenarios: released allocations are kept for reuse
     * (within the HBM limit), so admission and release call no cudaMalloc /
     * cudaFree on the steady path */
    CtxHost host;
    std::multimap<size_t, char *> cache;          /* size -> released block */
    std::unordered_map<char *, size_t> block_size; /* every block the pool owns */
    size_t cached_bytes = 0;
    int next_id = 1;
    bool dirty = true;
    int nrun = 0;
    int64_t total_tiles = 0, running_cells = 0;
};

#define PCK(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return swehr_err(e_ == cudaErrorMemoryAllocation ? SWEHR_OOM : SWEHR_CUDA_ERROR,          \
                             std::string(#call) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

static const size_t kBlockGrain = (size_t)2 << 20;
/* the header allocation (256 bytes) holds the batch header at 0 and the two
 * tile counters of the batched passes here */
#define HDR_GRAB_OFFSET 128
static_assert(sizeof(BatchHdr<double>) <= HDR_GRAB_OFFSET, "header overlaps the tile counters");

/* keep resident + cached within the HBM limit: drop the largest cached blocks */
static void trim_cache(swehr_pool *pl, size_t incoming)
{
    while (!pl->cache.empty() && pl->hbm_used + pl->cached_bytes + incoming > pl->hbm_limit) {
        auto it = std::prev(pl->cache.end());
        cudaFree(it->second);
        pl->block_size.erase(it->second);
        pl->cached_bytes -= it->first;
        pl->cache.erase(it);
    }
}

/* a scenario's device memory: the smallest cached block of at least `bytes`
 * (and at most a quarter more), else a new one */
static void *pool_alloc(void *self, size_t bytes)
{
    swehr_pool *pl = (swehr_pool *)self;
    const size_t want = (bytes + kBlockGrain - 1) / kBlockGrain * kBlockGrain;
    auto it = pl->cache.lower_bound(want);
    if (it != pl->cache.end() && it->first <= want + want / 4) {
        char *p = it->second;
        pl->cached_bytes -= it->first;
        pl->cache.erase(it);
        return p;
    }
    trim_cache(pl, want);                /* room for a new block within the limit */
    char *p = nullptr;
    if (cudaMalloc((void **)&p, want) != cudaSuccess) {
        cudaGetLastError();
        for (auto &c : pl->cache) {          /* give the cache back and retry once */
            cudaFree(c.second);
            pl->block_size.erase(c.second);
        }
        pl->cache.clear();
        pl->cached_bytes = 0;
        if (cudaMalloc((void **)&p, want) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
    }
    pl->block_size[p] = want;
    return p;
}

static void pool_release_block(void *self, void *ptr)
{
    swehr_pool *pl = (swehr_pool *)self;
    char *p = (char *)ptr;
    auto it = pl->block_size.find(p);
    if (it == pl->block_size.end()) return;
    pl->cache.insert({it->second, p});
    pl->cached_bytes += it->second;
}

static void pool_free(swehr_pool *pl)
{
    if (!pl) return;
    if (pl->stream) cudaStreamSynchronize(pl->stream);
    for (auto &s : pl->scen) swehr_ctx_destroy(s.ctx);
    pl->scen.clear();
    for (auto &c : pl->cache) cudaFree(c.second);
    pl->cache.clear();
    for (auto &g : pl->graphs) cudaGraphExecDestroy(g.exec);
    if (pl->ev0) cudaEventDestroy(pl->ev0);
    if (pl->ev1) cudaEventDestroy(pl->ev1);
    for (cudaEvent_t e : pl->ev_ring) cudaEventDestroy(e);
    if (pl->d_hdr) cudaFree(pl->d_hdr);
    if (pl->d_tab) cudaFree(pl->d_tab);
    if (pl->d_sum) cudaFree(pl->d_sum);
    if (pl->d_map) cudaFree(pl->d_map);
    if (pl->h_map) cudaFreeHost(pl->h_map);
    if (pl->h_hdr) cudaFreeHost(pl->h_hdr);
    if (pl->h_tab) cudaFreeHost(pl->h_tab);
    if (pl->h_sum) cudaFreeHost(pl->h_sum);
    if (pl->stream) cudaStreamDestroy(pl->stream);
    delete pl;
}

template <class RS>
static void fill_desc(const PoolScen &s, const BufsT<RS> &B, ScenSummary *d_sum, int64_t tile0, ScenDesc<RS> *out)
{
    ScenDesc<RS> d;
    memset(&d, 0, sizeof d);
    d.P = s.ctx->P;
    d.B = B;
    d.ctl = s.ctx->d_ctl;
    d.rain = s.ctx->d_rain;
    d.stage = s.ctx->d_stage;
    d.saveflow = s.ctx->d_saveflow;
    d.sum = d_sum + s.slot;
    d.tile0 = tile0;
    d.ntiles = s.ntiles;
    memcpy(out, &d, sizeof d);
}

static void apply_shape(swehr_pool *pl);

/* write the running scenarios into the device table and header */
static int rebuild_table(swehr_pool *pl)
{
    int k = 0, max_s = 1, min_s = 16;
    int64_t tile0 = 0, cells = 0;
    for (auto &s : pl->scen) {
        if (!s.running) continue;
        max_s = std::max(max_s, (int)s.ctx->P.S);
        min_s = std::min(min_s, (int)s.ctx->P.S);
        s.ntiles = tiles_of(s.ctx->P, pl->cfg);     /* in the tile shape in use */
        char *slot = pl->h_tab + (size_t)k * pl->desc_bytes;
        if (pl->precision == SWEHR_MIXED)
            fill_desc<float>(s, s.ctx->B32, pl->d_sum, tile0, (ScenDesc<float> *)slot);
        else
            fill_desc<double>(s, s.ctx->B64, pl->d_sum, tile0, (ScenDesc<double> *)slot);
        tile0 += s.ntiles;
        cells += s.cells;
        k++;
    }
    /* tile -> scenario map (grown on demand; nothing is in flight here) */
    if (tile0 > pl->map_cap) {
        PCK(cudaStreamSynchronize(pl->stream));
        const int64_t cap = std::max(tile0, 2 * pl->map_cap);
        if (pl->d_map) cudaFree(pl->d_map);
        if (pl->h_map) cudaFreeHost(pl->h_map);
        pl->d_map = nullptr;
        pl->h_map = nullptr;
        pl->map_cap = 0;
        PCK(cudaMalloc((void **)&pl->d_map, (size_t)cap * sizeof(int32_t)));
        PCK(cudaMallocHost((void **)&pl->h_map, (size_t)cap * sizeof(int32_t)));
        pl->map_cap = cap;
    }
    {
        int64_t at = 0;
        int sid = 0;
        for (auto &s : pl->scen) {
            if (!s.running) continue;
            for (int64_t t = 0; t < s.ntiles; t++) pl->h_map[at + t] = sid;
            at += s.ntiles;
            sid++;
        }
    }
    BatchHdr<double> h;   /* same layout for both forms: pointers and counts */
    static_assert(sizeof(BatchHdr<double>) == sizeof(BatchHdr<float>), "header layout");
    memset(&h, 0, sizeof h);
    h.tab = (const ScenDesc<double> *)pl->d_tab;
    h.nscen = k;
    h.pad = 0;
    h.total_tiles = tile0;
    h.tile_scen = pl->d_map;
    h.grab = reinterpret_cast<unsigned long long *>(pl->d_hdr + HDR_GRAB_OFFSET);
    memcpy(pl->h_hdr, &h, sizeof h);
    if (k > 0) PCK(cudaMemcpyAsync(pl->d_tab, pl->h_tab, (size_t)k * pl->desc_bytes, cudaMemcpyHostToDevice, pl->stream));
    if (tile0 > 0)
        PCK(cudaMemcpyAsync(pl->d_map, pl->h_map, (size_t)tile0 * sizeof(int32_t), cudaMemcpyHostToDevice, pl->stream));
    PCK(cudaMemcpyAsync(pl->d_hdr, pl->h_hdr, sizeof h, cudaMemcpyHostToDevice, pl->stream));
    pl->nrun = k;
    pl->total_tiles = tile0;
    pl->running_cells = cells;
    pl->max_s = max_s;
    pl->min_s = std::min(min_s, max_s);
    pl->dirty = false;
    apply_shape(pl);
    return SWEHR_OK;
}

static void launch_pool_step(swehr_pool *pl, cudaEvent_t e0, cudaEvent_t e1, cudaEvent_t e2)
{
    void *args[] = {(void *)&pl->d_hdr};
    if (e0) cudaEventRecord(e0, pl->stream);
    cudaLaunchKernel(pl->cfg.fn_wave, dim3(pl->grid_wave), dim3(pl->cfg.threads), args, pl->cfg.smem_wave, pl->stream);
    if (e1) cudaEventRecord(e1, pl->stream);
    cudaLaunchKernel(pl->fn_update, dim3(pl->grid_update), dim3(pl->cfg.threads), args, pl->smem_update, pl->stream);
    if (e2) cudaEventRecord(e2, pl->stream);
}

/* The graph of GRAPH_STEPS pool steps for the current launch shape, built
 * on first use and kept: serving mixes change the largest class count (and
 * with it the staging size and grid) as scenarios come and go, and a shape
 * seen once is usually seen again. */
static int pool_graph(swehr_pool *pl, cudaGraphExec_t *out)
{
    for (auto &g : pl->graphs)
        if (g.smem == pl->smem_update && g.gw == pl->grid_wave && g.gu == pl->grid_update && g.fn == pl->fn_update) {
            *out = g.exec;
            return SWEHR_OK;
        }
    cudaGraph_t g;
    PCK(cudaStreamBeginCapture(pl->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < GRAPH_STEPS; s++) launch_pool_step(pl, nullptr, nullptr, nullptr);
    PCK(cudaStreamEndCapture(pl->stream, &g));
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return swehr_err(SWEHR_CUDA_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    pl->graphs.push_back({pl->smem_update, pl->grid_wave, pl->grid_update, pl->fn_update, ex});
    *out = ex;
    return SWEHR_OK;
}

static void set_grids(swehr_pool *pl, int kw, int ku)
{
    pl->grid_wave = pl->num_sms * kw;
    pl->grid_update = pl->num_sms * ku;
}

/* shared memory and grids for the scenarios running now: the update
 * kernel's staging is sized by the largest class count present, so a pool
 * that admits up to 16 classes still runs 7-class batches at the 7-class
 * occupancy */
/* the running scenarios all have the class count of a kernel built for
 * exactly that many classes */
static bool exact_classes(const swehr_pool *pl, const BatchConfig &c)
{
    return pl->min_s == pl->max_s && c.fn_update_x[pl->max_s] != nullptr;
}

static int update_occupancy(const swehr_pool *pl, const BatchConfig &c)
{
    return exact_classes(pl, c) ? c.occ_update_x[pl->max_s] : c.occ_update_s[pl->max_s];
}

static void apply_shape(swehr_pool *pl)
{
    const int S = pl->max_s;
    const bool exact = exact_classes(pl, pl->cfg);
    pl->smem_update = exact ? pl->cfg.smem_update_x[S] : pl->cfg.smem_update_s[S];
    pl->fn_update = exact ? pl->cfg.fn_update_x[S] : pl->cfg.fn_update_s[S];
    const int occ_u = update_occupancy(pl, pl->cfg);
    const int ku = pl->ku_sel ? std::min(pl->ku_sel, occ_u) : occ_u;
    const int kw = pl->kw_sel ? pl->kw_sel : pl->cfg.occ_wave;
    set_grids(pl, kw, ku);
}

/* copy the summaries back (after the stream's work) and fold them in */
static int collect(swehr_pool *pl, swehr_pool_stats *st)
{
    PCK(cudaMemcpyAsync(pl->h_sum, pl->d_sum, (size_t)pl->max_scen * sizeof(ScenSummary), cudaMemcpyDeviceToHost,
                        pl->stream));
    PCK(cudaStreamSynchronize(pl->stream));
    for (auto &s : pl->scen) {
        const ScenSummary &q = pl->h_sum[s.slot];
        if (st) st->cell_steps += (q.step - s.step_seen) * s.cells;
        s.step_seen = q.step;
        if (s.running && !q.active) {
            s.running = 0;
            pl->dirty = true;
            if (st) st->finished_now++;
        }
    }
    return SWEHR_OK;
}

static void fill_stats(swehr_pool *pl, swehr_pool_stats *st)
{
    st->resident = (int32_t)pl->scen.size();
    int r = 0;
    for (auto &s : pl->scen) r += s.running;
    st->running = r;
    st->tuned = pl->tuned;
    st->hbm_used = pl->hbm_used;
    st->hbm_limit = pl->hbm_limit;
    st->grid_wave = pl->grid_wave;
    st->grid_update = pl->grid_update;
    st->tile_i = pl->cfg.tile_i;
    st->tile_j = pl->cfg.tile_j;
}

static PoolScen *find(swehr_pool *pl, int id)
{
    for (auto &s : pl->scen)
        if (s.id == id) return &s;
    return nullptr;
}

extern "C" {

int swehr_pool_create(int precision, int max_classes, int budget, size_t hbm_limit, int max_scenarios,
                      swehr_pool **out)
{
    if (!out) return swehr_err(SWEHR_INVALID, "NULL out");
    *out = nullptr;
    if (precision != SWEHR_FP64 && precision != SWEHR_MIXED) return swehr_err(SWEHR_INVALID, "unknown precision");
    if (max_classes < 1 || max_classes > SWEHR_MAX_CLASSES) return swehr_err(SWEHR_INVALID, "max_classes must be 1..16");
    if (max_scenarios < 1 || max_scenarios > (1 << 20)) return swehr_err(SWEHR_INVALID, "max_scenarios must be 1..2^20");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return swehr_err(SWEHR_NO_DEVICE, "no CUDA device");
    swehr_pool *pl = new swehr_pool();
    pl->precision = precision;
    pl->max_classes = max_classes;
    pl->budget = budget ? 1 : 0;
    pl->max_scen = max_scenarios;
    /* the kernels index the table as ScenDesc<RS>[]: the host stride must be the struct size */
    pl->desc_bytes = precision == SWEHR_MIXED ? sizeof(ScenDesc<float>) : sizeof(ScenDesc<double>);
    int rc = SWEHR_OK;
#define PCKF(call)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            rc = swehr_err(e_ == cudaErrorMemoryAllocation ? SWEHR_OOM : SWEHR_CUDA_ERROR,            \
                           std::string(#call) + ": " + cudaGetErrorString(e_));                       \
            pool_free(pl);                                                                            \
            return rc;                                                                                \
        }                                                                                             \
    } while (0)
    PCKF(cudaGetDevice(&pl->device));
    PCKF(cudaDeviceGetAttribute(&pl->num_sms, cudaDevAttrMultiProcessorCount, pl->device));
    {
        const bool b = pl->budget != 0;
        int ce = precision == SWEHR_MIXED ? configure_batch_f32(max_classes, b, pl->shapes[0])
                                          : configure_batch_f64(max_classes, b, pl->shapes[0]);
        if (!ce)
            ce = precision == SWEHR_MIXED ? configure_batch_f32_t16(max_classes, b, pl->shapes[1])
                                          : configure_batch_f64_t16(max_classes, b, pl->shapes[1]);
        pl->cfg = pl->shapes[0];
        if (ce) {
            rc = swehr_err(SWEHR_CUDA_ERROR, std::string("configure: ") + cudaGetErrorString((cudaError_t)ce));
            pool_free(pl);
            return rc;
        }
    }
    PCKF(cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking));
    pl->host.stream = pl->stream;
    pl->host.self = pl;
    pl->host.alloc = pool_alloc;
    pl->host.release = pool_release_block;
    PCKF(cudaEventCreate(&pl->ev0));
    PCKF(cudaEventCreate(&pl->ev1));
    PCKF(cudaMalloc((void **)&pl->d_hdr, 256));
    PCKF(cudaMallocHost((void **)&pl->h_hdr, 256));
    PCKF(cudaMemsetAsync(pl->d_hdr, 0, 256, pl->stream));   /* tile counters start at 0 */
    PCKF(cudaMalloc((void **)&pl->d_tab, (size_t)max_scenarios * pl->desc_bytes));
    PCKF(cudaMallocHost((void **)&pl->h_tab, (size_t)max_scenarios * pl->desc_bytes));
    PCKF(cudaMalloc((void **)&pl->d_sum, (size_t)max_scenarios * sizeof(ScenSummary)));
    PCKF(cudaMallocHost((void **)&pl->h_sum, (size_t)max_scenarios * sizeof(ScenSummary)));
    memset(pl->h_sum, 0, (size_t)max_scenarios * sizeof(ScenSummary));
    PCKF(cudaMemsetAsync(pl->d_sum, 0, (size_t)max_scenarios * sizeof(ScenSummary), pl->stream));
    rc = rebuild_table(pl);
    if (rc) { pool_free(pl); return rc; }
    PCKF(cudaStreamSynchronize(pl->stream));
    if (hbm_limit == 0) {
        size_t fr = 0, tot = 0;
        PCKF(cudaMemGetInfo(&fr, &tot));
        hbm_limit = (size_t)(0.9 * (double)fr);
    }
    pl->hbm_limit = hbm_limit;
    for (int s = max_scenarios - 1; s >= 0; s--) pl->free_slots.push_back(s);
    *out = pl;
    return SWEHR_OK;
#undef PCKF
}

int swehr_pool_submit(swehr_pool *pl, const swehr_params *p, const swehr_inputs *in, int64_t max_steps, int *id)
{
    if (!pl || !p || !in || !id) return swehr_err(SWEHR_INVALID, "NULL argument");
    *id = -1;
    if (p->sclass > pl->max_classes) return swehr_err(SWEHR_INVALID, "sclass above the pool's max_classes");
    if (p->budget && !pl->budget) return swehr_err(SWEHR_INVALID, "pool created without budgets");
    if (p->nx < 2 || p->ny < 2 || p->sclass < 1) return swehr_err(SWEHR_INVALID, "nx, ny >= 2 and sclass >= 1 required");
    /* admission by the largest block this scenario can occupy (grain, reuse slack) */
    const size_t fp = swehr_ctx_footprint(p, in->ks != nullptr, in->solid != nullptr, pl->precision, 0);
    const size_t want = (fp + kBlockGrain - 1) / kBlockGrain * kBlockGrain;
    const size_t bytes = want + want / 4;
    if (bytes > pl->hbm_limit) return swehr_err(SWEHR_INVALID, "scenario footprint exceeds the pool's HBM limit");
    if (pl->free_slots.empty()) return swehr_err(SWEHR_BUSY, "no free scenario slot");
    if (pl->hbm_used + bytes > pl->hbm_limit) return swehr_err(SWEHR_BUSY, "HBM limit reached");
    swehr_ctx *c = nullptr;
    int rc = swehr_ctx_create(p, in, pl->precision, &pl->host, &c);
    if (rc) return rc;
    /* arm the control block: active from the first pool step on */
    Ctl *h = c->h_ctl;
    h->active = p->tend > 0 && max_steps != 0;
    h->pending = 0;
    h->max_step = max_steps < 0 ? INT64_MAX : max_steps;
    h->t_stop = INFINITY;
    cudaError_t e = cudaMemcpyAsync(c->d_ctl, h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        swehr_ctx_destroy(c);
        return swehr_err(SWEHR_CUDA_ERROR, std::string("arming: ") + cudaGetErrorString(e));
    }
    PoolScen s;
    s.id = pl->next_id++;
    s.ctx = c;
    s.bytes = pl->block_size.count(c->mem) ? pl->block_size[c->mem] : bytes;   /* what it holds */
    s.ntiles = tiles_of(c->P, pl->cfg);
    s.cells = (int64_t)p->nx * p->ny;
    s.slot = pl->free_slots.back();
    pl->free_slots.pop_back();
    s.running = h->active;
    s.step_seen = 0;
    ScenSummary q;
    memset(&q, 0, sizeof q);
    q.active = h->active;
    pl->h_sum[s.slot] = q;
    e = cudaMemcpyAsync(pl->d_sum + s.slot, &pl->h_sum[s.slot], sizeof q, cudaMemcpyHostToDevice, pl->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(pl->stream);
    if (e != cudaSuccess) {
        pl->free_slots.push_back(s.slot);
        swehr_ctx_destroy(c);
        return swehr_err(SWEHR_CUDA_ERROR, std::string("summary: ") + cudaGetErrorString(e));
    }
    pl->hbm_used += s.bytes;
    pl->scen.push_back(s);
    pl->dirty = true;
    *id = s.id;
    return SWEHR_OK;
}

int swehr_pool_run(swehr_pool *pl, int64_t steps, swehr_pool_stats *st)
{
    if (!pl) return swehr_err(SWEHR_INVALID, "NULL pool");
    swehr_pool_stats local;
    memset(&local, 0, sizeof local);
    if (pl->dirty) {
        int rc = rebuild_table(pl);
        if (rc) return rc;
    }
    float ms = 0;
    if (pl->nrun > 0 && steps != 0) {
        cudaGraphExec_t graph = nullptr;
        if (steps < 0 || steps >= GRAPH_STEPS) {
            int rc = pool_graph(pl, &graph);
            if (rc) return rc;
        }
        int rc = SWEHR_OK;
        PCK(cudaEventRecord(pl->ev0, pl->stream));
        if (steps > 0) {
            const int64_t full = steps / GRAPH_STEPS, rem = steps % GRAPH_STEPS;
            for (int64_t g = 0; g < full; g++) PCK(cudaGraphLaunch(graph, pl->stream));
            for (int64_t s = 0; s < rem; s++) launch_pool_step(pl, nullptr, nullptr, nullptr);
            PCK(cudaGetLastError());
            local.pool_steps = steps;
            PCK(cudaEventRecord(pl->ev1, pl->stream));
            rc = collect(pl, &local);
            if (rc) return rc;
        } else {
            for (;;) {
                for (int g = 0; g < 4; g++) PCK(cudaGraphLaunch(graph, pl->stream));
                local.pool_steps += 4 * GRAPH_STEPS;
                PCK(cudaEventRecord(pl->ev1, pl->stream));
                rc = collect(pl, &local);
                if (rc) return rc;
                bool any = false;
                for (auto &s : pl->scen) any = any || s.running;
                if (!any) break;
            }
        }
        PCK(cudaEventElapsedTime(&ms, pl->ev0, pl->ev1));
    }
    local.device_ms = ms;
    fill_stats(pl, &local);
    if (st) *st = local;
    return SWEHR_OK;
}

int swehr_pool_tune(swehr_pool *pl, int64_t steps_per_trial, swehr_pool_stats *st)
{
    if (!pl) return swehr_err(SWEHR_INVALID, "NULL pool");
    if (steps_per_trial < 1 || steps_per_trial > 4096) return swehr_err(SWEHR_INVALID, "steps_per_trial must be 1..4096");
    swehr_pool_stats local;
    memset(&local, 0, sizeof local);
    if (pl->dirty) {
        int rc = rebuild_table(pl);
        if (rc) return rc;
    }
    const size_t need = (size_t)3 * steps_per_trial;
    while (pl->ev_ring.size() < need) {
        cudaEvent_t e;
        PCK(cudaEventCreate(&e));
        pl->ev_ring.push_back(e);
    }
    /* Candidates: each tile shape with 1..occupancy blocks per SM for each
     * kernel.  Every candidate runs steps_per_trial real pool steps in each
     * of kRounds round-robin passes and keeps its best time per running cell
     * (cells, not tiles: the shapes cut the same scenarios into different
     * tile counts), so the state drifting between trials and one-off noise
     * do not decide.  A shape's best wave and update grids are chosen
     * separately; the shape with the smaller sum wins. */
    const int kRounds = 3;
    const int nsh = 2;
    int trials[2], occ_u[2];
    std::vector<std::pair<int, int>> cand;
    for (int sh = 0; sh < nsh; sh++) {
        occ_u[sh] = update_occupancy(pl, pl->shapes[sh]);
        trials[sh] = std::max(pl->shapes[sh].occ_wave, occ_u[sh]);
        for (int k = 1; k <= trials[sh]; k++) cand.push_back({sh, k});
    }
    std::vector<double> bw[2], bu[2];
    for (int sh = 0; sh < nsh; sh++) {
        bw[sh].assign((size_t)trials[sh] + 1, INFINITY);
        bu[sh].assign((size_t)trials[sh] + 1, INFINITY);
    }
    auto use_shape = [&](int sh) {
        if (pl->shape == sh) return;
        pl->shape = sh;
        pl->cfg = pl->shapes[sh];
        pl->dirty = true;                /* tile counts change: rebuild the table */
    };
    for (int trial = 0; trial < kRounds * (int)cand.size(); trial++) {
        const int sh = cand[trial % cand.size()].first, k = cand[trial % cand.size()].second;
        use_shape(sh);
        if (pl->dirty) {
            int rc = rebuild_table(pl);
            if (rc) return rc;
        }
        if (pl->nrun == 0) break;
        const int kw = std::min(k, pl->cfg.occ_wave), ku = std::min(k, occ_u[sh]);
        set_grids(pl, kw, ku);
        const double cells = (double)std::max<int64_t>(pl->running_cells, 1);
        for (int64_t s = 0; s < steps_per_trial; s++)
            launch_pool_step(pl, pl->ev_ring[3 * s], pl->ev_ring[3 * s + 1], pl->ev_ring[3 * s + 2]);
        PCK(cudaGetLastError());
        local.pool_steps += steps_per_trial;
        int rc = collect(pl, &local);
        if (rc) return rc;
        double w = 0, u = 0;
        for (int64_t s = 0; s < steps_per_trial; s++) {
            float a = 0, b = 0;
            PCK(cudaEventElapsedTime(&a, pl->ev_ring[3 * s], pl->ev_ring[3 * s + 1]));
            PCK(cudaEventElapsedTime(&b, pl->ev_ring[3 * s + 1], pl->ev_ring[3 * s + 2]));
            w += a;
            u += b;
        }
        local.device_ms += w + u;
        if (kw == k) bw[sh][k] = std::min(bw[sh][k], w / cells);
        if (ku == k) bu[sh][k] = std::min(bu[sh][k], u / cells);
    }
    int best_sh = 0, kw_best[2], ku_best[2];
    double best_t = INFINITY;
    for (int sh = 0; sh < nsh; sh++) {
        kw_best[sh] = pl->shapes[sh].occ_wave;
        ku_best[sh] = occ_u[sh];
        for (int k = 1; k <= trials[sh]; k++) {
            if (bw[sh][k] < bw[sh][kw_best[sh]]) kw_best[sh] = k;
            if (bu[sh][k] < bu[sh][ku_best[sh]]) ku_best[sh] = k;
        }
        const double t = bw[sh][kw_best[sh]] + bu[sh][ku_best[sh]];
        if (t < best_t) {
            best_t = t;
            best_sh = sh;
        }
    }
    use_shape(best_sh);
    pl->kw_sel = kw_best[best_sh];
    pl->ku_sel = ku_best[best_sh];
    if (pl->dirty) {
        int rc = rebuild_table(pl);
        if (rc) return rc;
    }
    set_grids(pl, pl->kw_sel, std::min(pl->ku_sel, occ_u[best_sh]));
    pl->tuned = 1;
    fill_stats(pl, &local);
    if (st) *st = local;
    return SWEHR_OK;
}

int swehr_pool_poll(swehr_pool *pl, int id, swehr_progress *pr)
{
    if (!pl || !pr) return swehr_err(SWEHR_INVALID, "NULL argument");
    PoolScen *s = find(pl, id);
    if (!s) return swehr_err(SWEHR_INVALID, "unknown scenario id");
    const ScenSummary &q = pl->h_sum[s->slot];
    memset(pr, 0, sizeof *pr);
    pr->t = q.t;
    pr->dt = q.dt;
    pr->courant = q.courant;
    pr->steps = q.step;
    pr->status = q.status;
    pr->done = !s->running;
    return SWEHR_OK;
}

int swehr_pool_scenario(swehr_pool *pl, int id, swehr_ctx **ctx)
{
    if (!pl || !ctx) return swehr_err(SWEHR_INVALID, "NULL argument");
    PoolScen *s = find(pl, id);
    if (!s) return swehr_err(SWEHR_INVALID, "unknown scenario id");
    *ctx = s->ctx;
    return SWEHR_OK;
}

int swehr_pool_release(swehr_pool *pl, int id)
{
    if (!pl) return swehr_err(SWEHR_INVALID, "NULL pool");
    for (size_t k = 0; k < pl->scen.size(); k++) {
        if (pl->scen[k].id != id) continue;
        PCK(cudaStreamSynchronize(pl->stream));
        PoolScen s = pl->scen[k];
        pl->scen.erase(pl->scen.begin() + (long)k);
        swehr_ctx_destroy(s.ctx);
        pl->free_slots.push_back(s.slot);
        pl->hbm_used -= s.bytes;
        if (s.running) pl->dirty = true;
        return SWEHR_OK;
    }
    return swehr_err(SWEHR_INVALID, "unknown scenario id");
}

int swehr_pool_stats_get(swehr_pool *pl, swehr_pool_stats *st)
{
    if (!pl || !st) return swehr_err(SWEHR_INVALID, "NULL argument");
    memset(st, 0, sizeof *st);
    fill_stats(pl, st);
    return SWEHR_OK;
}

void swehr_pool_destroy(swehr_pool *pl) { pool_free(pl); }

}  // extern "C"
