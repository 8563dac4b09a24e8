/*
 * swehr_slab.cu -- one domain split into slabs of whole rows (include/swehr.h,
 * swehr_slab_*).
 *
 * A slab context is an ordinary context over the slab's rows plus up to
 * HALO = 2 rows of each neighbour.  Its kernels update only its own rows
 * (DevParams own_lo..own_hi); the rows around them are read exactly as the
 * whole-domain kernels read them, because a step of row i reads rows i-1..i+1
 * of the previous state and rows i-2..i+2 of the topography (SWEHR.c:1135,
 * 1203, 1243-1312).  The wave pass leaves its largest speed in the control
 * block instead of computing dt (DevParams slab), so the caller can take the
 * maximum over every slab (SWEHR.c:1408) before k_slab_finalize computes the
 * same dt in every slab.  After the update each slab packs its first and last
 * two own rows of every state plane and of the new topography, the caller
 * moves them into the neighbours' receive buffers (NCCL, peer copies or
 * swehr_slab_copy_halo), and unpack writes them into the halo rows.
 * Compiled with --fmad=false like every FP64 kernel (the finalize divides).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "swehr_ctx.h"
#include "swehr_tile.cuh"

using namespace swehr;

namespace {

const int HALO = 2;

/* dt of the step from the largest speed over every slab, SWEHR.c:1409-1413 */
__global__ void k_slab_finalize(const DevParams P, Ctl *ctl)
{
    if (threadIdx.x == 0 && blockIdx.x == 0 && ctl->active) wave_finalize(P, ctl);
}

/* The planes of a state set as up to two blocks of equal-sized planes: the
 * plain form's set is one FP64 block, the mixed form's an FP32 block
 * followed by an FP64 block (swehr_device.cuh, swehr_capi.cu set_views). */
struct SetBlocks {
    char *base[2];
    int planes[2];
    int esize[2];
};

template <class RS>
__host__ __device__ inline SetBlocks set_blocks(const SetV<RS> &s, int S)
{
    SetBlocks b;
    if (sizeof(RS) == sizeof(double)) {
        b.base[0] = (char *)s.h; b.planes[0] = P_FIXED + 2 * S; b.esize[0] = 8;
        b.base[1] = nullptr; b.planes[1] = 0; b.esize[1] = 8;
    } else {
        b.base[0] = (char *)s.h; b.planes[0] = 9 + S; b.esize[0] = 4;
        b.base[1] = (char *)s.vinf; b.planes[1] = 1 + S; b.esize[1] = 8;
    }
    return b;
}

/* bytes of one side's buffer: HALO rows of every plane of a set and of z */
size_t halo_bytes_for(int ny, int S, bool mixed)
{
    const size_t per_row = mixed ? (size_t)(9 + S) * 4 + (size_t)(1 + S) * 8 + 8 : (size_t)(P_FIXED + 2 * S) * 8 + 8;
    return (size_t)HALO * ny * per_row;
}

/* Copy HALO rows of the set the last step wrote (and of its topography)
 * between the grid and a side's buffer.  pack: rows `row` .. row+1 -> buf;
 * otherwise buf -> rows.  Element e of the buffer runs over (block, plane,
 * row, column) in that order, then the topography rows. */
template <class RS>
__global__ void k_slab_rows(const DevParams P, const BufsT<RS> B, const Ctl *ctl, char *buf, int row, int pack)
{
    const int64_t n = ctl->step;
    const SetBlocks sb = set_blocks<RS>(B.set[n & 1], P.S);
    char *zb = (char *)B.z[n % 3];
    const int64_t ny = P.ny, rowel = HALO * ny;
    const int64_t e0 = (int64_t)sb.planes[0] * rowel, e1 = e0 + (int64_t)sb.planes[1] * rowel, e2 = e1 + rowel;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < e2; e += (int64_t)gridDim.x * blockDim.x) {
        char *grid_el;
        int64_t boff;
        int es;
        if (e < e1) {
            const int blk = e < e0 ? 0 : 1;
            const int64_t f = e - (blk ? e0 : 0);
            const int64_t p = f / rowel, rj = f - p * rowel, r = rj / ny, j = rj - r * ny;
            es = sb.esize[blk];
            grid_el = sb.base[blk] + ((int64_t)p * P.plane + (int64_t)(row - 1 + r) * P.pitch + j) * es;
            boff = (blk ? e0 * sb.esize[0] : 0) + f * es;
        } else {
            const int64_t f = e - e1, r = f / ny, j = f - r * ny;
            es = 8;
            grid_el = zb + ((int64_t)(row - 1 + r) * P.pitch + j) * 8;
            boff = e0 * sb.esize[0] + (int64_t)sb.planes[1] * rowel * sb.esize[1] + f * 8;
        }
        char *b = buf + boff;
        if (es == 8) {
            if (pack) *(double *)b = *(const double *)grid_el;
            else *(double *)grid_el = *(const double *)b;
        } else {
            if (pack) *(float *)b = *(const float *)grid_el;
            else *(float *)grid_el = *(const float *)b;
        }
    }
}

int check_slab(swehr_ctx *c)
{
    if (!c) return swehr_err(SWEHR_INVALID, "NULL ctx");
    if (!c->slab) return swehr_err(SWEHR_INVALID, "not a slab context (swehr_slab_create)");
    if (cudaSetDevice(c->device) != cudaSuccess) return swehr_err(SWEHR_CUDA_ERROR, "cudaSetDevice");
    return SWEHR_OK;
}

#define SCK(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return swehr_err(SWEHR_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

/* the pack (pack = 1) or unpack of both sides that have a neighbour */
int slab_rows(swehr_ctx *c, int pack)
{
    const int grid = 2 * c->num_sms;
    for (int side = 0; side < 2; side++) {
        if ((side == 0 ? c->halo_lo : c->halo_hi) == 0) continue;
        /* own edge rows to send, halo rows to receive */
        const int row = pack ? (side == 0 ? c->P.own_lo : c->P.own_hi - HALO + 1)
                             : (side == 0 ? c->P.own_lo - HALO : c->P.own_hi + 1);
        char *buf = c->d_halo + (size_t)(pack ? side : 2 + side) * c->halo_bytes;
        if (c->precision == SWEHR_MIXED)
            k_slab_rows<float><<<grid, 256, 0, c->stream>>>(c->P, c->B32, c->d_ctl, buf, row, pack);
        else
            k_slab_rows<double><<<grid, 256, 0, c->stream>>>(c->P, c->B64, c->d_ctl, buf, row, pack);
        SCK(cudaGetLastError());
    }
    return SWEHR_OK;
}

/* make stream `later` wait for what stream `earlier` has enqueued so far */
int order_after(cudaStream_t later, cudaStream_t earlier, int earlier_dev)
{
    cudaEvent_t ev;
    int cur = 0;
    SCK(cudaGetDevice(&cur));
    SCK(cudaSetDevice(earlier_dev));
    SCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    SCK(cudaEventRecord(ev, earlier));
    SCK(cudaSetDevice(cur));
    SCK(cudaStreamWaitEvent(later, ev, 0));
    SCK(cudaEventDestroy(ev));
    return SWEHR_OK;
}

}  // namespace

extern "C" {

int swehr_slab_create(const swehr_params *p, const swehr_inputs *in, int precision, int row_lo, int row_hi,
                      swehr_ctx **out)
{
    if (!out) return swehr_err(SWEHR_INVALID, "NULL out");
    *out = nullptr;
    if (!p || !in || !in->topo) return swehr_err(SWEHR_INVALID, "NULL params or inputs");
    const int nx = p->nx, ny = p->ny;
    if (row_lo < 1 || row_hi > nx || row_hi - row_lo + 1 < HALO)
        return swehr_err(SWEHR_INVALID, "slab rows must lie in 1..nx and number at least 2");
    if ((row_lo > 1 && row_lo < 1 + HALO) || (row_hi < nx && row_hi > nx - HALO))
        return swehr_err(SWEHR_INVALID, "every slab must own at least 2 rows (neighbours' rows 1..2 and nx-1..nx)");
    if (p->budget) return swehr_err(SWEHR_INVALID, "budgets are not available for slabs");
    if (in->solid) return swehr_err(SWEHR_INVALID, "interior solid cells are not available for slabs");
    const int hl = std::min(HALO, row_lo - 1), hh = std::min(HALO, nx - row_hi);
    const int a = row_lo - hl, b = row_hi + hh;     /* global rows held */
    swehr_params pl = *p;
    pl.nx = b - a + 1;
    swehr_inputs il = *in;
    const size_t off = (size_t)(a - 1) * ny;
    il.topo = in->topo + off;
    if (in->ks) il.ks = in->ks + off;
    swehr_ctx *c = nullptr;
    int rc = swehr_ctx_create(&pl, &il, precision, nullptr, &c);
    if (rc) return rc;
    c->slab = 1;
    c->halo_lo = hl;
    c->halo_hi = hh;
    c->P.own_lo = hl + 1;
    c->P.own_hi = hl + (row_hi - row_lo + 1);
    c->P.row0 = a - 1;
    c->P.slab = 1;
    c->halo_bytes = halo_bytes_for(ny, p->sclass, precision == SWEHR_MIXED);
    cudaError_t e = cudaMalloc((void **)&c->d_halo, 4 * c->halo_bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_halo, 0, 4 * c->halo_bytes, c->stream);
    if (e == cudaSuccess) {
        /* stepping armed, no stage rows (a slab holds part of the outlet row) */
        Ctl *h = c->h_ctl;
        h->active = p->tend > 0;
        h->pending = 0;
        h->max_step = INT64_MAX;
        h->t_stop = INFINITY;
        h->stagecap = 0;
        e = cudaMemcpyAsync(c->d_ctl, h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        swehr_ctx_destroy(c);
        return swehr_err(e == cudaErrorMemoryAllocation ? SWEHR_OOM : SWEHR_CUDA_ERROR,
                         std::string("slab set-up: ") + cudaGetErrorString(e));
    }
    *out = c;
    return SWEHR_OK;
}

int swehr_slab_rows(swehr_ctx *c, int *halo_lo, int *own, int *halo_hi)
{
    int rc = check_slab(c);
    if (rc) return rc;
    if (halo_lo) *halo_lo = c->halo_lo;
    if (own) *own = c->P.own_hi - c->P.own_lo + 1;
    if (halo_hi) *halo_hi = c->halo_hi;
    return SWEHR_OK;
}

int swehr_slab_wave(swehr_ctx *c)
{
    int rc = check_slab(c);
    if (rc) return rc;
    const int e = c->precision == SWEHR_MIXED ? launch_wave_f32(c->P, c->B32, c->d_ctl, c->cfg, c->stream)
                                              : launch_wave_f64(c->P, c->B64, c->d_ctl, c->cfg, c->stream);
    if (e) return swehr_err(SWEHR_CUDA_ERROR, std::string("wave: ") + cudaGetErrorString((cudaError_t)e));
    return SWEHR_OK;
}

int swehr_slab_smax_ptr(swehr_ctx *c, void **dev_ptr)
{
    int rc = check_slab(c);
    if (rc) return rc;
    if (!dev_ptr) return swehr_err(SWEHR_INVALID, "NULL dev_ptr");
    *dev_ptr = (void *)&c->d_ctl->smax_bits;
    return SWEHR_OK;
}

int swehr_slab_update(swehr_ctx *c)
{
    int rc = check_slab(c);
    if (rc) return rc;
    k_slab_finalize<<<1, 32, 0, c->stream>>>(c->P, c->d_ctl);
    SCK(cudaGetLastError());
    const int e = c->precision == SWEHR_MIXED
                      ? launch_update_f32(c->P, c->B32, c->d_ctl, c->d_rain, c->d_partials, c->d_stage, c->d_saveflow,
                                          c->tm, c->cfg, c->stream)
                      : launch_update_f64(c->P, c->B64, c->d_ctl, c->d_rain, c->d_partials, c->d_stage, c->d_saveflow,
                                          c->tm, c->cfg, c->stream);
    if (e) return swehr_err(SWEHR_CUDA_ERROR, std::string("update: ") + cudaGetErrorString((cudaError_t)e));
    return SWEHR_OK;
}

int swehr_slab_buffers(swehr_ctx *c, int side, void **send, void **recv, size_t *bytes)
{
    int rc = check_slab(c);
    if (rc) return rc;
    if (side != 0 && side != 1) return swehr_err(SWEHR_INVALID, "side must be 0 or 1");
    if (send) *send = c->d_halo + (size_t)side * c->halo_bytes;
    if (recv) *recv = c->d_halo + (size_t)(2 + side) * c->halo_bytes;
    if (bytes) *bytes = c->halo_bytes;
    return SWEHR_OK;
}

int swehr_slab_pack(swehr_ctx *c)
{
    int rc = check_slab(c);
    return rc ? rc : slab_rows(c, 1);
}

int swehr_slab_unpack(swehr_ctx *c)
{
    int rc = check_slab(c);
    return rc ? rc : slab_rows(c, 0);
}

int swehr_slab_progress(swehr_ctx *c, swehr_progress *pr)
{
    int rc = check_slab(c);
    if (rc) return rc;
    if (!pr) return swehr_err(SWEHR_INVALID, "NULL progress");
    SCK(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    SCK(cudaStreamSynchronize(c->stream));
    const Ctl *h = c->h_ctl;
    memset(pr, 0, sizeof *pr);
    pr->t = h->t;
    pr->dt = h->dt;
    pr->courant = h->courant;
    pr->rain = h->rain_now;
    pr->steps = h->step;
    pr->status = h->status;      /* the control block's codes are swehr_status values */
    pr->done = !h->active;
    pr->t_step = h->t_prev;
    return SWEHR_OK;
}

int swehr_slab_stream(swehr_ctx *c, void **stream)
{
    int rc = check_slab(c);
    if (rc) return rc;
    if (!stream) return swehr_err(SWEHR_INVALID, "NULL stream");
    *stream = (void *)c->stream;
    return SWEHR_OK;
}

int swehr_slab_reduce_local(swehr_ctx *const *ctxs, int n)
{
    if (!ctxs || n < 1) return swehr_err(SWEHR_INVALID, "need at least one slab");
    unsigned long long m = 0;
    std::vector<unsigned long long> v((size_t)n);
    for (int k = 0; k < n; k++) {
        int rc = check_slab(ctxs[k]);
        if (rc) return rc;
        SCK(cudaMemcpyAsync(&v[k], &ctxs[k]->d_ctl->smax_bits, 8, cudaMemcpyDeviceToHost, ctxs[k]->stream));
    }
    for (int k = 0; k < n; k++) {
        SCK(cudaSetDevice(ctxs[k]->device));
        SCK(cudaStreamSynchronize(ctxs[k]->stream));
        m = std::max(m, v[k]);      /* non-negative doubles: their bit patterns order as the values */
    }
    for (int k = 0; k < n; k++) {
        SCK(cudaSetDevice(ctxs[k]->device));
        SCK(cudaMemcpyAsync(&ctxs[k]->d_ctl->smax_bits, &m, 8, cudaMemcpyHostToDevice, ctxs[k]->stream));
    }
    for (int k = 0; k < n; k++) {    /* m lives on this stack frame: the copies finish before returning */
        SCK(cudaSetDevice(ctxs[k]->device));
        SCK(cudaStreamSynchronize(ctxs[k]->stream));
    }
    return SWEHR_OK;
}

int swehr_slab_copy_halo(swehr_ctx *a, int side, swehr_ctx *b)
{
    int rc = check_slab(a);
    if (!rc) rc = check_slab(b);
    if (rc) return rc;
    if (side != 0 && side != 1) return swehr_err(SWEHR_INVALID, "side must be 0 or 1");
    if (a->halo_bytes != b->halo_bytes) return swehr_err(SWEHR_INVALID, "slabs of different domains");
    if ((side == 0 ? a->halo_lo : a->halo_hi) == 0 || (side == 0 ? b->halo_hi : b->halo_lo) == 0)
        return swehr_err(SWEHR_INVALID, "no neighbour on that side");
    /* a's send buffer of `side` lands in b's receive buffer facing a */
    const char *src = a->d_halo + (size_t)side * a->halo_bytes;
    char *dst = b->d_halo + (size_t)(2 + (1 - side)) * b->halo_bytes;
    SCK(cudaSetDevice(b->device));
    rc = order_after(b->stream, a->stream, a->device);
    if (rc) return rc;
    SCK(cudaSetDevice(b->device));
    SCK(cudaMemcpyPeerAsync(dst, b->device, src, a->device, a->halo_bytes, b->stream));
    /* a may refill its send buffer only once the copy is done */
    SCK(cudaSetDevice(a->device));
    rc = order_after(a->stream, b->stream, b->device);
    if (rc) return rc;
    return SWEHR_OK;
}

}  // extern "C"
