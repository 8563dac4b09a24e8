/*
 * swehr_cfl_noalloc.cu -- the CFL time step of one state, computed without
 * allocating any memory.
 *
 * Who needs this: a caller that must not (or cannot) call cudaMalloc -- for
 * example a host framework that owns every device allocation through its
 * own pool, a plugin that runs where the allocator is locked, or code that
 * must keep the device's allocation state unchanged between checkpoints.
 * Such a caller owns the state planes and the result buffer; this entry point
 * only launches a kernel.
 *
 * Scratch: the kernel needs one partial maximum per block and a ticket
 * counter.  They live in the file-scope array g_cfl_scratch below, which
 * every GPU that loads the library holds until the process exits
 * (SWEHR_NOALLOC_MAX_BLOCKS doubles + 256 bytes = 128.25 KiB).  With 1024
 * cells per block that bounds the domain at SWEHR_NOALLOC_MAX_CELLS =
 * 16,777,216 cells (4096 x 4096); larger domains are rejected.
 *
 * The array's name in host code is a host-side stand-in, not a device
 * address: its device address is looked up with cudaGetSymbolAddress, once
 * per device, with that device current, on the first call made on that
 * device.  Make that first call before any stream capture begins.
 *
 * Every call shares the one array and it keeps the last call's contents:
 * the ticket counter is cleared (cudaMemsetAsync on the caller's stream)
 * before each launch, and calls that overlap on the GPU -- two streams, or
 * two host threads on one device -- race on it and give wrong results.
 * Serialise them.
 */
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/swehr.h"
#include "swehr_tile.cuh"

namespace swehr {

static const int NOALLOC_CELLS_PER_BLOCK = 1024;

/* [0, SWEHR_NOALLOC_MAX_BLOCKS): per-block maxima; then the ticket counter (256-byte slot) */
static __device__ __align__(256) double g_cfl_scratch[SWEHR_NOALLOC_MAX_BLOCKS + 32];

__global__ void __launch_bounds__(NB_THREADS) k_cfl_noalloc(const DevParams P, const double *__restrict__ h,
                                                             const double *__restrict__ hu,
                                                             const double *__restrict__ hv,
                                                             const double *__restrict__ zp, double t,
                                                             double *scratch, double *result)
{
    /* The faces each cell owns and their wave speeds are those of the
     * stepping path's wave pass (wave_cell_g, one definition); only the
     * cell's lagged GZ comes from the caller's previous-step topography
     * instead of the state's GZ plane. */
    double inh = 0, inhv = 0, insed = 0;
    if (P.inflow) inflow_ghost(t, inh, inhv, insed);
    SetV<double> src{};
    src.h = const_cast<double *>(h);
    src.hu = const_cast<double *>(hu);
    src.hv = const_cast<double *>(hv);
    const int64_t total = (int64_t)P.nx * P.ny;
    const int64_t first = (int64_t)blockIdx.x * NOALLOC_CELLS_PER_BLOCK;
    double smax = 0;
    for (int64_t c = first + threadIdx.x; c < first + NOALLOC_CELLS_PER_BLOCK && c < total; c += blockDim.x) {
        const int i = (int)(c / P.ny) + 1, j = (int)(c % P.ny) + 1;
        const double s = wave_cell_g<PolicyF64, double>(P, src, i, j, inh, inhv, lagged_gz<PolicyF64>(P, zp, i, j));
        smax = (s > smax) ? s : smax;
    }
    __shared__ double red[NB_THREADS / 32];
    __shared__ bool last;
    smax = warp_max(smax);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = smax;
    __syncthreads();
    unsigned int *ticket = reinterpret_cast<unsigned int *>(scratch + SWEHR_NOALLOC_MAX_BLOCKS);
    if (threadIdx.x == 0) {
        double m = 0;
        for (int w = 0; w < NB_THREADS / 32; w++) m = (red[w] > m) ? red[w] : m;
        scratch[blockIdx.x] = m;
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double Smax = 0;
    for (unsigned b = 0; b < gridDim.x; b++) {
        double v = ((volatile double *)scratch)[b];
        Smax = (v > Smax) ? v : Smax;
    }
    /* SWEHR.c:1409-1411 */
    double dt = P.cstable * P.dx / Smax;
    if (dt > P.maxstep) dt = P.maxstep;
    if (t + dt > P.tend) dt = P.tend - t;
    result[0] = Smax;
    result[1] = dt;
    *ticket = 0u;
}

}  // namespace swehr

using namespace swehr;

static std::mutex g_noalloc_mu;
static double *g_noalloc_addr[64];

extern "C" void swehr_set_last_error(const char *msg);

static int noalloc_err(int code, const char *msg)
{
    swehr_set_last_error(msg);
    return code;
}

extern "C" int swehr_cfl_noalloc(const swehr_params *p, const double *d_h, const double *d_hu, const double *d_hv,
                                 const double *d_zprev, int64_t pitch, double t, double *d_result, void *stream)
{
    if (!p || !d_h || !d_hu || !d_hv || !d_zprev || !d_result)
        return noalloc_err(SWEHR_INVALID, "swehr_cfl_noalloc: NULL argument");
    if (p->nx < 2 || p->ny < 2 || pitch < p->ny)
        return noalloc_err(SWEHR_INVALID, "swehr_cfl_noalloc: need nx, ny >= 2 and pitch >= ny");
    /* the kernel indexes rows with a 32-bit pitch: nx rows of it must stay addressable */
    if (pitch > INT32_MAX || (int64_t)p->nx > INT64_MAX / pitch)
        return noalloc_err(SWEHR_INVALID, "swehr_cfl_noalloc: pitch exceeds INT32_MAX (or nx*pitch overflows)");
    if ((int64_t)p->nx * p->ny > SWEHR_NOALLOC_MAX_CELLS)
        return noalloc_err(SWEHR_INVALID, "swehr_cfl_noalloc: nx*ny exceeds SWEHR_NOALLOC_MAX_CELLS (16777216), "
                                          "the size its fixed scratch array can reduce");
    for (int k = 0; k < 4; k++)
        if (p->bndry[k] != 0 && p->bndry[k] != 1) return noalloc_err(SWEHR_INVALID, "swehr_cfl_noalloc: bndry must be 0/1");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return noalloc_err(SWEHR_NO_DEVICE, "swehr_cfl_noalloc: no current CUDA device");
    double *scratch;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void *a = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&a, g_cfl_scratch);
            if (e != cudaSuccess || !a) return noalloc_err(SWEHR_CUDA_ERROR, "swehr_cfl_noalloc: cudaGetSymbolAddress failed");
            g_noalloc_addr[dev] = (double *)a;
        }
        scratch = g_noalloc_addr[dev];
    }
    DevParams P;
    memset(&P, 0, sizeof P);
    P.nx = p->nx; P.ny = p->ny; P.pitch = (int32_t)pitch;
    P.inflow = p->inflow ? 1 : 0;
    for (int k = 0; k < 4; k++) P.bndry[k] = p->bndry[k];
    P.dx = p->dx; P.oneoverdx = 1 / p->dx; P.half_odx = 0.5 * P.oneoverdx; P.tend = p->tend;
    P.g = p->g; P.hfilm = p->hfilm; P.cstable = p->cstable; P.maxstep = p->maxstep;
    P.kd.g = p->g; P.kd.hfilm = p->hfilm;   /* the constants the per-cell wave routine reads */
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t total = (int64_t)p->nx * p->ny;
    const int grid = (int)((total + NOALLOC_CELLS_PER_BLOCK - 1) / NOALLOC_CELLS_PER_BLOCK);
    if (cudaMemsetAsync(scratch + SWEHR_NOALLOC_MAX_BLOCKS, 0, 256, s) != cudaSuccess)
        return noalloc_err(SWEHR_CUDA_ERROR, "swehr_cfl_noalloc: clearing the scratch ticket failed");
    k_cfl_noalloc<<<grid, NB_THREADS, 0, s>>>(P, d_h, d_hu, d_hv, d_zprev, t, scratch, d_result);
    if (cudaGetLastError() != cudaSuccess) return noalloc_err(SWEHR_CUDA_ERROR, "swehr_cfl_noalloc: launch failed");
    return SWEHR_OK;
}
