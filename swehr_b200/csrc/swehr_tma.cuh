/*
 * swehr_tma.cuh -- tile loads through the tensor memory accelerator for the
 * update kernel of one domain (both forms).
 *
 * The staging of a tile (its halo planes, the two topography windows and
 * the cell planes, see swehr_tile.cuh) is a handful of rectangular boxes of
 * HBM planes.  With tensor maps of those planes one thread issues one
 * cp.async.bulk.tensor per box instead of every thread issuing 16-byte
 * copies with its own address arithmetic; the copies complete on a shared-memory
 * mbarrier that carries the byte count, and parts of a box outside the grid
 * arrive as zeros (no cell reads them: ghost cells take their source cell's
 * values).  Loads only, from this GPU's own memory, no cluster multicast.
 *
 * Every wait on the mbarrier gives up after a bounded number of polls and
 * reports it through the control block (the step then ends with
 * SWEHR_TIMEOUT) instead of spinning forever.
 */
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace swehr {

/* tensor maps of one simulation, passed to the update kernel as a
 * __grid_constant__ parameter.  The halo and cell maps cover the set's
 * planes of its storage type (every plane in the plain form, the FP32 block
 * in the mixed form), the CELLD maps its FP64 planes. */
enum {
    TM_HALO0 = 0,    /* state set 0, every plane; box staged columns x halo rows x 1 */
    TM_HALO1,        /* state set 1 */
    TM_CELL0,        /* state set 0, every plane; box tile columns x tile rows x 1 */
    TM_CELL1,        /* state set 1 */
    TM_ZP,           /* the three topography planes; box R_J x (tile rows + 4) x 1 */
    TM_ZC,           /* the three topography planes; box R_J x (tile rows + 2) x 1 */
    TM_KS,           /* the Ks plane; box tile columns x tile rows x 1 */
    TM_CELLD0,       /* state set 0, its FP64 planes (vinf, M_k); box tile columns x tile rows x 1 */
    TM_CELLD1,       /* state set 1 */
    TM_COUNT
};

struct alignas(64) TmaMaps {
    CUtensorMap m[TM_COUNT];
};

/* polls of a tile-load wait before it is reported as timed out (each poll
 * is a bounded hardware wait; together far longer than any tile load) */
#define SWEHR_TMA_MAX_POLLS (1u << 24)

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

/* make the initialised barrier visible to the copy engine */
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

/* arrive once and announce the bytes the phase's copies will deliver */
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

/* order this CTA's earlier shared-memory accesses before copies that write it */
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

/* box (x, y, z) of a 3-D tensor map into shared memory (x is the
 * contiguous coordinate and must be a multiple of 16 bytes) */
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
            "r"(smem_addr(dst)),
        "l"((uint64_t)map), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

/* Wait for the phase with the given parity; false when the bounded number of
 * polls ran out. */
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    for (uint32_t k = 0; k < SWEHR_TMA_MAX_POLLS; k++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace swehr
