// hype_tma.cuh -- device helpers shared by the stage kernels: TMA tensor
// loads and mbarriers (inline PTX), ghost-index mapping of the boundary
// conditions, and the device error word.
#pragma once
#include <cuda.h>
#include <cstdint>
#include "hype_internal.h"

namespace hype {

// ---------------------------------------------------------------------------
// TMA / mbarrier helpers (inline PTX, sm_90+ forms, valid on sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                 ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded waits on TMA row loads.  Every mbarrier wait of the stage tiles (FP64
// and mixed) gives up once TMA_WAIT_NS nanoseconds of the GPU's global timer have
// passed without the load completing: the block then raises ERR_TMA_TIMEOUT (the
// host call returns HYPE_ERR_TIMEOUT) instead of waiting for ever.  Before it
// returns, the block waits, against one more deadline of the same length, for the
// loads it has already issued (mbar_drain), so no copy is left writing into the
// shared memory of a block that has exited; only if that drain also runs out does
// it leave them.
constexpr unsigned long long TMA_WAIT_NS = 2000000000ull;   // 2 s
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_wait_until(uint64_t *bar, unsigned parity, unsigned long long deadline)
{
    for (unsigned it = 0;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 31u) == 31u && global_ns() > deadline) return false;
    }
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    return mbar_wait_until(bar, parity, global_ns() + TMA_WAIT_NS);
}

// Ghost source index along one axis (rhs_function_prim.c:75-315 and the DMDA
// periodic wrap): transmissive copies the edge cell, reflective mirrors; the
// edge of a slab or block of a decomposed grid (BC_HALO) reads its halo rows or
// columns as they are.
__device__ __forceinline__ int map_axis(int g, int n, int bc_lo, int bc_hi)
{
    if (g < 0) {
        if (bc_lo == BC_HALO) return g;
        if (bc_lo == BC_PERIODIC || bc_hi == BC_PERIODIC) return g + n;
        if (bc_lo == BC_REFLECTIVE) return -1 - g;
        return 0;   // transmissive (inlet columns are replaced after conversion)
    }
    if (g >= n) {
        if (bc_hi == BC_HALO) return g;
        if (bc_lo == BC_PERIODIC || bc_hi == BC_PERIODIC) return g - n;
        if (bc_hi == BC_REFLECTIVE) return 2 * (n - 1) - g + 1;
        return n - 1;
    }
    return g;
}

__device__ __forceinline__ void raise_error(DevScalars *sc, unsigned bits, unsigned cell)
{
    atomicOr(&sc->err, bits);
    atomicMin(&sc->err_cell, cell);
}

// A tensor map in global memory written by the host (or an earlier kernel)
// between launches: order those writes before the TMA unit reads it.
__device__ __forceinline__ void fence_tensormap_acquire(const void *map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

// Work distribution of the persistent (batched) kernels over a list of
// (instance, tile) items: sched[0] = item count, sched[1] = next item,
// sched[2] = blocks finished.  Blocks take items in list order (the host sorts
// it longest first); the last block to finish zeroes sched[1] and sched[2], so
// back-to-back launches (graph replays) need no reset in between.  A block
// stops taking items once the instance of its last tile saw a TMA timeout.
__device__ __forceinline__ int work_take(int *sched, int nwork, const DevScalars *last_sc, int *item_s)
{
    if (threadIdx.x == 0) {
        const bool stop = last_sc && (*(volatile const unsigned *)&last_sc->err & ERR_TMA_TIMEOUT);
        *item_s = stop ? nwork : atomicAdd(&sched[1], 1);
    }
    __syncthreads();
    const int w = *item_s;
    __syncthreads();
    return w;
}
// A work item's tile: it.y = (log2 f << 28) | (run' * strips + strip), where run' is a
// run of the instance's row decomposition refined f times (run r split into runs
// r f .. r f + f-1).  The refined boundaries floor(run' ny / (f runs)) equal the
// instance's own floor(r ny / runs) at run' = r f, so plain and refined tiles of one
// instance cover its rows exactly once.
__device__ __forceinline__ int item_refine(int y) { return 1 << ((unsigned)y >> 28); }
__device__ __forceinline__ int item_tile(int y) { return y & 0x0fffffff; }

__device__ __forceinline__ void work_finish(int *sched)
{
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&sched[2], 1) == (int)gridDim.x - 1) {
            atomicExch(&sched[1], 0);
            atomicExch(&sched[2], 0);
        }
    }
}

}  // namespace hype
