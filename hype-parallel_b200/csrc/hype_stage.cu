// hype_stage.cu -- the primitive-variable stage kernels (RHSFunctionPrim,
// rhs_function_prim.c:12-626) in their grid form (one block per tile) and
// persistent form (blocks walk a work-list of tiles of many grids), and the
// host dispatch over (system, order, tile width).  The tile itself is
// stage_tile in hype_stage_tile.cuh.
//
// Built with --fmad=false: arithmetic rounds exactly as the reference's C does.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdio>
#include "hype_stage_tile.cuh"

namespace hype {

template <int SYS, int N, int CELLS>
__global__ void __launch_bounds__(2 * CELLS, (StageKernel<SYS, N, CELLS>::MIN_BLOCKS))
stage_kernel(const __grid_constant__ CUtensorMap tmap, const StageParams p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * CELLS / 32];
    stage_tile<SYS, N, CELLS, false>(p, &tmap, blockIdx.x, p.run0 + (int)blockIdx.y, smem_raw, red_s);
}

// Persistent form: the block walks a list of (grid, tile) work items; every grid
// has its own parameters, tensor map and device scalars.
template <int SYS, int N, int CELLS>
__global__ void __launch_bounds__(2 * CELLS, (StageKernel<SYS, N, CELLS>::MIN_BLOCKS))
stage_batch_kernel(const StageParams *__restrict__ inst, const CUtensorMap *__restrict__ tmaps,
                   const int2 *__restrict__ work, int *__restrict__ sched)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * CELLS / 32];
    __shared__ int item_s;
    // the item's parameters live in shared memory: re-read after every barrier
    // of the tile instead of pinning registers for the whole tile
    __shared__ StageParams p_s;
    const int nwork = sched[0];
    const DevScalars *last = nullptr;
    for (;;) {
        const int w = work_take(sched, nwork, last, &item_s);
        if (w >= nwork) break;
        const int2 it = work[w];
        if (threadIdx.x == 0) {
            p_s = inst[it.x];
            p_s.runs *= item_refine(it.y);
            fence_tensormap_acquire(&tmaps[it.x]);
        }
        __syncthreads();
        const int tile = item_tile(it.y);
        stage_tile<SYS, N, CELLS, false>(p_s, &tmaps[it.x], tile % p_s.strips, tile / p_s.strips, smem_raw, red_s);
        last = p_s.sc;
    }
    work_finish(sched);
}

// ---------------------------------------------------------------------------
// host dispatch over (system, order, tile width)
// ---------------------------------------------------------------------------
struct StageEntry {
    const void *single;
    const void *batch;
    size_t smem;
    int threads;
};

template <int SYS, int N, int CELLS>
static StageEntry entry_of()
{
    return StageEntry{reinterpret_cast<const void *>(stage_kernel<SYS, N, CELLS>),
                      reinterpret_cast<const void *>(stage_batch_kernel<SYS, N, CELLS>),
                      StageKernel<SYS, N, CELLS>::smem_bytes(), 2 * CELLS};
}

template <int SYS, int CELLS>
static StageEntry entry_sys(int order)
{
    switch (order) {
    case 0: return entry_of<SYS, 0, CELLS>();
    case 1: return entry_of<SYS, 1, CELLS>();
    case 2: return entry_of<SYS, 2, CELLS>();
    default: return entry_of<SYS, 3, CELLS>();
    }
}

template <int CELLS>
static StageEntry entry_cells(int sys, int order)
{
    switch (sys) {
    case SYS_EULER: return entry_sys<SYS_EULER, CELLS>(order);
    case SYS_KAPILA: return entry_sys<SYS_KAPILA, CELLS>(order);
    default: return entry_sys<SYS_BN, CELLS>(order);
    }
}

static StageEntry stage_entry(int sys, int order, int cells)
{
    return cells == 64 ? entry_cells<64>(sys, order) : entry_cells<128>(sys, order);
}

size_t stage_smem_bytes(int sys, int order, int cells) { return stage_entry(sys, order, cells).smem; }
int stage_threads(int cells) { return 2 * cells; }

cudaError_t stage_configure(int sys, int order, int cells)
{
    const StageEntry e = stage_entry(sys, order, cells);
    cudaError_t r = cudaFuncSetAttribute(e.single, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
    if (r != cudaSuccess) return r;
    return cudaFuncSetAttribute(e.batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
}

int stage_blocks_per_sm(int sys, int order, int cells)
{
    const StageEntry e = stage_entry(sys, order, cells);
    int nb = 0;
    if (stage_configure(sys, order, cells) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.single, e.threads, e.smem) != cudaSuccess) return 0;
    return nb;
}

int stage_batch_blocks_per_sm(int sys, int order, int cells)
{
    const StageEntry e = stage_entry(sys, order, cells);
    int nb = 0;
    if (stage_configure(sys, order, cells) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.batch, e.threads, e.smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_stage(int sys, int order, int cells, const CUtensorMap &tmap, const StageParams &p, cudaStream_t s)
{
    const StageEntry e = stage_entry(sys, order, cells);
    CUtensorMap tm = tmap;
    StageParams pp = p;
    void *args[] = {&tm, &pp};
    const unsigned gy = (unsigned)(p.run_count > 0 ? p.run_count : p.runs);
    return cudaLaunchKernel(e.single, dim3((unsigned)p.strips, gy, 1), dim3((unsigned)e.threads, 1, 1), args, e.smem, s);
}

cudaError_t launch_stage_batch(int sys, int order, int cells, const StageParams *inst, const CUtensorMap *tmaps,
                               const int2 *work, int *sched, int blocks, cudaStream_t s)
{
    const StageEntry e = stage_entry(sys, order, cells);
    void *args[] = {&inst, &tmaps, &work, &sched};
    return cudaLaunchKernel(e.batch, dim3((unsigned)blocks, 1, 1), dim3((unsigned)e.threads, 1, 1), args, e.smem, s);
}

}  // namespace hype
