// hype_stage_paths_batch.cu -- the persistent (batched) form of the stage kernels
// of the conservative-variable path (RHSFunction, rhs_function.c:12-625) and of
// the reference's VISCOUS build (Kapila, N = 1..3, primitive and conservative):
// the same work-list loop as stage_batch_kernel around stage_tile with CONS /
// VISC set, 128-column tiles.
//
// Built with --fmad=false: arithmetic rounds exactly as the reference's C does.
#include <cuda.h>
#include <cuda_runtime.h>
#include "hype_stage_tile.cuh"

namespace hype {

template <int SYS, int N, bool CONS, bool VISC>
struct PathKernel {
    using K = StageKernel<SYS, N, STAGE_CELLS>;
    static constexpr int NG = CONS ? 4 : 2;
    // the viscous tile keeps top-face gradients behind the carries
    static constexpr size_t smem_bytes()
    {
        return K::smem_bytes() + (VISC ? (size_t)Quad<N>::NFGP * NG * 2 * STAGE_CELLS * 8 : 0);
    }
    static constexpr int MIN_BLOCKS = VISC ? 1 : K::MIN_BLOCKS;
};

template <int SYS, int N, bool CONS, bool VISC>
__global__ void __launch_bounds__(2 * STAGE_CELLS, (PathKernel<SYS, N, CONS, VISC>::MIN_BLOCKS))
path_batch_kernel(const StageParams *__restrict__ inst, const CUtensorMap *__restrict__ tmaps, const int2 *__restrict__ work,
                  int *__restrict__ sched)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * STAGE_CELLS / 32];
    __shared__ int item_s;
    __shared__ StageParams p_s;   // the item's parameters, re-read after every barrier of the tile
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
        stage_tile<SYS, N, STAGE_CELLS, CONS, VISC>(p_s, &tmaps[it.x], tile % p_s.strips, tile / p_s.strips, smem_raw, red_s);
        last = p_s.sc;
    }
    work_finish(sched);
}

struct PathEntry {
    const void *fn;
    size_t smem;
};

template <int SYS, int N, bool CONS, bool VISC>
static PathEntry path_of()
{
    return PathEntry{reinterpret_cast<const void *>(path_batch_kernel<SYS, N, CONS, VISC>), PathKernel<SYS, N, CONS, VISC>::smem_bytes()};
}

template <int SYS>
static PathEntry cons_order(int order)
{
    switch (order) {
    case 0: return path_of<SYS, 0, true, false>();
    case 1: return path_of<SYS, 1, true, false>();
    case 2: return path_of<SYS, 2, true, false>();
    default: return path_of<SYS, 3, true, false>();
    }
}

template <bool CONS>
static PathEntry visc_order(int order)
{
    switch (order) {
    case 1: return path_of<SYS_KAPILA, 1, CONS, true>();
    case 2: return path_of<SYS_KAPILA, 2, CONS, true>();
    default: return path_of<SYS_KAPILA, 3, CONS, true>();
    }
}

static PathEntry path_entry(int path, int sys, int order)
{
    if (path == BATCH_PATH_VISC) return visc_order<false>(order);
    if (path == BATCH_PATH_VISC_CONS) return visc_order<true>(order);
    switch (sys) {
    case SYS_EULER: return cons_order<SYS_EULER>(order);
    case SYS_KAPILA: return cons_order<SYS_KAPILA>(order);
    default: return cons_order<SYS_BN>(order);
    }
}

cudaError_t path_batch_configure(int path, int sys, int order)
{
    const PathEntry e = path_entry(path, sys, order);
    return cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
}

int path_batch_blocks_per_sm(int path, int sys, int order)
{
    const PathEntry e = path_entry(path, sys, order);
    int nb = 0;
    if (path_batch_configure(path, sys, order) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.fn, 2 * STAGE_CELLS, e.smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_path_batch(int path, int sys, int order, const StageParams *inst, const CUtensorMap *tmaps, const int2 *work,
                              int *sched, int blocks, cudaStream_t s)
{
    const PathEntry e = path_entry(path, sys, order);
    void *args[] = {&inst, &tmaps, &work, &sched};
    return cudaLaunchKernel(e.fn, dim3((unsigned)blocks, 1, 1), dim3(2 * STAGE_CELLS, 1, 1), args, e.smem, s);
}

}  // namespace hype
