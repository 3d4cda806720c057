// hype_stage_cons.cu -- the conservative-variable stage kernels: HyPE-2D's
// RHSFunction (rhs_function.c:12-625), the path hype.c selects when
// Ctx.ReconsPrimitive is false (hype.c:341-352).  Same tile as the primitive
// path (hype_stage_tile.cuh with CONS = true), grid form only, 128-column
// tiles.
//
// Built with --fmad=false: arithmetic rounds exactly as the reference's C does.
#include <cuda.h>
#include <cuda_runtime.h>
#include "hype_stage_tile.cuh"

namespace hype {

template <int SYS, int N>
__global__ void __launch_bounds__(2 * STAGE_CELLS, (StageKernel<SYS, N, STAGE_CELLS>::MIN_BLOCKS))
stage_cons_kernel(const __grid_constant__ CUtensorMap tmap, const StageParams p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * STAGE_CELLS / 32];
    stage_tile<SYS, N, STAGE_CELLS, true>(p, &tmap, blockIdx.x, p.run0 + (int)blockIdx.y, smem_raw, red_s);
}

struct ConsEntry {
    const void *fn;
    size_t smem;
};

template <int SYS, int N>
static ConsEntry cons_of()
{
    return ConsEntry{reinterpret_cast<const void *>(stage_cons_kernel<SYS, N>), StageKernel<SYS, N, STAGE_CELLS>::smem_bytes()};
}

template <int SYS>
static ConsEntry cons_sys(int order)
{
    switch (order) {
    case 0: return cons_of<SYS, 0>();
    case 1: return cons_of<SYS, 1>();
    case 2: return cons_of<SYS, 2>();
    default: return cons_of<SYS, 3>();
    }
}

static ConsEntry cons_entry(int sys, int order)
{
    switch (sys) {
    case SYS_EULER: return cons_sys<SYS_EULER>(order);
    case SYS_KAPILA: return cons_sys<SYS_KAPILA>(order);
    default: return cons_sys<SYS_BN>(order);
    }
}

cudaError_t stage_cons_configure(int sys, int order)
{
    const ConsEntry e = cons_entry(sys, order);
    return cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
}

int stage_cons_blocks_per_sm(int sys, int order)
{
    const ConsEntry e = cons_entry(sys, order);
    int nb = 0;
    if (stage_cons_configure(sys, order) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.fn, 2 * STAGE_CELLS, e.smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_stage_cons(int sys, int order, const CUtensorMap &tmap, const StageParams &p, cudaStream_t s)
{
    const ConsEntry e = cons_entry(sys, order);
    CUtensorMap tm = tmap;
    StageParams pp = p;
    void *args[] = {&tm, &pp};
    const unsigned gy = (unsigned)(p.run_count > 0 ? p.run_count : p.runs);
    return cudaLaunchKernel(e.fn, dim3((unsigned)p.strips, gy, 1), dim3(2 * STAGE_CELLS, 1, 1), args, e.smem, s);
}

}  // namespace hype
