// hype_stage_visc.cu -- the stage kernels of the reference's VISCOUS build
// (hype.h:36 leaves it off; kapila_5eqn.c has the viscous fluxes, the other
// systems' builds do not link or write past nVar): Kapila, N = 1..3, the
// primitive (RHSFunctionPrim) and conservative (RHSFunction) paths, grid
// form, 128-column tiles.  The tile is stage_tile with VISC = true, which
// keeps the top-face gradients of the variables the viscous flux reads in an
// extra shared-memory array behind the carries.
//
// Built with --fmad=false: arithmetic rounds exactly as the reference's C does.
#include <cuda.h>
#include <cuda_runtime.h>
#include "hype_stage_tile.cuh"

namespace hype {

template <bool CONS, int N>
struct ViscKernel {
    using K = StageKernel<SYS_KAPILA, N, STAGE_CELLS>;
    static constexpr int NG = CONS ? 4 : 2;
    static constexpr size_t smem_bytes() { return K::smem_bytes() + (size_t)Quad<N>::NFGP * NG * 2 * STAGE_CELLS * 8; }
};

template <bool CONS, int N>
__global__ void __launch_bounds__(2 * STAGE_CELLS, 1)
stage_visc_kernel(const __grid_constant__ CUtensorMap tmap, const StageParams p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * STAGE_CELLS / 32];
    stage_tile<SYS_KAPILA, N, STAGE_CELLS, CONS, true>(p, &tmap, blockIdx.x, p.run0 + (int)blockIdx.y, smem_raw, red_s);
}

struct ViscEntry {
    const void *fn;
    size_t smem;
};

template <bool CONS, int N>
static ViscEntry visc_of()
{
    return ViscEntry{reinterpret_cast<const void *>(stage_visc_kernel<CONS, N>), ViscKernel<CONS, N>::smem_bytes()};
}

template <bool CONS>
static ViscEntry visc_order(int order)
{
    switch (order) {
    case 1: return visc_of<CONS, 1>();
    case 2: return visc_of<CONS, 2>();
    default: return visc_of<CONS, 3>();
    }
}

static ViscEntry visc_entry(int order, bool cons) { return cons ? visc_order<true>(order) : visc_order<false>(order); }

cudaError_t stage_visc_configure(int order, bool cons)
{
    const ViscEntry e = visc_entry(order, cons);
    return cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
}

int stage_visc_blocks_per_sm(int order, bool cons)
{
    const ViscEntry e = visc_entry(order, cons);
    int nb = 0;
    if (stage_visc_configure(order, cons) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.fn, 2 * STAGE_CELLS, e.smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_stage_visc(int order, bool cons, const CUtensorMap &tmap, const StageParams &p, cudaStream_t s)
{
    const ViscEntry e = visc_entry(order, cons);
    CUtensorMap tm = tmap;
    StageParams pp = p;
    void *args[] = {&tm, &pp};
    const unsigned gy = (unsigned)(p.run_count > 0 ? p.run_count : p.runs);
    return cudaLaunchKernel(e.fn, dim3((unsigned)p.strips, gy, 1), dim3(2 * STAGE_CELLS, 1, 1), args, e.smem, s);
}

}  // namespace hype
