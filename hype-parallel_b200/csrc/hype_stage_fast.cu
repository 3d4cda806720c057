// hype_stage_fast.cu -- the FP64 performance form of the primitive-variable
// stage kernel (HYPE_PREC_FP64_FAST): stage_tile with FastSystem / ReconFast
// (hype_physics_fast.cuh).  This translation unit is built with FMA contraction
// (no --fmad=false): products and sums fuse where the compiler finds them, so
// its results differ from the reference's in the last bits; the tests hold
// them to a relative L-infinity difference of 1e-12 per RHS evaluation.
#include <cuda.h>
#include <cuda_runtime.h>
#include "hype_stage_tile.cuh"

namespace hype {

template <int SYS, int N, int CELLS>
__global__ void __launch_bounds__(2 * CELLS, (StageKernel<SYS, N, CELLS>::MIN_BLOCKS))
stage_fast_kernel(const __grid_constant__ CUtensorMap tmap, const StageParams p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * CELLS / 32];
    stage_tile<SYS, N, CELLS, false, false, true>(p, &tmap, blockIdx.x, p.run0 + (int)blockIdx.y, smem_raw, red_s);
}

struct FastEntry {
    const void *fn;
    size_t smem;
    int threads;
};

template <int SYS, int N, int CELLS>
static FastEntry fast_of()
{
    return FastEntry{reinterpret_cast<const void *>(stage_fast_kernel<SYS, N, CELLS>), StageKernel<SYS, N, CELLS>::smem_bytes(),
                     2 * CELLS};
}

template <int SYS, int CELLS>
static FastEntry fast_sys(int order)
{
    switch (order) {
    case 0: return fast_of<SYS, 0, CELLS>();
    case 1: return fast_of<SYS, 1, CELLS>();
    case 2: return fast_of<SYS, 2, CELLS>();
    default: return fast_of<SYS, 3, CELLS>();
    }
}

template <int CELLS>
static FastEntry fast_cells(int sys, int order)
{
    switch (sys) {
    case SYS_EULER: return fast_sys<SYS_EULER, CELLS>(order);
    case SYS_KAPILA: return fast_sys<SYS_KAPILA, CELLS>(order);
    default: return fast_sys<SYS_BN, CELLS>(order);
    }
}

static FastEntry fast_entry(int sys, int order, int cells)
{
    return cells == 64 ? fast_cells<64>(sys, order) : fast_cells<128>(sys, order);
}

cudaError_t stage_fast_configure(int sys, int order, int cells)
{
    const FastEntry e = fast_entry(sys, order, cells);
    return cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
}

int stage_fast_blocks_per_sm(int sys, int order, int cells)
{
    const FastEntry e = fast_entry(sys, order, cells);
    int nb = 0;
    if (stage_fast_configure(sys, order, cells) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.fn, e.threads, e.smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_stage_fast(int sys, int order, int cells, const CUtensorMap &tmap, const StageParams &p, cudaStream_t s)
{
    const FastEntry e = fast_entry(sys, order, cells);
    CUtensorMap tm = tmap;
    StageParams pp = p;
    void *args[] = {&tm, &pp};
    const unsigned gy = (unsigned)(p.run_count > 0 ? p.run_count : p.runs);
    return cudaLaunchKernel(e.fn, dim3((unsigned)p.strips, gy, 1), dim3((unsigned)e.threads, 1, 1), args, e.smem, s);
}

// fast_rcp and IEEE division of the same arguments, for the accuracy test
__global__ void rcp_check_kernel(const double *x, double *fast, double *ieee, int n)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        fast[k] = fast_rcp(x[k]);
        ieee[k] = 1.0 / x[k];
    }
}

}  // namespace hype

// Test entry point (no counterpart in the reference): fast_rcp(x[k]) and the
// IEEE quotient 1.0 / x[k] on `device`, for host arrays of n values.
extern "C" HYPE_API int hype_test_fast_rcp(int device, const double *x, int n, double *fast, double *ieee)
{
    if (!x || !fast || !ieee || n <= 0) return HYPE_ERR_INVALID;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return HYPE_ERR_NO_DEVICE;
    struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};
    double *d = nullptr;
    const size_t bytes = sizeof(double) * (size_t)n;
    if (cudaMalloc(&d, 3 * bytes) != cudaSuccess) return HYPE_ERR_NOMEM;
    int rc = HYPE_OK;
    if (cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice) != cudaSuccess) rc = HYPE_ERR_CUDA;
    if (rc == HYPE_OK) {
        hype::rcp_check_kernel<<<(n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024, 256>>>(d, d + n, d + 2 * (size_t)n, n);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = HYPE_ERR_CUDA;
    }
    if (rc == HYPE_OK && (cudaMemcpy(fast, d + n, bytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
                          cudaMemcpy(ieee, d + 2 * (size_t)n, bytes, cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = HYPE_ERR_CUDA;
    cudaFree(d);
    return rc;
}
