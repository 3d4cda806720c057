// hype_aux.cu -- small kernels around the stage kernel: layout changes at the
// C-ABI boundary (the reference's interleaved Vec <-> field planes) and the
// per-step time-step control that HyPE-2D's MonitorFunction and PETSc TS do on
// the host (post_process.c:19, hype.c:356-359).  Built with --fmad=false.
#include <cuda_runtime.h>
#include "hype_internal.h"

namespace hype {

// Interleaved cell-major array (Field{comp[nVar]}, hype.h:68-70) -> planes.
// One thread per (cell, field); reads and writes are both contiguous in the
// thread index through a shared-memory tile.
template <int TILE>
__global__ void aos_to_planes_kernel(const double *__restrict__ aos, double *__restrict__ planes,
                                     int nx, int ny, int nv, int pitch, long long plane)
{
    __shared__ double tile[TILE * 9];
    const long long cell0 = (long long)blockIdx.x * TILE;
    const long long ncell = (long long)nx * ny;
    const int ncur = (int)min((long long)TILE, ncell - cell0);
    for (int k = threadIdx.x; k < ncur * nv; k += blockDim.x) tile[k] = aos[cell0 * nv + k];
    __syncthreads();
    for (int k = threadIdx.x; k < ncur * nv; k += blockDim.x) {
        const int c = k / ncur, m = k % ncur;
        const long long cell = cell0 + m;
        const int j = (int)(cell / nx), i = (int)(cell % nx);
        planes[(long long)c * plane + (long long)j * pitch + i] = tile[m * nv + c];
    }
}

template <int TILE>
__global__ void planes_to_aos_kernel(const double *__restrict__ planes, double *__restrict__ aos,
                                     int nx, int ny, int nv, int pitch, long long plane)
{
    __shared__ double tile[TILE * 9];
    const long long cell0 = (long long)blockIdx.x * TILE;
    const long long ncell = (long long)nx * ny;
    const int ncur = (int)min((long long)TILE, ncell - cell0);
    for (int k = threadIdx.x; k < ncur * nv; k += blockDim.x) {
        const int c = k / ncur, m = k % ncur;
        const long long cell = cell0 + m;
        const int j = (int)(cell / nx), i = (int)(cell % nx);
        tile[m * nv + c] = planes[(long long)c * plane + (long long)j * pitch + i];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < ncur * nv; k += blockDim.x) aos[cell0 * nv + k] = tile[k];
}

cudaError_t launch_aos_to_planes(const double *aos, double *planes, int nx, int ny, int nv, int pitch, long long plane, cudaStream_t s)
{
    constexpr int TILE = 256;
    const long long ncell = (long long)nx * ny;
    const unsigned blocks = (unsigned)((ncell + TILE - 1) / TILE);
    aos_to_planes_kernel<TILE><<<blocks, 256, 0, s>>>(aos, planes, nx, ny, nv, pitch, plane);
    return cudaGetLastError();
}

cudaError_t launch_planes_to_aos(const double *planes, double *aos, int nx, int ny, int nv, int pitch, long long plane, cudaStream_t s)
{
    constexpr int TILE = 256;
    const long long ncell = (long long)nx * ny;
    const unsigned blocks = (unsigned)((ncell + TILE - 1) / TILE);
    planes_to_aos_kernel<TILE><<<blocks, 256, 0, s>>>(planes, aos, nx, ny, nv, pitch, plane);
    return cudaGetLastError();
}

// dt of the first step from the seeding RHS call (hype.c:343, 356):
// dt = CFL h / (2 s_max)  (rhs_function_prim.c:620)
__global__ void seed_dt_kernel(DevScalars *sc, double cfl_h)
{
    const double smax = __longlong_as_double((long long)sc->smax);
    sc->time_step = cfl_h / (2.0 * smax);
    sc->smax = 0ull;
}

// Start of a step: the monitor hands TS the last RHS's dt; TS stops at
// max_steps or t_final and clips the last step to land on t_final (MATCHSTEP).
__global__ void begin_step_kernel(DevScalars *sc)
{
    if (sc->done) return;
    if (sc->steps >= sc->max_steps || sc->t >= sc->t_final) { sc->done = 1; return; }
    double dt = sc->time_step;
    if (sc->t + dt > sc->t_final) dt = sc->t_final - sc->t;
    sc->dt = dt;
    sc->smax = 0ull;
}

// End of a step: the last stage's RHS set Ctx->dt for the next step.
__global__ void end_step_kernel(DevScalars *sc, double cfl_h)
{
    if (sc->done) return;
    const double smax = __longlong_as_double((long long)sc->smax);
    sc->time_step = cfl_h / (2.0 * smax);
    sc->t = sc->t + sc->dt;
    sc->steps = sc->steps + 1;
}

cudaError_t launch_seed_dt(DevScalars *sc, double cfl_h, cudaStream_t s)
{
    seed_dt_kernel<<<1, 1, 0, s>>>(sc, cfl_h);
    return cudaGetLastError();
}
cudaError_t launch_begin_step(DevScalars *sc, cudaStream_t s)
{
    begin_step_kernel<<<1, 1, 0, s>>>(sc);
    return cudaGetLastError();
}
cudaError_t launch_end_step(DevScalars *sc, double cfl_h, cudaStream_t s)
{
    end_step_kernel<<<1, 1, 0, s>>>(sc, cfl_h);
    return cudaGetLastError();
}

// Conservation totals: per-block partial sums over whole rows (FP64, fixed
// order), then one block adds the partials in block order.  Slot nv holds the
// minimum and nv+1 the maximum of field `acomp` (the volume fraction), or 0.
constexpr int TOT_BLOCKS = 512;
constexpr int TOT_THREADS = 256;

__global__ void totals_partial_kernel(const double *__restrict__ planes, double *__restrict__ part, int nx, int ny,
                                      int nv, int pitch, long long plane, int acomp)
{
    __shared__ double red[TOT_THREADS];
    const int j0 = (int)(((long long)blockIdx.x * ny) / gridDim.x);
    const int j1 = (int)(((long long)(blockIdx.x + 1) * ny) / gridDim.x);
    for (int c = 0; c < nv + 2; ++c) {
        double acc = (c == nv) ? 1e300 : (c == nv + 1 ? -1e300 : 0.0);
        const int cc = c < nv ? c : acomp;
        if (cc >= 0) {
            for (int j = j0; j < j1; ++j)
                for (int i = threadIdx.x; i < nx; i += blockDim.x) {
                    const double v = planes[(long long)cc * plane + (long long)j * pitch + i];
                    if (c < nv) acc += v;
                    else if (c == nv) acc = fmin(acc, v);
                    else acc = fmax(acc, v);
                }
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) {
                const double a = red[threadIdx.x], b = red[threadIdx.x + o];
                red[threadIdx.x] = c < nv ? a + b : (c == nv ? fmin(a, b) : fmax(a, b));
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * (nv + 2) + c] = cc >= 0 ? red[0] : 0.0;
        __syncthreads();
    }
}

__global__ void totals_final_kernel(double *part, int nblocks, int nv)
{
    const int c = threadIdx.x;
    if (c >= nv + 2) return;
    double acc = part[c];
    for (int b = 1; b < nblocks; ++b) {
        const double v = part[(size_t)b * (nv + 2) + c];
        acc = c < nv ? acc + v : (c == nv ? fmin(acc, v) : fmax(acc, v));
    }
    part[(size_t)nblocks * (nv + 2) + c] = acc;
}

__global__ void copy_out_kernel(const double *src, double *dst, int n)
{
    const int k = threadIdx.x;
    if (k < n) dst[k] = src[k];
}

cudaError_t launch_totals(const double *planes, double *red, int nx, int ny, int nv, int pitch, long long plane, int acomp,
                          cudaStream_t s)
{
    const int nb = ny < TOT_BLOCKS ? ny : TOT_BLOCKS;
    double *part = red + 64;   // red[0..nv+1] receives the result
    totals_partial_kernel<<<nb, TOT_THREADS, 0, s>>>(planes, part, nx, ny, nv, pitch, plane, acomp);
    totals_final_kernel<<<1, 32, 0, s>>>(part, nb, nv);
    copy_out_kernel<<<1, 32, 0, s>>>(part + (size_t)nb * (nv + 2), red, nv + 2);
    return cudaGetLastError();
}

}  // namespace hype
