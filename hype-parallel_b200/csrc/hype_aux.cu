// hype_aux.cu -- small kernels around the stage kernel: layout changes at the
// C-ABI boundary (the reference's interleaved Vec <-> field planes) and the
// per-step time-step control that HyPE-2D's MonitorFunction and PETSc TS do on
// the host (post_process.c:19, hype.c:356-359).  Built with --fmad=false.
#include <cuda_runtime.h>
#include <algorithm>
#include "hype_internal.h"
#include "hype_div.cuh"

namespace hype {

// Interleaved cell-major array (Field{comp[nVar]}, hype.h:68-70) -> planes,
// over the cells [cell_begin, cell_end).  One thread per (cell, field); reads
// and writes are both contiguous in the thread index through a shared-memory tile.
template <int TILE>
__global__ void aos_to_planes_kernel(const double *__restrict__ aos, double *__restrict__ planes, int nx, long long cell_begin,
                                     long long cell_end, int nv, int pitch, long long plane)
{
    __shared__ double tile[TILE * 9];
    const long long cell0 = cell_begin + (long long)blockIdx.x * TILE;
    const int ncur = (int)min((long long)TILE, cell_end - cell0);
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
__global__ void planes_to_aos_kernel(const double *__restrict__ planes, double *__restrict__ aos, int nx, long long cell_begin,
                                     long long cell_end, int nv, int pitch, long long plane)
{
    __shared__ double tile[TILE * 9];
    const long long cell0 = cell_begin + (long long)blockIdx.x * TILE;
    const int ncur = (int)min((long long)TILE, cell_end - cell0);
    for (int k = threadIdx.x; k < ncur * nv; k += blockDim.x) {
        const int c = k / ncur, m = k % ncur;
        const long long cell = cell0 + m;
        const int j = (int)(cell / nx), i = (int)(cell % nx);
        tile[m * nv + c] = planes[(long long)c * plane + (long long)j * pitch + i];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < ncur * nv; k += blockDim.x) aos[cell0 * nv + k] = tile[k];
}

constexpr int XPOSE_TILE = 256;

cudaError_t launch_aos_to_planes_rows(const double *aos, double *planes, int nx, int row0, int nrows, int nv, int pitch, long long plane,
                                      cudaStream_t s)
{
    const long long c0 = (long long)row0 * nx, c1 = c0 + (long long)nrows * nx;
    if (c1 <= c0) return cudaSuccess;
    const unsigned blocks = (unsigned)((c1 - c0 + XPOSE_TILE - 1) / XPOSE_TILE);
    aos_to_planes_kernel<XPOSE_TILE><<<blocks, 256, 0, s>>>(aos, planes, nx, c0, c1, nv, pitch, plane);
    return cudaGetLastError();
}

cudaError_t launch_planes_to_aos_rows(const double *planes, double *aos, int nx, int row0, int nrows, int nv, int pitch, long long plane,
                                      cudaStream_t s)
{
    const long long c0 = (long long)row0 * nx, c1 = c0 + (long long)nrows * nx;
    if (c1 <= c0) return cudaSuccess;
    const unsigned blocks = (unsigned)((c1 - c0 + XPOSE_TILE - 1) / XPOSE_TILE);
    planes_to_aos_kernel<XPOSE_TILE><<<blocks, 256, 0, s>>>(planes, aos, nx, c0, c1, nv, pitch, plane);
    return cudaGetLastError();
}

cudaError_t launch_aos_to_planes(const double *aos, double *planes, int nx, int ny, int nv, int pitch, long long plane, cudaStream_t s)
{
    return launch_aos_to_planes_rows(aos, planes, nx, 0, ny, nv, pitch, plane, s);
}

cudaError_t launch_planes_to_aos(const double *planes, double *aos, int nx, int ny, int nv, int pitch, long long plane, cudaStream_t s)
{
    return launch_planes_to_aos_rows(planes, aos, nx, 0, ny, nv, pitch, plane, s);
}

// dt from the last RHS's maxima: CFL h / (2 s_max) (rhs_function_prim.c:620),
// or, for a viscous solver, CFL h / (2 (s_max + (s_max_v / h) 2))
// (rhs_function_prim.c:617).  Both in one expression: r1h_v = 0 makes the
// viscous term an exact +0, and s_max + 0 = s_max.
__device__ __forceinline__ double next_dt(const DevScalars *sc, double cfl_h)
{
    const double smax = __longlong_as_double((long long)sc->smax);
    const double smaxv = __longlong_as_double((long long)sc->smax_v);
    return cfl_h / (2.0 * (smax + (sc->r1h_v * smaxv) * 2.0));
}

// dt of the first step from the seeding RHS call (hype.c:343, 356)
__global__ void seed_dt_kernel(DevScalars *sc, double cfl_h)
{
    sc->time_step = next_dt(sc, cfl_h);
    sc->smax = 0ull;
    sc->smax_v = 0ull;
}

// Start of a step: the monitor hands TS the last RHS's dt; TS stops at
// max_steps or t_final and clips the last step to land on t_final (MATCHSTEP).
// A run whose RHS raised an error stops there (the reference aborts the job).
// A finished or held run sits this step out: `idle` tells the stages and
// end_step to leave it untouched.
__device__ __forceinline__ void begin_step(DevScalars *sc)
{
    sc->idle = 1;
    if (sc->done) return;
    if (sc->err || sc->steps >= sc->max_steps || sc->t >= sc->t_final) { sc->done = 1; return; }
    if (sc->hold) return;
    sc->idle = 0;
    double dt = sc->time_step;
    if (sc->t + dt > sc->t_final) dt = sc->t_final - sc->t;
    sc->dt = dt;
    sc->smax = 0ull;
    sc->smax_v = 0ull;
}

// End of a step: the last stage's RHS set Ctx->dt for the next step.
__device__ __forceinline__ void end_step(DevScalars *sc, double cfl_h)
{
    if (sc->idle) return;
    sc->time_step = next_dt(sc, cfl_h);
    sc->t = sc->t + sc->dt;
    sc->steps = sc->steps + 1;
}

__global__ void begin_step_kernel(DevScalars *sc) { begin_step(sc); }
__global__ void end_step_kernel(DevScalars *sc, double cfl_h) { end_step(sc, cfl_h); }

__global__ void begin_step_batch_kernel(DevScalars *sc, const int *members, const int *hold)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < members[0]; k += gridDim.x * blockDim.x) {
        const int m = members[1 + k];
        sc[m].hold = hold[m];
        begin_step(&sc[m]);
    }
}
__global__ void end_step_batch_kernel(DevScalars *sc, const int *members)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < members[0]; k += gridDim.x * blockDim.x) {
        DevScalars *p = &sc[members[1 + k]];
        end_step(p, p->cfl_h);
    }
}
// one block per member; skipped for idle instances like the stages
__global__ void copy_batch_kernel(double *const *dst, const double *const *src, const long long *n, const int *members,
                                  const DevScalars *sc)
{
    for (int k = blockIdx.x; k < members[0]; k += gridDim.x) {
        const int m = members[1 + k];
        if (sc[m].idle) continue;
        const double2 *a = reinterpret_cast<const double2 *>(src[m]);
        double2 *b = reinterpret_cast<double2 *>(dst[m]);
        for (long long i = threadIdx.x; i < n[m] / 2; i += blockDim.x) b[i] = a[i];
        if ((n[m] & 1) && threadIdx.x == 0) dst[m][n[m] - 1] = src[m][n[m] - 1];
    }
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
static unsigned member_blocks(int max_members, int per_block) { return (unsigned)((max_members + per_block - 1) / per_block > 0 ? (max_members + per_block - 1) / per_block : 1); }
cudaError_t launch_begin_step_batch(DevScalars *sc, const int *members, const int *hold, int max_members, cudaStream_t s)
{
    begin_step_batch_kernel<<<member_blocks(max_members, 128), 128, 0, s>>>(sc, members, hold);
    return cudaGetLastError();
}
cudaError_t launch_end_step_batch(DevScalars *sc, const int *members, int max_members, cudaStream_t s)
{
    end_step_batch_kernel<<<member_blocks(max_members, 128), 128, 0, s>>>(sc, members);
    return cudaGetLastError();
}
cudaError_t launch_copy_batch(double *const *dst, const double *const *src, const long long *n, const int *members,
                              int max_members, const DevScalars *sc, cudaStream_t s)
{
    copy_batch_kernel<<<member_blocks(max_members, 1), 512, 0, s>>>(dst, src, n, members, sc);
    return cudaGetLastError();
}

// The SSP schemes of hype.c:362-382 as stage lists.  PETSc's TSSSP writes
// each stage as VecAXPY(w, dt/kb, F) or VecAXPBYPCZ; the coefficients below
// are computed with the expressions of its step functions so that they round
// identically.
int ssp_plan(int order, PlanStage *st, int *copy_back)
{
    auto S = [&](int k, int in, int out, int mode, double ka, double kb, double kc, int x, int out2, int reduce) {
        st[k] = PlanStage{in, out, mode, ka, kb, kc, x, out2, reduce};
    };
    *copy_back = 0;
    switch (order) {
    case 0:   // TSEULER: S0 = u + dt F(u); u = S0
        S(0, B_U, B_S0, OUT_AXPY, 0, 1.0, 0, B_NONE, B_NONE, 1);
        *copy_back = 1;
        return 1;
    case 1: { // SSPRKS2, s = 2: w = u + (dt/(s-1)) F(u); u = ((s-1)/s) w + (dt/s) F(w) + (1/s) u
        const int ns = 2;
        S(0, B_U, B_S0, OUT_AXPY, 0, (ns - 1.), 0, B_NONE, B_NONE, 0);
        S(1, B_S0, B_U, OUT_ZSX, (ns - 1.) / ns, (double)ns, 1. / ns, B_U, B_NONE, 1);
        return 2;
    }
    case 2: { // SSPRKS3, s = 4, n = 2, r = 2
        const int n = 2, ns = 4, r = ns - n;
        S(0, B_U, B_S0, OUT_AXPY, 0, (double)r, 0, B_NONE, B_NONE, 0);
        S(1, B_S0, B_S1, OUT_AXPY, 0, (double)r, 0, B_NONE, B_NONE, 0);
        // VecAXPBYPCZ(w0, n/(2n-1), (n-1) dt/(r(2n-1)), (n-1)/(2n-1), w1 = u^n, F)
        S(2, B_S1, B_S0, OUT_ZXS, 1. * n / (2 * n - 1.), (double)(r * (2 * n - 1)), (n - 1.) / (2 * n - 1.), B_U, B_NONE, 0);
        S(3, B_S0, B_U, OUT_AXPY, 0, (double)r, 0, B_NONE, B_NONE, 1);
        return 4;
    }
    case 3: { // SSPRK(10,4)
        int in = B_U, k = 0, ns = 0;
        const int bufs[2] = {B_S0, B_S1};
        for (int i = 0; i < 4; ++i) { S(ns++, in, bufs[k], OUT_AXPY, 0, 6.0, 0, B_NONE, B_NONE, 0); in = bufs[k]; k ^= 1; }
        // fifth stage + w1 = u/25 + 9 w/25 (into S2) + w = 15 w1 - 5 w
        S(ns++, in, bufs[k], OUT_RK104_5, 0, 6.0, 0, B_U, B_S2, 0); in = bufs[k]; k ^= 1;
        for (int i = 5; i < 9; ++i) { S(ns++, in, bufs[k], OUT_AXPY, 0, 6.0, 0, B_NONE, B_NONE, 0); in = bufs[k]; k ^= 1; }
        // VecAXPBYPCZ(w1, 3/5, dt/10, 1, w0, F); sol = w1
        S(ns++, in, B_U, OUT_ZSX, 3. / 5, 10.0, 1.0, B_S2, B_NONE, 1);
        return ns;
    }
    default:
        return 0;
    }
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

// ---------------------------------------------------------------------------
// FP64 rate: 8 independent chains x = x*m + c per thread, which --fmad=false
// keeps as one multiply and one add each (FUSED: one explicit fused multiply-add,
// two FLOPs).  The data-dependent store keeps the chains alive; it never fires
// for these constants.
// ---------------------------------------------------------------------------
namespace {
constexpr int RATE_CHAINS = 8;
template <bool FUSED>
__global__ void __launch_bounds__(256) fp64_rate_kernel(double *sink, int iters, double seed)
{
    double x[RATE_CHAINS];
#pragma unroll
    for (int k = 0; k < RATE_CHAINS; ++k) x[k] = seed + 1e-3 * k + 1e-9 * threadIdx.x;
    const double m = 0.999999999, c = 1e-9;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < RATE_CHAINS; ++k) x[k] = FUSED ? fma(x[k], m, c) : x[k] * m + c;
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < RATE_CHAINS; ++k) s += x[k];
    if (s == -1.0) sink[0] = s;
}

// best of `reps` timed launches (one warm-up launch first); 2 operations per chain link
int fp64_rate_of(bool fused, int device, int reps, double *ops_per_s)
{
    if (!ops_per_s || reps < 1) return HYPE_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return HYPE_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return HYPE_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *sink = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = HYPE_OK;
    if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return HYPE_ERR_NOMEM;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess)
        rc = HYPE_ERR_CUDA;
    const int blocks = sms * 8, threads = 256, iters = fused ? 8192 : 4096;
    double best = 0.0;
    for (int r = 0; r <= reps && rc == HYPE_OK; ++r) {   // launch 0 warms up
        cudaEventRecord(e0, st);
        if (fused) fp64_rate_kernel<true><<<blocks, threads, 0, st>>>(sink, iters, 1.0 + r);
        else fp64_rate_kernel<false><<<blocks, threads, 0, st>>>(sink, iters, 1.0 + r);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) { rc = HYPE_ERR_CUDA; break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = 2.0 * RATE_CHAINS * (double)iters * blocks * threads;
        if (r > 0 && ms > 0.f) best = std::max(best, ops / (ms * 1e-3));
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaFree(sink);
    *ops_per_s = best;
    return rc;
}
}  // namespace

namespace {
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// a double of random sign, significand and a binary exponent in [-1100, 1100] (subnormal
// and out-of-range exponents clamp to zero / infinity through ldexp)
__device__ __forceinline__ double wide_double(unsigned long long u, unsigned long long v)
{
    const double m = 1.0 + (double)(u >> 12) * (1.0 / 4503599627370496.0);
    const int ex = (int)(v % 2201ull) - 1100;
    const double x = ldexp(m, ex);
    return (v >> 63) ? -x : x;
}
// the cases of hype_test_division, by index: 0 raw bit patterns, 1 operands of every
// exponent, 2 quotients next to a midpoint of two doubles, 3 all-ones divisors
__global__ void division_check_kernel(long long n, unsigned long long seed, unsigned long long *counts)
{
    unsigned long long mism = 0, spec = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
        const unsigned long long u0 = mix64(k), u1 = mix64(k ^ 0x5851F42D4C957F2Dull), u2 = mix64(k + 0x14057B7EF767814Full),
                                 u3 = mix64(k * 3 + 1);
        double a, b;
        switch ((int)(i & 3)) {
        case 0: a = __longlong_as_double((long long)u0); b = __longlong_as_double((long long)u1); break;
        case 1: a = wide_double(u0, u1); b = wide_double(u2, u3); break;
        case 2: {   // a = RN(b * q_mid), q_mid = 1 + (2m + 1) 2^-53: a/b lies within an ulp or so of a midpoint
            b = wide_double(u2, u3 % 1601ull + ((u3 >> 63) << 63));   // exponents [-1100, 500]
            const double qmid = 1.0 + (double)(2 * (u0 >> 12) + 1) * (1.0 / 9007199254740992.0);
            a = b * qmid;
            break;
        }
        default: {   // divisor with an all-ones significand
            const long long eb = (long long)(u3 % 2000ull) + 20;
            b = __longlong_as_double((long long)(((u1 >> 63) << 63) | ((unsigned long long)eb << 52) | 0x000FFFFFFFFFFFFFull));
            a = wide_double(u0, u2);
            break;
        }
        }
        bool sp = false;
        const double q = hype::cr_div(a, b, sp);
        const double ref = a / b;
        if (sp) ++spec;
        else if (__double_as_longlong(q) != __double_as_longlong(ref)) ++mism;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mism += __shfl_xor_sync(0xffffffffu, mism, o);
        spec += __shfl_xor_sync(0xffffffffu, spec, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counts[0], mism);
        atomicAdd(&counts[1], spec);
    }
}
}  // namespace

extern "C" int hype_test_division(int device, long long n, unsigned long long seed, long long *mismatches, long long *specials)
{
    if (!mismatches || !specials || n < 0) return HYPE_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return HYPE_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return HYPE_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned long long *d = nullptr, h[2] = {0, 0};
    if (cudaMalloc(&d, sizeof(h)) != cudaSuccess) return HYPE_ERR_NOMEM;
    int rc = HYPE_OK;
    if (cudaMemset(d, 0, sizeof(h)) != cudaSuccess) rc = HYPE_ERR_CUDA;
    if (rc == HYPE_OK) {
        division_check_kernel<<<sms * 8, 256>>>(n, seed, d);
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) rc = HYPE_ERR_CUDA;
    }
    cudaFree(d);
    *mismatches = (long long)h[0];
    *specials = (long long)h[1];
    return rc;
}

extern "C" int hype_fp64_rate(int device, int reps, double *ops_per_s) { return fp64_rate_of(false, device, reps, ops_per_s); }
extern "C" int hype_fp64_fma_rate(int device, int reps, double *flops_per_s) { return fp64_rate_of(true, device, reps, flops_per_s); }
