// hype_noalloc.cu -- hype_rhs_prim_noalloc: the RHSFunctionPrim drop-in for
// callers that cannot allocate device memory.
//
// Who needs it: code that runs with its device memory owned by someone else --
// a host application or framework whose memory pool has already claimed the
// GPU, a plug-in loaded into such a process, or a caller that must not trigger
// the device-wide synchronisation and fragmentation a cudaMalloc/cudaFree pair
// brings in the middle of its time loop.  hype_create allocates per-grid
// buffers; this entry point allocates nothing.  Its working memory (the field
// planes the stage kernel streams through TMA, and the dt/error scalars) lives
// in one file-scope __device__ array of HYPE_NOALLOC_MAX_BYTES, which every GPU
// that loads this library holds until the process exits.
//
// Set-up: every call (with the target device current) looks up the array's
// device address with cudaGetSymbolAddress -- the name is only a host stand-in
// in host code, never a device pointer.  The lookup allocates nothing; doing it
// per call rather than once means a module that was reloaded (after
// cudaDeviceReset, or a primary context released and re-created) is never
// addressed through a stale pointer.  The first call on a device loads the
// module there, so make it before any stream capture.
//
// Stream: the work runs on the legacy default stream, which waits for and is
// waited for by work on ordinary (blocking) streams.  A caller that produced dU
// on a stream created with cudaStreamNonBlocking must synchronise that stream
// (or the device) before the call.
//
// Sharing: every call uses the same array and it keeps the last call's
// contents.  Each call clears the scalars that must start at zero and
// overwrites every plane value it reads.  Calls that overlap on the GPU (from
// several host threads, or on streams that do not order them) race on the
// array; serialise them.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstring>
#include "../../include/hype_gpu.h"
#include "hype_internal.h"

using namespace hype;

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[HYPE_NOALLOC_MAX_BYTES];

constexpr int kMaxDevices = 64;
constexpr size_t kPlanesOffset = 256;   // DevScalars first, planes after (256-byte aligned)
static_assert(sizeof(DevScalars) <= kPlanesOffset, "DevScalars must fit ahead of the planes");

__global__ void noalloc_reset_kernel(DevScalars *sc)
{
    sc->dt = 0.0; sc->t = 0.0; sc->t_final = 0.0; sc->time_step = 0.0;
    sc->smax = 0ull;
    sc->smax_v = 0ull;
    sc->r1h_v = 0.0;
    sc->err = 0u;
    sc->err_cell = 0xffffffffu;
    sc->steps = 0; sc->max_steps = 0; sc->done = 0; sc->hold = 0; sc->idle = 0; sc->pad_ = 0;
}

typedef CUresult (*PFN_encodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                     const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// the scratch array's device address on the current device `dev`
int scratch_on(int dev, unsigned char **out)
{
    if (dev < 0 || dev >= kMaxDevices) return HYPE_ERR_INVALID;
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return HYPE_ERR_CUDA;
    *out = static_cast<unsigned char *>(p);
    return HYPE_OK;
}

int check(const hype_config *c)
{
    if (!c || hype_nvar(c->system) == 0) return HYPE_ERR_INVALID;
    if (c->order < 0 || c->order > 3 || c->nx < 3 || c->ny < 3) return HYPE_ERR_INVALID;
    if (!(c->x_max > c->x_min) || !(c->y_max > c->y_min) || !(c->cfl > 0.0)) return HYPE_ERR_INVALID;
    if (c->precision != HYPE_PREC_FP64) return HYPE_ERR_INVALID;
    if (c->flags & (HYPE_FLAG_CONSERVATIVE | HYPE_FLAG_VISCOUS)) return HYPE_ERR_INVALID;
    const int bcs[4] = {c->bc_left, c->bc_right, c->bc_bottom, c->bc_top};
    for (int k = 0; k < 4; ++k)   // inlet needs a per-call host table; wall is never filled by the reference
        if (bcs[k] != HYPE_BC_PERIODIC && bcs[k] != HYPE_BC_REFLECTIVE && bcs[k] != HYPE_BC_TRANSMISSIVE) return HYPE_ERR_INVALID;
    if ((c->bc_left == HYPE_BC_PERIODIC) != (c->bc_right == HYPE_BC_PERIODIC) ||
        (c->bc_bottom == HYPE_BC_PERIODIC) != (c->bc_top == HYPE_BC_PERIODIC))
        return HYPE_ERR_INVALID;
    return HYPE_OK;
}

}  // namespace

extern "C" HYPE_API int hype_rhs_prim_noalloc(const hype_config *cfg, double t, const double *dU, double *dRHS, double *dt)
{
    (void)t;
    int rc = check(cfg);
    if (rc) return rc;
    const int nv = hype_nvar(cfg->system);
    const int pitch = (cfg->nx + 15) & ~15;
    const long long plane = (long long)pitch * cfg->ny;
    const unsigned long long need = kPlanesOffset + (unsigned long long)plane * nv * sizeof(double);
    if (need > HYPE_NOALLOC_MAX_BYTES) return HYPE_ERR_NOMEM;   // grid larger than the static scratch
    if (!dU || !dRHS) return HYPE_ERR_INVALID;

    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return HYPE_ERR_NO_DEVICE;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return HYPE_ERR_NO_DEVICE;
    struct Restore { int d; ~Restore() { cudaSetDevice(d); } } restore{prev};

    unsigned char *base = nullptr;
    if ((rc = scratch_on(cfg->device, &base))) return rc;
    DevScalars *sc = reinterpret_cast<DevScalars *>(base);
    double *planes = reinterpret_cast<double *>(base + kPlanesOffset);

    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
        return HYPE_ERR_CUDA;
    CUtensorMap tm;
    cuuint64_t dims[3] = {(cuuint64_t)cfg->nx, (cuuint64_t)cfg->ny, (cuuint64_t)nv};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * 8ull, (cuuint64_t)plane * 8ull};
    cuuint32_t box[3] = {(cuuint32_t)stage_box_width(STAGE_CELLS, nv), 1u, (cuuint32_t)nv};
    cuuint32_t estr[3] = {1u, 1u, 1u};
    if (reinterpret_cast<PFN_encodeTiled>(fn)(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, planes, dims, strides, box, estr,
                                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return HYPE_ERR_CUDA;

    if (stage_configure(cfg->system, cfg->order, STAGE_CELLS) != cudaSuccess) return HYPE_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg->device) != cudaSuccess) return HYPE_ERR_CUDA;
    const int bps = stage_blocks_per_sm(cfg->system, cfg->order, STAGE_CELLS);
    if (bps < 1) return HYPE_ERR_CUDA;
    const int strips = stage_strips(cfg->nx, STAGE_CELLS);
    int runs = sms * bps / strips;
    if (runs < 1) runs = 1;
    if (runs > cfg->ny / 8) runs = cfg->ny / 8 > 0 ? cfg->ny / 8 : 1;

    StageParams p;
    std::memset(&p, 0, sizeof(p));
    p.nx = cfg->nx; p.ny = cfg->ny; p.pitch = pitch; p.plane = plane; p.strips = strips; p.runs = runs;
    p.bc[0] = cfg->bc_left; p.bc[1] = cfg->bc_right; p.bc[2] = cfg->bc_bottom; p.bc[3] = cfg->bc_top;
    p.eos.g1 = cfg->gamma1; p.eos.g2 = cfg->gamma2; p.eos.pi1 = cfg->pi1; p.eos.pi2 = cfg->pi2;
    p.eos.fix_p2 = (cfg->flags & HYPE_FLAG_BN_FIX_P2) ? 1 : 0;
    const double h = (cfg->x_max - cfg->x_min) / (double)cfg->nx;   // hype.c:57
    p.r1_h = 1. / h;
    p.cfl_h = cfg->cfl * h;
    p.in = planes; p.out = dRHS; p.out_aos = 1; p.mode = OUT_RHS; p.kb = 1.0;
    p.sc = sc; p.reduce_smax = 1;

    noalloc_reset_kernel<<<1, 1, 0, 0>>>(sc);
    if (cudaGetLastError() != cudaSuccess) return HYPE_ERR_CUDA;
    if (launch_aos_to_planes(dU, planes, cfg->nx, cfg->ny, nv, pitch, plane, 0) != cudaSuccess) return HYPE_ERR_CUDA;
    if (launch_stage(cfg->system, cfg->order, STAGE_CELLS, tm, p, 0) != cudaSuccess) return HYPE_ERR_CUDA;
    DevScalars h_sc;
    if (cudaMemcpy(&h_sc, sc, sizeof(h_sc), cudaMemcpyDeviceToHost) != cudaSuccess) return HYPE_ERR_CUDA;
    if (h_sc.err & ERR_TMA_TIMEOUT) return HYPE_ERR_TIMEOUT;
    if (h_sc.err & ERR_BAD_LAUNCH) return HYPE_ERR_CUDA;
    if (dt) {
        double smax;
        std::memcpy(&smax, &h_sc.smax, sizeof(smax));
        *dt = (cfg->cfl * h) / (2.0 * smax);   // rhs_function_prim.c:620
    }
    return (h_sc.err & ERR_INADMISSIBLE_FACE) ? HYPE_ERR_INADMISSIBLE : HYPE_OK;
}
