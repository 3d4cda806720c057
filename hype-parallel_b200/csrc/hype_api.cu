// hype_api.cu -- the C ABI of include/hype_gpu.h: solver objects, device
// buffers, TMA descriptors, the RHSFunctionPrim drop-in and the device-resident
// SSP-RK time loop (captured once per solver as a CUDA graph and replayed).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#include "../../include/hype_gpu.h"
#include "hype_internal.h"
#include "hype_solver.h"

using namespace hype;


// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
static int fail(hype_solver *s, int code, const char *fmt, ...)
{
    if (s) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(s->err, sizeof(s->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

int hype::solver_fail(hype_solver *s, int code, const char *fmt, ...)
{
    if (s) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(s->err, sizeof(s->err), fmt, ap);
        va_end(ap);
    }
    return code;
}
#define CUDA_TRY(s, expr)                                                                                  \
    do {                                                                                                   \
        cudaError_t e_ = (expr);                                                                           \
        if (e_ != cudaSuccess) return fail((s), HYPE_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

typedef CUresult (*PFN_tmapEncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                         const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                         CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_tmapEncodeTiled get_encode()
{
    static PFN_tmapEncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_tmapEncodeTiled>(p);
    }
    return fn;
}

namespace hype {
CUresult encode_planes_map(CUtensorMap *m, const void *base, bool fp32, int nx, int ny, int nplanes, int pitch, long long plane,
                           int box_w)
{
    PFN_tmapEncodeTiled enc = get_encode();
    if (!enc) return CUDA_ERROR_NOT_SUPPORTED;
    const cuuint64_t es = fp32 ? 4ull : 8ull;
    cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nplanes};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * es, (cuuint64_t)plane * es};
    cuuint32_t box[3] = {(cuuint32_t)box_w, 1u, (cuuint32_t)nplanes};
    cuuint32_t estr[3] = {1u, 1u, 1u};
    return enc(m, fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), dims,
               strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}
}  // namespace hype

// 3-D map over the field planes: dims (x = nx, y = ny, z = nvar), box (cells + 6, 1, nvar);
// a slab's map also covers its halo rows and starts row_off rows below row 0, a
// block's also its halo columns, starting col_off columns left of column 0.
static int make_tmap(hype_solver *s, CUtensorMap *m, double *base)
{
    CUresult r = encode_planes_map(m, base - (long long)s->row_off * s->pitch - s->col_off, false, s->cfg.nx + 2 * s->col_off,
                                   s->cfg.ny + 2 * s->row_off, s->nv, s->pitch, s->plane, stage_box_width(s->cells, s->nv));
    if (r != CUDA_SUCCESS) return fail(s, HYPE_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return HYPE_OK;
}

// kapila_5eqn.c:485-513 evaluated once on the host (the profile does not depend
// on t) for the three left ghost columns of every ghost-extended row.
void hype::inlet_table(const hype_config &c, double h, std::vector<double> &tab)
{
    const int ny = c.ny, nv = hype_nvar(c.system);
    tab.assign((size_t)3 * (ny + 6) * nv, 0.0);
    for (int g = -3; g < 0; ++g)
        for (int j = -3; j < ny + 3; ++j) {
            const double y = c.y_min + ((double)j + 0.5) * h;
            const double M = 2.0, rho_air = 1.0, rho_water = 1000.0, P = 1.013;
            const double U_avg = M * std::sqrt(c.gamma2 * P / rho_air);
            const double phi_R = 1.0 - 1.0e-6, phi_L = 1.0e-6;
            const double PHI = 0.5 * (phi_R + phi_L);
            const double dif_phi = (phi_L - phi_R) / 2.0;
            const double hh = 30.0 / 500.0;
            const double epsilon = 3.0 * hh;
            const double r_0 = 1.0;
            const double r = std::fabs(y);
            double *V = &tab[((size_t)(g + 3) * (ny + 6) + (j + 3)) * nv];
            V[0] = rho_water;
            V[1] = rho_air;
            V[2] = (r < 1.0) ? 2.0 * U_avg * (1.0 - y * y) : 0.0;
            V[3] = 0.0;
            V[4] = P;
            V[5] = PHI + dif_phi * std::tanh(-(r - r_0) / epsilon);
        }
}

// InletBC = PDEPrim2Cons(InletBCPrim(...)) (kapila_5eqn.c:289-320, 41-61),
// evaluated on the host for the conservative path's ghost columns.
void hype::inlet_to_conserved(const hype_config &c, std::vector<double> &tab)
{
    const double G1m1 = c.gamma1 - 1.0, G2m1 = c.gamma2 - 1.0;
    for (size_t k = 0; k + 6 <= tab.size(); k += 6) {
        double *V = &tab[k];
        const double alpha_1 = V[5];
        const double alpha_2 = 1.0 - alpha_1;
        const double rho = alpha_1 * V[0] + alpha_2 * V[1];
        const double u = V[2], v = V[3], p = V[4];
        const double ei = (p * (alpha_1 * G2m1 + alpha_2 * G1m1) + alpha_1 * c.gamma1 * c.pi1 * G2m1 + alpha_2 * c.gamma2 * c.pi2 * G1m1) / (G1m1 * G2m1);
        const double E = ei + 0.5 * rho * (u * u + v * v);
        const double Q[6] = {alpha_1 * V[0], alpha_2 * V[1], rho * V[2], rho * V[3], E, alpha_1};
        for (int q = 0; q < 6; ++q) V[q] = Q[q];
    }
}

static StageParams base_params(const hype_solver *s)
{
    StageParams p;
    std::memset(&p, 0, sizeof(p));
    p.nx = s->cfg.nx; p.ny = s->cfg.ny; p.pitch = s->pitch; p.plane = s->plane;
    p.strips = s->strips; p.runs = s->runs;
    p.bc[0] = s->cfg.bc_left; p.bc[1] = s->cfg.bc_right; p.bc[2] = s->cfg.bc_bottom; p.bc[3] = s->cfg.bc_top;
    p.eos.g1 = s->cfg.gamma1; p.eos.g2 = s->cfg.gamma2; p.eos.pi1 = s->cfg.pi1; p.eos.pi2 = s->cfg.pi2;
    p.eos.fix_p2 = (s->cfg.flags & HYPE_FLAG_BN_FIX_P2) ? 1 : 0;
    p.eos.derive();
    p.r1_h = s->r1_h;
    p.cfl_h = s->cfl_h;
    p.mu1 = s->cfg.mu1;
    p.mu2 = s->cfg.mu2;
    p.sc = s->dSc;
    p.inlet = s->dInlet;
    p.kb = 1.0;
    p.row_off = s->row_off;
    p.col_off = s->col_off;
    if (s->test_skip_row >= 0) { p.skip_loads = 1; p.skip_loads_from = s->test_skip_row; }
    return p;
}

// Tile width and decomposition: `waves` waves of strips x row runs (<= SMs x
// resident blocks each), at least 8 rows per run.  Rebuilds the TMA
// descriptors, whose box width follows the tile width, and drops the captured
// step graph (recaptured on the next hype_begin / hype_advance).
// FP32 (nf planes) and FP64 (nd planes) maps of a mixed state (MixedLayout), box
// (cells + 8, 1, planes); a slab's maps also cover its halo rows and start row_off
// rows below row 0
static int make_mixed_maps(hype_solver *s, MixedMaps *mm, float *pf, double *pd)
{
    const int bw = mixed_box_width(s->cells);
    const long long off = (long long)s->row_off * s->pitch;
    const int rows = s->cfg.ny + 2 * s->row_off;
    const MixedLayout L = mixed_layout(s->cfg.system);
    CUresult r = encode_planes_map(&mm->f, pf - off, true, s->cfg.nx, rows, L.nf, s->pitch, s->plane, bw);
    if (r != CUDA_SUCCESS) return fail(s, HYPE_ERR_CUDA, "cuTensorMapEncodeTiled (FP32 planes) failed (%d)", (int)r);
    r = encode_planes_map(&mm->d, pd - off, false, s->cfg.nx, rows, L.nd, s->pitch, s->plane, bw);
    if (r != CUDA_SUCCESS) return fail(s, HYPE_ERR_CUDA, "cuTensorMapEncodeTiled (FP64 planes) failed (%d)", (int)r);
    return HYPE_OK;
}

static int set_tiling(hype_solver *s, int cells, int waves = 1)
{
    const hype_config *cfg = &s->cfg;
    int rc;
    s->cells = cells;
    if (s->mixed) {
        s->bps = mixed_blocks_per_sm(cfg->system, cells);
        if (s->bps < 1) return fail(s, HYPE_ERR_CUDA, "mixed stage kernel does not fit on an SM");
        s->strips = mixed_strips(cfg->nx, cells);
        s->waves = waves > 0 ? waves : 1;
        int runs = s->sms * s->bps * s->waves / s->strips;
        if (runs < 1) runs = 1;
        if (runs > cfg->ny / 8) runs = cfg->ny / 8 > 0 ? cfg->ny / 8 : 1;
        s->runs = runs;
        for (int k = 0; k < 3; ++k)
            if ((rc = make_mixed_maps(s, &s->mm[k], s->mf[k], s->md[k]))) return rc;
        if (s->step_exec) { cudaGraphExecDestroy(s->step_exec); s->step_exec = nullptr; }
        return HYPE_OK;
    }
    if (cfg->flags & HYPE_FLAG_VISCOUS) {   // the viscous kernels come in 128-column tiles only
        cells = STAGE_CELLS;
        s->cells = cells;
        const bool cons = (cfg->flags & HYPE_FLAG_CONSERVATIVE) != 0;
        CUDA_TRY(s, stage_visc_configure(cfg->order, cons));
        s->bps = stage_visc_blocks_per_sm(cfg->order, cons);
    } else if (cfg->flags & HYPE_FLAG_CONSERVATIVE) {   // the conservative kernels come in 128-column tiles only
        cells = STAGE_CELLS;
        s->cells = cells;
        CUDA_TRY(s, stage_cons_configure(cfg->system, cfg->order));
        s->bps = stage_cons_blocks_per_sm(cfg->system, cfg->order);
    } else if (s->fast) {
        CUDA_TRY(s, stage_fast_configure(cfg->system, cfg->order, cells));
        s->bps = stage_fast_blocks_per_sm(cfg->system, cfg->order, cells);
    } else {
        CUDA_TRY(s, stage_configure(cfg->system, cfg->order, cells));
        s->bps = stage_blocks_per_sm(cfg->system, cfg->order, cells);
    }
    if (s->bps < 1) return fail(s, HYPE_ERR_CUDA, "stage kernel does not fit on an SM");
    s->strips = stage_strips(cfg->nx, cells);
    const int slots = s->sms * s->bps * (waves > 0 ? waves : 1);
    s->waves = waves > 0 ? waves : 1;
    int runs = slots / s->strips;
    if (runs < 1) runs = 1;
    if (runs > cfg->ny / 8) runs = cfg->ny / 8 > 0 ? cfg->ny / 8 : 1;
    s->runs = runs;
    if ((rc = make_tmap(s, &s->tmU, s->dU)) || (rc = make_tmap(s, &s->tmS0, s->dS0)) || (rc = make_tmap(s, &s->tmS1, s->dS1))) return rc;
    if (s->step_exec) { cudaGraphExecDestroy(s->step_exec); s->step_exec = nullptr; }
    return HYPE_OK;
}


static const CUtensorMap &tmap_for(const hype_solver *s, const double *buf)
{
    return buf == s->dU ? s->tmU : buf == s->dS0 ? s->tmS0 : s->tmS1;
}

static cudaError_t stage(hype_solver *s, const double *in, double *out, int mode, double ka, double kb, double kc,
                         const double *xn, double *out2, int reduce, int out_aos = 0, int run0 = 0, int run_count = 0,
                         int push_role = B_NONE)
{
    StageParams p = base_params(s);
    p.in = in; p.out = out; p.mode = mode; p.ka = ka; p.kb = kb; p.kc = kc; p.xn = xn; p.out2 = out2;
    p.reduce_smax = reduce;
    p.out_aos = out_aos;
    p.run0 = run0;
    p.run_count = run_count;
    if (push_role >= 0 && mode != OUT_RHS) {   // a slab's state output: edge rows to the neighbours' halos
        p.push_lo = s->nb_lo[push_role]; p.push_plane_lo = s->nb_plane_lo; p.push_shift_lo = s->nb_shift_lo;
        p.push_hi = s->nb_hi[push_role]; p.push_plane_hi = s->nb_plane_hi; p.push_shift_hi = s->nb_shift_hi;
    }
    if (s->cfg.flags & HYPE_FLAG_VISCOUS)
        return launch_stage_visc(s->cfg.order, (s->cfg.flags & HYPE_FLAG_CONSERVATIVE) != 0, tmap_for(s, in), p, s->stream);
    if (s->cfg.flags & HYPE_FLAG_CONSERVATIVE) return launch_stage_cons(s->cfg.system, s->cfg.order, tmap_for(s, in), p, s->stream);
    if (s->fast) return launch_stage_fast(s->cfg.system, s->cfg.order, s->cells, tmap_for(s, in), p, s->stream);
    return launch_stage(s->cfg.system, s->cfg.order, s->cells, tmap_for(s, in), p, s->stream);
}

// mixed-precision stage: input state k_in, output k_out (or the interleaved
// FP64 RHS for OUT_RHS), second state k_x
static cudaError_t stage_m(hype_solver *s, int k_in, int k_out, int mode, double ka, double kb, double kc, int k_x, int reduce,
                           double *out_rhs = nullptr, bool push = false, int run0 = 0, int run_count = 0)
{
    MixedParams p;
    std::memset(&p, 0, sizeof(p));
    p.nx = s->cfg.nx; p.ny = s->cfg.ny; p.pitch = s->pitch; p.plane = s->plane;
    p.bc[0] = s->cfg.bc_left; p.bc[1] = s->cfg.bc_right; p.bc[2] = s->cfg.bc_bottom; p.bc[3] = s->cfg.bc_top;
    p.eos.g1 = s->cfg.gamma1; p.eos.g2 = s->cfg.gamma2; p.eos.pi1 = s->cfg.pi1; p.eos.pi2 = s->cfg.pi2;
    p.eos.fix_p2 = (s->cfg.flags & HYPE_FLAG_BN_FIX_P2) ? 1 : 0;
    p.r1_h = s->r1_h; p.cfl_h = s->cfl_h;
    p.in_f = s->mf[k_in]; p.in_d = s->md[k_in];
    if (k_x >= 0) { p.xn_f = s->mf[k_x]; p.xn_d = s->md[k_x]; }
    if (k_out >= 0) { p.out_f = s->mf[k_out]; p.out_d = s->md[k_out]; }
    p.out_rhs = out_rhs;
    p.mode = mode; p.ka = ka; p.kb = kb; p.kc = kc;
    p.sc = s->dSc; p.reduce_smax = reduce;
    p.strips = s->strips; p.runs = s->runs;
    p.run0 = run0; p.run_count = run_count;
    p.row_off = s->row_off;
    if (s->test_skip_row >= 0) { p.skip_loads = 1; p.skip_loads_from = s->test_skip_row; }
    if (push && k_out >= 0 && mode != OUT_RHS) {   // a slab's state output: edge rows to the neighbours' halos
        p.push_lo_f = s->nbf_lo[k_out]; p.push_lo_d = s->nbd_lo[k_out];
        p.push_hi_f = s->nbf_hi[k_out]; p.push_hi_d = s->nbd_hi[k_out];
        p.push_plane_lo = s->nb_plane_lo; p.push_shift_lo = s->nb_shift_lo;
        p.push_plane_hi = s->nb_plane_hi; p.push_shift_hi = s->nb_shift_hi;
    }
    return launch_mixed(s->cfg.system, s->cells, s->mm[k_in], p, s->stream);
}

static double *buf_of(hype_solver *s, int b)
{
    switch (b) {
    case B_U: return s->dU;
    case B_S0: return s->dS0;
    case B_S1: return s->dS1;
    case B_S2: return s->dS2;
    default: return nullptr;
    }
}

double *hype::solver_buf(hype_solver *s, int role) { return buf_of(s, role); }
double *hype::solver_alloc_base(const hype_solver *s, double *buf)
{
    return buf ? buf - (long long)s->row_off * s->pitch - s->col_off : nullptr;
}

cudaError_t hype::solver_stage(hype_solver *s, const PlanStage &q)
{
    if (s->mixed) return stage_m(s, q.in, q.out, q.mode, q.ka, q.kb, q.kc, q.x, q.reduce, nullptr, true);
    return stage(s, buf_of(s, q.in), buf_of(s, q.out), q.mode, q.ka, q.kb, q.kc, buf_of(s, q.x), buf_of(s, q.out2), q.reduce, 0, 0, 0,
                 q.out);
}

// hype.c:343's seeding RHS of u: S1 takes the (unused) RHS planes
cudaError_t hype::solver_seed_rhs(hype_solver *s)
{
    if (s->mixed) return stage_m(s, 0, -1, OUT_RHS, 0, 1.0, 0, -1, 1, s->dAosOut);
    return stage(s, s->dU, s->dS1, OUT_RHS, 0, 1.0, 0, nullptr, nullptr, 1);
}

// One SSP-RK step on the device state: the stage list of ssp_plan between the
// step-control kernels.  The mixed state has the same buffer roles (U, S0, S1).
static cudaError_t enqueue_step(hype_solver *s)
{
    cudaError_t e;
    PlanStage plan[MAX_PLAN];
    int copy_back = 0;
    const int ns = ssp_plan(s->cfg.order, plan, &copy_back);
    if ((e = launch_begin_step(s->dSc, s->stream)) != cudaSuccess) return e;
    for (int k = 0; k < ns; ++k) {
        const PlanStage &q = plan[k];
        if (s->mixed) e = stage_m(s, q.in, q.out, q.mode, q.ka, q.kb, q.kc, q.x, q.reduce);
        else e = stage(s, buf_of(s, q.in), buf_of(s, q.out), q.mode, q.ka, q.kb, q.kc, buf_of(s, q.x), buf_of(s, q.out2), q.reduce);
        if (e != cudaSuccess) return e;
    }
    if (copy_back &&
        (e = cudaMemcpyAsync(solver_alloc_base(s, s->dU), solver_alloc_base(s, s->dS0), sizeof(double) * (size_t)s->plane * s->nv,
                             cudaMemcpyDeviceToDevice, s->stream)) != cudaSuccess)
        return e;
    return launch_end_step(s->dSc, s->cfl_h, s->stream);
}

static int check_config(const hype_config *c, hype_solver *s);
int hype::validate_config(const hype_config *c, char *err, size_t errlen)
{
    hype_solver tmp;
    const int rc = check_config(c, &tmp);
    if (rc && err && errlen) snprintf(err, errlen, "%s", tmp.err);
    return rc;
}

static int check_config(const hype_config *c, hype_solver *s)
{
    if (!c) return fail(s, HYPE_ERR_INVALID, "null config");
    if (hype_nvar(c->system) == 0) return fail(s, HYPE_ERR_INVALID, "unknown system %d", c->system);
    if (c->order < 0 || c->order > 3) return fail(s, HYPE_ERR_INVALID, "order must be 0..3 (got %d)", c->order);
    if (c->nx < 3 || c->ny < 3) return fail(s, HYPE_ERR_INVALID, "grid must be at least 3x3 (got %dx%d)", c->nx, c->ny);
    if ((long long)c->nx * c->ny > (1LL << 31) - 1) return fail(s, HYPE_ERR_INVALID, "grid too large");
    if (!(c->x_max > c->x_min) || !(c->y_max > c->y_min)) return fail(s, HYPE_ERR_INVALID, "empty domain");
    if (!(c->cfl > 0.0)) return fail(s, HYPE_ERR_INVALID, "CFL must be positive");
    const int bcs[4] = {c->bc_left, c->bc_right, c->bc_bottom, c->bc_top};
    for (int k = 0; k < 4; ++k) {
        if (bcs[k] < 0 || bcs[k] > 4) return fail(s, HYPE_ERR_INVALID, "unknown boundary type %d", bcs[k]);
        if (bcs[k] == HYPE_BC_WALL)
            return fail(s, HYPE_ERR_INVALID, "wall boundaries are not supported (the reference never fills their ghost cells)");
        if (bcs[k] == HYPE_BC_INLET && (k != 0 || c->system != HYPE_KAPILA_5EQN))
            return fail(s, HYPE_ERR_INVALID, "inlet boundary exists only on the left for the Kapila system (InletBCPrim)");
    }
    if ((c->bc_left == HYPE_BC_PERIODIC) != (c->bc_right == HYPE_BC_PERIODIC) ||
        (c->bc_bottom == HYPE_BC_PERIODIC) != (c->bc_top == HYPE_BC_PERIODIC))
        return fail(s, HYPE_ERR_INVALID, "periodic boundaries must be set on both sides of an axis");
    if (c->precision != HYPE_PREC_FP64 && c->precision != HYPE_PREC_MIXED && c->precision != HYPE_PREC_FP64_FAST)
        return fail(s, HYPE_ERR_INVALID, "unknown precision %d", c->precision);
    if (c->precision == HYPE_PREC_FP64_FAST && (c->flags & (HYPE_FLAG_CONSERVATIVE | HYPE_FLAG_VISCOUS)))
        return fail(s, HYPE_ERR_INVALID, "the FP64 performance form covers the primitive-variable inviscid path");
    if (c->precision == HYPE_PREC_MIXED && (c->order != 2 || c->bc_left == HYPE_BC_INLET))
        return fail(s, HYPE_ERR_INVALID, "mixed precision is implemented for N = 2 without inlet boundaries");
    if (c->precision == HYPE_PREC_MIXED && (c->flags & HYPE_FLAG_CONSERVATIVE))
        return fail(s, HYPE_ERR_INVALID, "the conservative-variable path is FP64 only");
    if (c->flags & ~(HYPE_FLAG_BN_FIX_P2 | HYPE_FLAG_CONSERVATIVE | HYPE_FLAG_VISCOUS))
        return fail(s, HYPE_ERR_INVALID, "unknown flags 0x%x", c->flags);
    if ((c->flags & HYPE_FLAG_VISCOUS) &&
        (c->system != HYPE_KAPILA_5EQN || c->order < 1 || c->precision != HYPE_PREC_FP64))
        return fail(s, HYPE_ERR_INVALID, "the viscous path exists for the Kapila system, N = 1..3, FP64 "
                                         "(the reference's other systems have no usable viscous flux; N = 0 has no gradients)");
    return HYPE_OK;
}

// ---------------------------------------------------------------------------
// Banded host calls.  The grid's rows are split into row bands, each a set of
// row runs launched on its own, so that device work starts before the whole
// state has arrived and the result leaves band by band:
//  - host->device: every band's rows are copied back to back on `cin`; the
//    conversion to planes runs on `cvin` behind each copy, so the copy engine
//    never waits for SM slots (ev_cp: copied, ev_in: converted);
//  - device->host: a band's result is converted on `cvout` once computed and
//    copied out on `cout` (ev_dc: converted);
//  - up to 16 bands, each launch covering half a wave of blocks (host_bands);
//  - hype_rhs_prim: its one RHS launch, band by band behind the uploads
//    (banded_upload_stage).  On a 2048^2 Kapila grid a call took 5.4-5.5 ms
//    with 8 full-wave bands and 4.8 ms this way (the copies alone: 3.6 ms each
//    way, 4.1 ms both ways at once);
//  - hype_advance_host: every stage of the step as a wavefront over the bands
//    (enqueue_step_banded).  Stage s runs on compute stream s % 4, so the four
//    SSPRK(4,3) stages advance together, each band of stage s waiting only for
//    the bands of stage s-1 its stencils read (band k-1..k+1), and launches of
//    neighbouring stages share the SMs.  On the same grid one step with its
//    copies took 12.0-12.6 ms with 8 full-wave bands and alternating stages on
//    two streams, and 10.2-10.5 ms this way (the device-only step: 8.6 ms).
// Results do not depend on the decomposition.
// ---------------------------------------------------------------------------
struct Bands {
    int n;
    int runs;                              // runs of the banded launches
    int run[hype_solver::MAX_BANDS + 1];   // band k: runs run[k] .. run[k+1]-1
    int row[hype_solver::MAX_BANDS + 1];   //         rows row[k] .. row[k+1]-1 (those runs' own rows)
    int order[hype_solver::MAX_BANDS];     // launch order: band 0 last on a periodic y axis (it reads the last band)
};

// up to `max_bands` bands of at least `per` runs each (fewer bands on short grids,
// so that no launch shrinks below `per` runs), at least 8 rows per run
static Bands make_bands(const hype_solver *s, int max_bands, int per)
{
    Bands b;
    const int ny = s->cfg.ny;
    if (max_bands > hype_solver::MAX_BANDS) max_bands = hype_solver::MAX_BANDS;
    if (per < 1) per = 1;
    int runs = max_bands * per;
    const int cap = ny / 8 > s->runs ? ny / 8 : s->runs;
    if (runs > cap) runs = cap;
    if (runs < 1) runs = 1;
    b.runs = runs;
    b.n = runs / per < 1 ? 1 : (runs / per > max_bands ? max_bands : runs / per);
    for (int k = 0; k <= b.n; ++k) {
        b.run[k] = (int)(((long long)k * runs) / b.n);
        b.row[k] = (int)(((long long)b.run[k] * ny) / runs);
    }
    const bool py = s->cfg.bc_bottom == HYPE_BC_PERIODIC && b.n > 1;
    for (int k = 0; k < b.n; ++k) b.order[k] = py ? (k + 1) % b.n : k;
    return b;
}

// row runs of one wave of stage blocks
static int wave_runs(const hype_solver *s)
{
    const int r = s->sms * s->bps / (s->strips > 0 ? s->strips : 1);
    return r > 0 ? r : 1;
}

// the bands of the host calls: launches of half a wave of blocks
static Bands host_bands(const hype_solver *s) { return make_bands(s, hype_solver::MAX_BANDS, wave_runs(s) / 2); }

// the last band whose rows band k's stencils read (the halo is 3 rows, bands are >= 8)
static int band_needs(const hype_solver *s, const Bands &b, int k)
{
    if (k == 0 && s->cfg.bc_bottom == HYPE_BC_PERIODIC) return b.n - 1;
    return k + 1 < b.n ? k + 1 : b.n - 1;
}

// the copy streams start after the compute stream's work enqueued so far
static int fence_copy_streams(hype_solver *s)
{
    CUDA_TRY(s, cudaEventRecord(s->ev_fence, s->stream));
    CUDA_TRY(s, cudaStreamWaitEvent(s->cin, s->ev_fence, 0));
    CUDA_TRY(s, cudaStreamWaitEvent(s->cout, s->ev_fence, 0));
    CUDA_TRY(s, cudaStreamWaitEvent(s->cvin, s->ev_fence, 0));
    CUDA_TRY(s, cudaStreamWaitEvent(s->cvout, s->ev_fence, 0));
    return HYPE_OK;
}

// rows r0 .. r0+nr-1 of the input staging array (cell-major) -> state buffer `role`
// (FP64 planes, or the FP32 and FP64 planes of the mixed state)
static cudaError_t rows_to_state(hype_solver *s, int role, int r0, int nr, cudaStream_t on)
{
    if (s->mixed) {
        const long long o = (long long)r0 * s->pitch;
        return launch_aos_to_mixed(s->cfg.system, s->dAosIn + (size_t)r0 * s->cfg.nx * s->nv, s->mf[role] + o, s->md[role] + o,
                                   s->cfg.nx, nr, s->pitch, s->plane, on);
    }
    return launch_aos_to_planes_rows(s->dAosIn, buf_of(s, role), s->cfg.nx, r0, nr, s->nv, s->pitch, s->plane, on);
}

// rows r0 .. r0+nr-1 of state buffer `role` -> the output staging array (cell-major)
static cudaError_t state_to_rows(hype_solver *s, int role, int r0, int nr, cudaStream_t on)
{
    if (s->mixed) {
        const long long o = (long long)r0 * s->pitch;
        return launch_mixed_to_aos(s->cfg.system, s->mf[role] + o, s->md[role] + o, s->dAosOut + (size_t)r0 * s->cfg.nx * s->nv,
                                   s->cfg.nx, nr, s->pitch, s->plane, on);
    }
    return launch_planes_to_aos_rows(buf_of(s, role), s->dAosOut, s->cfg.nx, r0, nr, s->nv, s->pitch, s->plane, on);
}

// Host side of a banded call: a pageable caller array goes through pinned staging
// (its bands copied by the host copy pool, hype_hostcopy.cu), a pinned one is
// copied directly.  Downloads into staging are finished on the host, band by
// band as they land, by finish_downloads.
struct HostIO {
    bool stage_in = false, stage_out = false;
    int nd = 0;   // staged downloads enqueued
    struct Pending { int k; size_t off, n; } d[hype_solver::MAX_BANDS];
};

static HostIO host_io(hype_solver *s, const void *in, const void *out)
{
    HostIO io;
    const bool want_in = in && host_is_pageable(in), want_out = out && host_is_pageable(out);
    if ((want_in || want_out) && !s->hStageIn) {   // first use; without pinned memory the copies stay direct
        void *a = nullptr, *o = nullptr;
        const bool ok_a = cudaHostAlloc(&a, s->aos_bytes, cudaHostAllocDefault) == cudaSuccess;
        const bool ok_o = ok_a && cudaHostAlloc(&o, s->aos_bytes, cudaHostAllocDefault) == cudaSuccess;
        if (ok_a && ok_o) {
            s->hStageIn = (double *)a;
            s->hStageOut = (double *)o;
        } else {
            cudaGetLastError();   // the failed allocation's error is not the call's
            if (ok_a) cudaFreeHost(a);
        }
    }
    io.stage_in = want_in && s->hStageIn;
    io.stage_out = want_out && s->hStageOut;
    return io;
}

// n elements at element offset `off` of the output staging array (dAosOut) to
// dst + off, on `cout` behind what it waits for (band k of the call)
static int download_rows(hype_solver *s, HostIO &io, int k, double *dst, size_t off, size_t n)
{
    if (!io.stage_out) {
        CUDA_TRY(s, cudaMemcpyAsync(dst + off, s->dAosOut + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->cout));
        return HYPE_OK;
    }
    CUDA_TRY(s, cudaMemcpyAsync(s->hStageOut + off, s->dAosOut + off, sizeof(double) * n, cudaMemcpyDeviceToHost, s->cout));
    CUDA_TRY(s, cudaEventRecord(s->ev_dl[k], s->cout));
    io.d[io.nd++] = {k, off, n};
    return HYPE_OK;
}

// the staged downloads to dst as they land, then every copy of the call done
static int finish_downloads(hype_solver *s, HostIO &io, double *dst)
{
    for (int j = 0; j < io.nd; ++j) {
        const HostIO::Pending &d = io.d[j];
        CUDA_TRY(s, cudaEventSynchronize(s->ev_dl[d.k]));
        host_copy(dst + d.off, s->hStageOut + d.off, sizeof(double) * d.n);
    }
    io.nd = 0;
    CUDA_TRY(s, cudaStreamSynchronize(s->cout));
    return HYPE_OK;
}

// host Vec rows of band k -> state buffer `role` (via the staging array); ev_in[k] marks them ready
static int upload_band(hype_solver *s, const Bands &b, int k, const double *U, int role, const HostIO &io)
{
    const size_t row_elems = (size_t)s->cfg.nx * s->nv;
    const int r0 = b.row[k], nr = b.row[k + 1] - r0;
    const double *from = U + r0 * row_elems;
    if (io.stage_in) {
        host_copy(s->hStageIn + r0 * row_elems, from, sizeof(double) * row_elems * nr);
        from = s->hStageIn + r0 * row_elems;
    }
    CUDA_TRY(s, cudaMemcpyAsync(s->dAosIn + r0 * row_elems, from, sizeof(double) * row_elems * nr, cudaMemcpyHostToDevice, s->cin));
    CUDA_TRY(s, cudaEventRecord(s->ev_cp[k], s->cin));
    CUDA_TRY(s, cudaStreamWaitEvent(s->cvin, s->ev_cp[k], 0));
    CUDA_TRY(s, rows_to_state(s, role, r0, nr, s->cvin));
    CUDA_TRY(s, cudaEventRecord(s->ev_in[k], s->cvin));
    return HYPE_OK;
}

// one stage of `q` over band k's runs of the banded decomposition, on stream `on`
// (the solver's compute stream by default); `out` (with out_aos) replaces q.out,
// for the mixed state an RHS output (OUT_RHS) only
static cudaError_t stage_band(hype_solver *s, const Bands &b, int k, const PlanStage &q, int out_aos = 0, double *out = nullptr,
                              cudaStream_t on = nullptr)
{
    const int saved = s->runs;
    cudaStream_t saved_stream = s->stream;
    s->runs = b.runs;
    if (on) s->stream = on;
    const int r0 = b.run[k], nr = b.run[k + 1] - b.run[k];
    const cudaError_t e = s->mixed ? stage_m(s, q.in, out ? -1 : q.out, q.mode, q.ka, q.kb, q.kc, q.x, q.reduce, out, false, r0, nr)
                                   : stage(s, buf_of(s, q.in), out ? out : buf_of(s, q.out), q.mode, q.ka, q.kb, q.kc, buf_of(s, q.x),
                                           buf_of(s, q.out2), q.reduce, out_aos, r0, nr);
    s->runs = saved;
    s->stream = saved_stream;
    return e;
}

// First stage of a banded call: uploads of bands 0..n-1 in order (`upload(k)`,
// which records ev_in[k]), each band launched as soon as the uploads it reads
// are enqueued (and waited for); `after` runs behind every band launch (e.g. its
// download).
template <typename Upload, typename After>
static int banded_upload_stage(hype_solver *s, const Bands &b, Upload upload, const PlanStage &q, int out_aos, double *out,
                               After after)
{
    int rc, next = 0;
    for (int u = 0; u < b.n; ++u) {
        if ((rc = upload(u))) return rc;
        while (next < b.n && band_needs(s, b, b.order[next]) <= u) {
            const int k = b.order[next++];
            CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->ev_in[band_needs(s, b, k)], 0));
            CUDA_TRY(s, stage_band(s, b, k, q, out_aos, out));
            if ((rc = after(k))) return rc;
        }
    }
    return HYPE_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void hype_config_default(hype_config *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->system = HYPE_KAPILA_5EQN;       // hype.h:35
    c->order = 1;                       // hype.c:32
    c->nx = 128; c->ny = 128;           // hype.c:37-38
    c->x_min = 0.0; c->x_max = 12.0;    // hype.c:33-36
    c->y_min = 0.0; c->y_max = 12.0;
    c->cfl = 0.9;                       // hype.c:39
    c->bc_left = HYPE_BC_TRANSMISSIVE; c->bc_right = HYPE_BC_TRANSMISSIVE;   // hype.c:46-49
    c->bc_bottom = HYPE_BC_REFLECTIVE; c->bc_top = HYPE_BC_REFLECTIVE;
    c->gamma1 = 4.4; c->gamma2 = 1.4; c->pi1 = 6000.0; c->pi2 = 0.0;         // hype.h:42-45
    c->precision = HYPE_PREC_FP64;
    c->flags = 0;
    c->device = 0;
    c->mu1 = 1.0e-2; c->mu2 = 0.0;      // hype.h:46-47
}

int hype_nvar(int system)
{
    switch (system) {
    case HYPE_EULER: return 4;
    case HYPE_KAPILA_5EQN: return 6;
    case HYPE_BAER_NUNZIATO: return 9;
    default: return 0;
    }
}

const char *hype_status_string(int st)
{
    switch (st) {
    case HYPE_OK: return "ok";
    case HYPE_ERR_INVALID: return "invalid argument or configuration";
    case HYPE_ERR_CUDA: return "CUDA error";
    case HYPE_ERR_INADMISSIBLE: return "inadmissible face state (the reference aborts here)";
    case HYPE_ERR_TIMEOUT: return "device wait timed out";
    case HYPE_ERR_NOMEM: return "out of device memory";
    case HYPE_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case HYPE_ERR_BUSY: return "solver busy";
    default: return "unknown status";
    }
}

const char *hype_last_error(const hype_solver *s) { return s ? s->err : "null solver"; }

int hype_destroy(hype_solver *s)
{
    if (!s) return HYPE_OK;
    int dev = s->cfg.device;
    cudaSetDevice(dev);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->step_exec) cudaGraphExecDestroy(s->step_exec);
    double *bufs[] = {solver_alloc_base(s, s->dU), solver_alloc_base(s, s->dS0), solver_alloc_base(s, s->dS1),
                      solver_alloc_base(s, s->dS2), s->dAosIn, s->dAosOut, s->dInlet, s->dRed};
    for (double *b : bufs) if (b) cudaFree(b);
    const long long moff = (long long)s->row_off * s->pitch;
    for (int k = 0; k < 3; ++k) { if (s->mf[k]) cudaFree(s->mf[k] - moff); if (s->md[k]) cudaFree(s->md[k] - moff); }
    if (s->dSc) cudaFree(s->dSc);
    if (s->hSc) cudaFreeHost(s->hSc);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    for (int k = 0; k < hype_solver::MAX_BANDS; ++k) {
        if (s->ev_cp[k]) cudaEventDestroy(s->ev_cp[k]);
        if (s->ev_in[k]) cudaEventDestroy(s->ev_in[k]);
        if (s->ev_dc[k]) cudaEventDestroy(s->ev_dc[k]);
        if (s->ev_done[k]) cudaEventDestroy(s->ev_done[k]);
        if (s->ev_dl[k]) cudaEventDestroy(s->ev_dl[k]);
    }
    if (s->hStageIn) cudaFreeHost(s->hStageIn);
    if (s->hStageOut) cudaFreeHost(s->hStageOut);
    if (s->ev_fence) cudaEventDestroy(s->ev_fence);
    for (cudaEvent_t e : s->ev_sb) if (e) cudaEventDestroy(e);
    for (cudaStream_t *q : {&s->stream2, &s->stream3, &s->stream4, &s->cin, &s->cout, &s->cvin, &s->cvout})
        if (*q) { cudaStreamSynchronize(*q); cudaStreamDestroy(*q); }
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return HYPE_OK;
}

}  // extern "C"

// Device buffers, streams and descriptors of a checked configuration.  row_off > 0
// makes a y-slab: every plane carries row_off halo rows below and above the slab's
// rows; col_off > 0 (a block of a grid split in x, FP64 only) adds col_off halo
// columns left and right of its columns; `inlet` replaces the inlet table computed
// from cfg (a slab's rows of the whole grid's table).
static int create_common(hype_solver *s, const hype_config *cfg, int row_off, const std::vector<double> *inlet, int col_off = 0)
{
    s->cfg = *cfg;
    s->row_off = row_off;
    s->col_off = col_off;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0)
        return fail(s, HYPE_ERR_NO_DEVICE, "CUDA device %d not available", cfg->device);
    CUDA_TRY(s, cudaSetDevice(cfg->device));
    cudaDeviceProp prop;
    CUDA_TRY(s, cudaGetDeviceProperties(&prop, cfg->device));
    if (prop.major != 10) return fail(s, HYPE_ERR_NO_DEVICE, "device %d is sm_%d%d; the library is built for sm_100a", cfg->device, prop.major, prop.minor);
    s->mixed = cfg->precision == HYPE_PREC_MIXED;
    s->fast = cfg->precision == HYPE_PREC_FP64_FAST;

    s->nv = hype_nvar(cfg->system);
    if (s->mixed && col_off) return fail(s, HYPE_ERR_INVALID, "a block of a grid split in x takes an FP64 precision");
    s->pitch = s->mixed ? ((cfg->nx + 31) & ~31) : ((cfg->nx + 2 * col_off + 15) & ~15);   // 128-byte rows
    s->plane = (long long)s->pitch * (cfg->ny + 2 * row_off);
    s->h = (cfg->x_max - cfg->x_min) / (double)cfg->nx;   // hype.c:57
    s->r1_h = 1. / s->h;                                  // rhs_function_prim.c:26
    s->cfl_h = cfg->cfl * s->h;                           // rhs_function_prim.c:620
    const size_t state_bytes = sizeof(double) * (size_t)s->plane * s->nv;
    const size_t aos_bytes = sizeof(double) * (size_t)(cfg->nx + 2 * col_off) * (cfg->ny + 2 * row_off) * s->nv;
    CUDA_TRY(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    CUDA_TRY(s, cudaEventCreate(&s->ev0));
    CUDA_TRY(s, cudaEventCreate(&s->ev1));
    for (cudaStream_t *q : {&s->cin, &s->cout, &s->cvin, &s->cvout, &s->stream2, &s->stream3, &s->stream4})
        CUDA_TRY(s, cudaStreamCreateWithFlags(q, cudaStreamNonBlocking));
    for (int k = 0; k < hype_solver::MAX_BANDS; ++k)
        for (cudaEvent_t *e : {&s->ev_cp[k], &s->ev_in[k], &s->ev_dc[k], &s->ev_done[k], &s->ev_dl[k]})
            CUDA_TRY(s, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    CUDA_TRY(s, cudaEventCreateWithFlags(&s->ev_fence, cudaEventDisableTiming));
    for (cudaEvent_t &e : s->ev_sb) CUDA_TRY(s, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    double **bufs[] = {&s->dU, &s->dS0, &s->dS1, &s->dS2};
    const long long off = (long long)row_off * s->pitch + col_off;   // the buffers point at cell (0, 0)
    for (double **b : bufs) {
        if (b == &s->dS2 && cfg->order != 3) continue;
        if (cudaMalloc(b, state_bytes) != cudaSuccess) return fail(s, HYPE_ERR_NOMEM, "cudaMalloc(%zu) failed", state_bytes);
        CUDA_TRY(s, cudaMemset(*b, 0, state_bytes));
        *b += off;
    }
    if (s->mixed) {
        const MixedLayout L = mixed_layout(cfg->system);
        for (int k = 0; k < 3; ++k) {
            if (cudaMalloc(&s->mf[k], sizeof(float) * L.nf * (size_t)s->plane) != cudaSuccess ||
                cudaMalloc(&s->md[k], sizeof(double) * L.nd * (size_t)s->plane) != cudaSuccess)
                return fail(s, HYPE_ERR_NOMEM, "cudaMalloc of the mixed state failed");
            CUDA_TRY(s, cudaMemset(s->mf[k], 0, sizeof(float) * L.nf * (size_t)s->plane));
            CUDA_TRY(s, cudaMemset(s->md[k], 0, sizeof(double) * L.nd * (size_t)s->plane));
            s->mf[k] += off;   // row 0 of the slab
            s->md[k] += off;
        }
    }
    if (cudaMalloc(&s->dAosIn, aos_bytes) != cudaSuccess || cudaMalloc(&s->dAosOut, aos_bytes) != cudaSuccess)
        return fail(s, HYPE_ERR_NOMEM, "cudaMalloc(%zu) failed", aos_bytes);
    s->aos_bytes = aos_bytes;
    CUDA_TRY(s, cudaMalloc(&s->dRed, sizeof(double) * TOTALS_SCRATCH));
    CUDA_TRY(s, cudaMalloc(&s->dSc, sizeof(DevScalars)));
    CUDA_TRY(s, cudaMemset(s->dSc, 0, sizeof(DevScalars)));
    CUDA_TRY(s, cudaMallocHost(&s->hSc, sizeof(DevScalars)));
    if (cfg->bc_left == HYPE_BC_INLET) {
        std::vector<double> tab;
        if (inlet) tab = *inlet;
        else inlet_table(*cfg, s->h, tab);
        if (cfg->flags & HYPE_FLAG_CONSERVATIVE) inlet_to_conserved(*cfg, tab);
        CUDA_TRY(s, cudaMalloc(&s->dInlet, sizeof(double) * tab.size()));
        CUDA_TRY(s, cudaMemcpy(s->dInlet, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
    }

    s->sms = prop.multiProcessorCount;
    return set_tiling(s, s->mixed ? MIXED_CELLS : STAGE_CELLS);
}

int hype::create_block(const hype_config *global, int col0, int cols, int row0, int rows, const bool halo[4], hype_solver **out)
{
    if (!out) return HYPE_ERR_INVALID;
    *out = nullptr;
    hype_solver *s = new (std::nothrow) hype_solver();
    if (!s) return HYPE_ERR_NOMEM;
    *out = s;
    int rc = check_config(global, s);
    if (rc) return rc;
    if (rows < 3 || row0 < 0 || row0 + rows > global->ny) return fail(s, HYPE_ERR_INVALID, "bad slab rows %d..%d", row0, row0 + rows - 1);
    if (cols < 3 || col0 < 0 || col0 + cols > global->nx)
        return fail(s, HYPE_ERR_INVALID, "bad block columns %d..%d", col0, col0 + cols - 1);
    const bool xsplit = cols != global->nx;
    hype_config c = *global;
    const double h = (global->x_max - global->x_min) / (double)global->nx;   // hype.c:57, the whole grid's spacing
    c.nx = cols;
    c.ny = rows;
    const double hy = (global->y_max - global->y_min) / (double)global->ny;   // the block's extent (informative)
    c.y_min = global->y_min + (double)row0 * hy;
    c.y_max = global->y_min + (double)(row0 + rows) * hy;
    if (xsplit) {
        c.x_min = global->x_min + (double)col0 * h;
        c.x_max = global->x_min + (double)(col0 + cols) * h;
    }
    if (halo[0]) c.bc_left = BC_HALO;
    if (halo[1]) c.bc_right = BC_HALO;
    if (halo[2]) c.bc_bottom = BC_HALO;
    if (halo[3]) c.bc_top = BC_HALO;
    s->row0 = row0;
    s->col0 = col0;
    const int col_off = xsplit ? 4 : 0;   // 3 halo columns, 4 to keep TMA x origins 16-byte aligned
    if (c.bc_left != HYPE_BC_INLET) {
        rc = create_common(s, &c, 3, nullptr, col_off);
    } else {
        // the slab's ghost-extended rows -3 .. rows+2 are rows row0-3 .. row0+rows+2 of the whole table
        std::vector<double> whole, tab;
        const int nv = hype_nvar(global->system);
        inlet_table(*global, h, whole);
        tab.assign((size_t)3 * (rows + 6) * nv, 0.0);
        for (int g = 0; g < 3; ++g)
            std::memcpy(&tab[(size_t)g * (rows + 6) * nv], &whole[((size_t)g * (global->ny + 6) + row0) * nv],
                        sizeof(double) * (rows + 6) * nv);
        rc = create_common(s, &c, 3, &tab, col_off);
    }
    if (rc == HYPE_OK && xsplit) {   // the whole grid's h, not the block extent's rounding of it
        s->h = h;
        s->r1_h = 1. / s->h;                                  // rhs_function_prim.c:26
        s->cfl_h = global->cfl * s->h;                        // rhs_function_prim.c:620
    }
    return rc;
}

int hype::create_slab(const hype_config *global, int row0, int rows, bool halo_lo, bool halo_hi, hype_solver **out)
{
    const bool halo[4] = {false, false, halo_lo, halo_hi};
    return create_block(global, 0, global ? global->nx : 0, row0, rows, halo, out);
}

extern "C" {

int hype_create(const hype_config *cfg, hype_solver **out)
{
    if (!out) return HYPE_ERR_INVALID;
    *out = nullptr;
    hype_solver *s = new (std::nothrow) hype_solver();
    if (!s) return HYPE_ERR_NOMEM;
    *out = s;
    const int rc = check_config(cfg, s);
    if (rc) return rc;   // caller reads hype_last_error, then destroys
    return create_common(s, cfg, 0, nullptr);
}

// dt of the last RHS: CFL h / (2 s_max) (rhs_function_prim.c:620), or
// CFL h / (2 (s_max + (s_max_v / h) 2)) for a viscous solver (:617); the two
// agree bit for bit when s_max_v and r1h_v are 0
static double host_dt(const hype_solver *s)
{
    double smax, smaxv;
    const unsigned long long b0 = s->hSc->smax, b1 = s->hSc->smax_v;
    std::memcpy(&smax, &b0, sizeof(smax));
    std::memcpy(&smaxv, &b1, sizeof(smaxv));
    if (!(s->cfg.flags & HYPE_FLAG_VISCOUS)) return (s->cfg.cfl * s->h) / (2.0 * smax);
    return (s->cfg.cfl * s->h) / (2.0 * (smax + (s->r1_h * smaxv) * 2.0));
}

static int read_scalars(hype_solver *s)
{
    CUDA_TRY(s, cudaMemcpyAsync(s->hSc, s->dSc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if (s->hSc->err & ERR_TMA_TIMEOUT) return fail(s, HYPE_ERR_TIMEOUT, "TMA row load did not complete");
    if (s->hSc->err & ERR_BAD_LAUNCH) return fail(s, HYPE_ERR_CUDA, "stage kernel launched with a geometry it does not cover");
    if (s->hSc->err & ERR_INADMISSIBLE_FACE) {
        const unsigned cell = s->hSc->err_cell;
        return fail(s, HYPE_ERR_INADMISSIBLE, "inadmissible face state near cell (i=%u, j=%u)",
                    cell % (unsigned)s->cfg.nx + (unsigned)s->col0, cell / (unsigned)s->cfg.nx + (unsigned)s->row0);
    }
    return HYPE_OK;
}

static int reset_scalars(hype_solver *s)
{
    std::memset(s->hSc, 0, sizeof(DevScalars));
    s->hSc->err_cell = 0xffffffffu;
    s->hSc->r1h_v = (s->cfg.flags & HYPE_FLAG_VISCOUS) ? s->r1_h : 0.0;
    CUDA_TRY(s, cudaMemcpyAsync(s->dSc, s->hSc, sizeof(DevScalars), cudaMemcpyHostToDevice, s->stream));
    return HYPE_OK;
}

// interleaved FP64 state (device) -> state k (0 = U, 1 = S0) in the solver's layout
static cudaError_t load_state(hype_solver *s, const double *aos, int k)
{
    if (s->mixed) return launch_aos_to_mixed(s->cfg.system, aos, s->mf[k], s->md[k], s->cfg.nx, s->cfg.ny, s->pitch, s->plane, s->stream);
    return launch_aos_to_planes(aos, k == 0 ? s->dU : s->dS0, s->cfg.nx, s->cfg.ny, s->nv, s->pitch, s->plane, s->stream);
}
static cudaError_t store_state(hype_solver *s, int k, double *aos)
{
    if (s->mixed) return launch_mixed_to_aos(s->cfg.system, s->mf[k], s->md[k], aos, s->cfg.nx, s->cfg.ny, s->pitch, s->plane, s->stream);
    return launch_planes_to_aos(k == 0 ? s->dU : s->dS0, aos, s->cfg.nx, s->cfg.ny, s->nv, s->pitch, s->plane, s->stream);
}

// RHS of state S0 into an interleaved device array
static int rhs_common(hype_solver *s, double *dRHS_aos, double *dt)
{
    int rc;
    if ((rc = reset_scalars(s))) return rc;
    if (s->mixed) CUDA_TRY(s, stage_m(s, 1, -1, OUT_RHS, 0, 1.0, 0, -1, 1, dRHS_aos));
    else CUDA_TRY(s, stage(s, s->dS0, dRHS_aos, OUT_RHS, 0, 1.0, 0, nullptr, nullptr, 1, 1));
    if ((rc = read_scalars(s))) return rc;
    if (dt) {
        *dt = host_dt(s);
    }
    return HYPE_OK;
}

int hype_rhs_prim(hype_solver *s, double t, const double *U, double *RHS, double *dt)
{
    (void)t;
    if (!s || !U || !RHS) return fail(s, HYPE_ERR_INVALID, "null argument");
    if (s->row_off) return fail(s, HYPE_ERR_INVALID, "a slab solver takes hype_rhs_prim_slab");
    if (!s->dSc) return fail(s, HYPE_ERR_INVALID, "solver not created");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    int rc;
    // banded: U's rows stream in while earlier bands compute, RHS rows stream out
    const Bands b = host_bands(s);
    const size_t row_elems = (size_t)s->cfg.nx * s->nv;
    if ((rc = fence_copy_streams(s)) || (rc = reset_scalars(s))) return rc;
    const PlanStage q{B_S0, B_NONE, OUT_RHS, 0.0, 1.0, 0.0, B_NONE, B_NONE, 1};
    HostIO io = host_io(s, U, RHS);
    rc = banded_upload_stage(s, b, [&](int k) { return upload_band(s, b, k, U, B_S0, io); }, q, 1, s->dAosOut, [&](int k) -> int {
        // band k's RHS rows are final: copy them out while later bands compute
        const int r0 = b.row[k], nr = b.row[k + 1] - r0;
        CUDA_TRY(s, cudaEventRecord(s->ev_done[k], s->stream));
        CUDA_TRY(s, cudaStreamWaitEvent(s->cout, s->ev_done[k], 0));
        return download_rows(s, io, k, RHS, r0 * row_elems, row_elems * nr);
    });
    if (rc) return rc;
    if ((rc = finish_downloads(s, io, RHS))) return rc;
    if ((rc = read_scalars(s)) && rc != HYPE_ERR_INADMISSIBLE) return rc;
    if (dt) {
        *dt = host_dt(s);
    }
    return rc;
}

int hype_create_slab(const hype_config *cfg, int row0, int rows, hype_solver **out)
{
    if (!cfg) return HYPE_ERR_INVALID;
    const bool whole = row0 == 0 && rows == cfg->ny;
    const bool periodic = cfg->bc_bottom == HYPE_BC_PERIODIC;
    return create_slab(cfg, row0, rows, !whole && (row0 > 0 || periodic), !whole && (row0 + rows < cfg->ny || periodic), out);
}

int hype_create_block(const hype_config *cfg, int col0, int cols, int row0, int rows, hype_solver **out)
{
    if (!cfg) return HYPE_ERR_INVALID;
    const bool px = cfg->bc_left == HYPE_BC_PERIODIC, py = cfg->bc_bottom == HYPE_BC_PERIODIC;
    const bool wx = col0 == 0 && cols == cfg->nx, wy = row0 == 0 && rows == cfg->ny;
    const bool halo[4] = {!wx && (col0 > 0 || px), !wx && (col0 + cols < cfg->nx || px),
                          !wy && (row0 > 0 || py), !wy && (row0 + rows < cfg->ny || py)};
    return create_block(cfg, col0, cols, row0, rows, halo, out);
}

int hype_rhs_prim_slab(hype_solver *s, double t, const double *U, long long row_stride, double *RHS, double *dt)
{
    (void)t;
    if (!s || !U || !RHS) return fail(s, HYPE_ERR_INVALID, "null argument");
    if (!s->dSc || s->row_off == 0) return fail(s, HYPE_ERR_INVALID, "not a slab or block solver (hype_create_slab, hype_create_block)");
    const int nx = s->cfg.nx;
    const int lo = s->cfg.bc_bottom == BC_HALO ? 3 : 0, hi = s->cfg.bc_top == BC_HALO ? 3 : 0;
    const int cl = s->cfg.bc_left == BC_HALO ? 3 : 0, cr = s->cfg.bc_right == BC_HALO ? 3 : 0;
    const int width = cl + nx + cr;   // cells per staged row
    if (row_stride < (long long)width * s->nv) return fail(s, HYPE_ERR_INVALID, "row_stride below the staged row width * nvar");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    const size_t srow = (size_t)width * s->nv;   // elements per staged row; staging row j + 3 holds local row j
    int rc;
    // banded as hype_rhs_prim: band k's rows (with the ghost rows below band 0 and above
    // the last band) are copied from the local array and converted, its RHS launch runs
    // once the rows its stencils read are there, and its RHS rows go to the host while
    // later bands compute
    const Bands b = host_bands(s);
    if ((rc = fence_copy_streams(s)) || (rc = reset_scalars(s))) return rc;
    HostIO io = host_io(s, U, RHS);
    auto upload = [&](int k) -> int {
        const int a = b.row[k] - (k == 0 ? lo : 0), e = b.row[k + 1] + (k == b.n - 1 ? hi : 0);   // local rows a .. e-1
        double *stg = s->dAosIn + (size_t)(a + 3) * srow;
        const double *from = U + (long long)a * row_stride - (long long)cl * s->nv;
        if (io.stage_in) {   // the rows compacted into pinned staging, then one contiguous copy
            double *h = s->hStageIn + (size_t)(a + 3) * srow;
            host_copy_2d(h, sizeof(double) * srow, from, sizeof(double) * (size_t)row_stride, sizeof(double) * srow, (size_t)(e - a));
            CUDA_TRY(s, cudaMemcpyAsync(stg, h, sizeof(double) * srow * (e - a), cudaMemcpyHostToDevice, s->cin));
        } else {
            CUDA_TRY(s, cudaMemcpy2DAsync(stg, sizeof(double) * srow, from, sizeof(double) * (size_t)row_stride, sizeof(double) * srow,
                                          (size_t)(e - a), cudaMemcpyHostToDevice, s->cin));
        }
        CUDA_TRY(s, cudaEventRecord(s->ev_cp[k], s->cin));
        CUDA_TRY(s, cudaStreamWaitEvent(s->cvin, s->ev_cp[k], 0));
        if (s->mixed) {   // FP32 and FP64 planes of S0 (a mixed solver is never split in x)
            const long long o = (long long)a * s->pitch;
            CUDA_TRY(s, launch_aos_to_mixed(s->cfg.system, stg, s->mf[1] + o, s->md[1] + o, nx, e - a, s->pitch, s->plane, s->cvin));
        } else {          // planes of S0 from local row -3, column -cl on
            CUDA_TRY(s, launch_aos_to_planes_rows(s->dAosIn, s->dS0 - 3LL * s->pitch - cl, width, a + 3, e - a, s->nv, s->pitch,
                                                  s->plane, s->cvin));
        }
        CUDA_TRY(s, cudaEventRecord(s->ev_in[k], s->cvin));
        return HYPE_OK;
    };
    const PlanStage q{B_S0, B_NONE, OUT_RHS, 0.0, 1.0, 0.0, B_NONE, B_NONE, 1};
    const size_t row_elems = (size_t)nx * s->nv;
    rc = banded_upload_stage(s, b, upload, q, 1, s->dAosOut, [&](int k) -> int {
        const int r0 = b.row[k], nr = b.row[k + 1] - r0;
        CUDA_TRY(s, cudaEventRecord(s->ev_done[k], s->stream));
        CUDA_TRY(s, cudaStreamWaitEvent(s->cout, s->ev_done[k], 0));
        return download_rows(s, io, k, RHS, r0 * row_elems, row_elems * nr);
    });
    if (rc) return rc;
    if ((rc = finish_downloads(s, io, RHS))) return rc;
    if ((rc = read_scalars(s)) && rc != HYPE_ERR_INADMISSIBLE) return rc;
    if (dt) *dt = host_dt(s);
    return rc;
}

int hype_rhs_prim_device(hype_solver *s, double t, const double *dU, double *dRHS, double *dt)
{
    (void)t;
    if (!s || !dU || !dRHS) return fail(s, HYPE_ERR_INVALID, "null argument");
    if (s->row_off) return fail(s, HYPE_ERR_INVALID, "a slab solver takes hype_rhs_prim_slab");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    CUDA_TRY(s, load_state(s, dU, 1));
    return rhs_common(s, dRHS, dt);
}

// A whole cell-major array from the caller into dAosIn, or from dAosOut to the caller,
// on the solver's stream.  Pageable arrays go through the pinned staging in up to
// MAX_BANDS chunks, so that the host copy of one chunk overlaps the DMA of another.
static size_t whole_chunk(size_t bytes)
{
    const size_t c = (bytes + hype_solver::MAX_BANDS - 1) / hype_solver::MAX_BANDS;
    return c < ((size_t)1 << 20) ? ((size_t)1 << 20) : c;
}

static int copy_in_whole(hype_solver *s, const double *U, size_t bytes)
{
    const HostIO io = host_io(s, U, nullptr);
    if (!io.stage_in) {
        CUDA_TRY(s, cudaMemcpyAsync(s->dAosIn, U, bytes, cudaMemcpyHostToDevice, s->stream));
        return HYPE_OK;
    }
    const size_t chunk = whole_chunk(bytes);
    for (size_t off = 0; off < bytes; off += chunk) {
        const size_t n = bytes - off < chunk ? bytes - off : chunk;
        host_copy((char *)s->hStageIn + off, (const char *)U + off, n);
        CUDA_TRY(s, cudaMemcpyAsync((char *)s->dAosIn + off, (char *)s->hStageIn + off, n, cudaMemcpyHostToDevice, s->stream));
    }
    return HYPE_OK;
}

static int copy_out_whole(hype_solver *s, double *U, size_t bytes)
{
    const HostIO io = host_io(s, nullptr, U);
    if (!io.stage_out) {
        CUDA_TRY(s, cudaMemcpyAsync(U, s->dAosOut, bytes, cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(s, cudaStreamSynchronize(s->stream));
        return HYPE_OK;
    }
    const size_t chunk = whole_chunk(bytes);
    int k = 0;
    for (size_t off = 0; off < bytes; off += chunk, ++k) {
        const size_t n = bytes - off < chunk ? bytes - off : chunk;
        CUDA_TRY(s, cudaMemcpyAsync((char *)s->hStageOut + off, (char *)s->dAosOut + off, n, cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(s, cudaEventRecord(s->ev_dl[k], s->stream));
    }
    k = 0;
    for (size_t off = 0; off < bytes; off += chunk, ++k) {
        const size_t n = bytes - off < chunk ? bytes - off : chunk;
        CUDA_TRY(s, cudaEventSynchronize(s->ev_dl[k]));
        host_copy((char *)U + off, (const char *)s->hStageOut + off, n);
    }
    return HYPE_OK;
}

int hype_set_state(hype_solver *s, const double *U)
{
    if (!s || !U) return fail(s, HYPE_ERR_INVALID, "null argument");
    if (s->row_off) return fail(s, HYPE_ERR_INVALID, "a slab solver has no time loop of its own (hype_group runs slabs)");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    const size_t aos_bytes = sizeof(double) * (size_t)s->cfg.nx * s->cfg.ny * s->nv;
    int rc;
    if ((rc = copy_in_whole(s, U, aos_bytes))) return rc;
    CUDA_TRY(s, load_state(s, s->dAosIn, 0));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return HYPE_OK;
}

int hype_get_state(hype_solver *s, double *U)
{
    if (!s || !U) return fail(s, HYPE_ERR_INVALID, "null argument");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    const size_t aos_bytes = sizeof(double) * (size_t)s->cfg.nx * s->cfg.ny * s->nv;
    CUDA_TRY(s, store_state(s, 0, s->dAosOut));
    return copy_out_whole(s, U, aos_bytes);
}

// One SSP-RK step (begin_step, the stages, end_step) captured once as a CUDA
// graph and replayed by hype_advance.
static int ensure_step_graph(hype_solver *s)
{
    if (s->step_exec) return HYPE_OK;
    cudaGraph_t g;
    CUDA_TRY(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_step(s);
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess) return fail(s, HYPE_ERR_CUDA, "step capture: %s", cudaGetErrorString(e));
    if (e2 != cudaSuccess) return fail(s, HYPE_ERR_CUDA, "step capture end: %s", cudaGetErrorString(e2));
    e = cudaGraphInstantiate(&s->step_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(s, HYPE_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return HYPE_OK;
}

int hype_begin(hype_solver *s, double t0, double t_final, int max_steps)
{
    if (!s) return HYPE_ERR_INVALID;
    if (s->row_off) return fail(s, HYPE_ERR_INVALID, "a slab solver has no time loop of its own (hype_group runs slabs)");
    if (max_steps < 0) return fail(s, HYPE_ERR_INVALID, "max_steps < 0");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    int rc;
    if ((rc = reset_scalars(s))) return rc;
    s->hSc->t = t0; s->hSc->t_final = t_final; s->hSc->max_steps = max_steps;
    CUDA_TRY(s, cudaMemcpyAsync(s->dSc, s->hSc, sizeof(DevScalars), cudaMemcpyHostToDevice, s->stream));
    // hype.c:343: one RHS evaluation of the initial state seeds Ctx.dt
    if (s->mixed) CUDA_TRY(s, stage_m(s, 0, -1, OUT_RHS, 0, 1.0, 0, -1, 1, s->dAosOut));
    else CUDA_TRY(s, stage(s, s->dU, s->dS1, OUT_RHS, 0, 1.0, 0, nullptr, nullptr, 1));
    CUDA_TRY(s, launch_seed_dt(s->dSc, s->cfl_h, s->stream));
    if ((rc = ensure_step_graph(s))) return rc;
    s->began = true;
    return HYPE_OK;
}

int hype_advance(hype_solver *s, int nsteps)
{
    if (!s) return HYPE_ERR_INVALID;
    if (!s->began) return fail(s, HYPE_ERR_INVALID, "hype_begin not called");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    int rc;
    if ((rc = ensure_step_graph(s))) return rc;
    CUDA_TRY(s, cudaEventRecord(s->ev0, s->stream));
    for (int k = 0; k < nsteps; ++k) CUDA_TRY(s, cudaGraphLaunch(s->step_exec, s->stream));
    CUDA_TRY(s, cudaEventRecord(s->ev1, s->stream));
    return HYPE_OK;
}

// One step enqueued by hand (the graph's content) as a wavefront of row bands:
// band k of stage s reads the rows of bands k-1..k+1 of stage s-1 (3-row stencils,
// bands of >= 8 rows; bands 0 and n-1 are neighbours on a periodic y axis) and
// waits for their events, stage 0 for the uploads of those bands (U_in).  Stage s
// writes a buffer that only stage s-1 (or, for the combination's second operand,
// the same band of an earlier stage) still reads, so the same dependency covers
// every overwrite.  Stage s is enqueued band by band on compute stream s % 4, in
// b.order (band 0 last on a periodic y axis, where it reads the last band), so no
// band waits behind another that is not ready.  After each band's upload every
// launch whose inputs are enqueued is enqueued too, so the device starts while
// the host still stages later bands; the last stage's bands are converted and
// copied out as they finish (U_out).  Results equal the unbanded step's.
static int enqueue_step_banded(hype_solver *s, const Bands &b, const double *U_in, double *U_out, HostIO &io)
{
    PlanStage plan[MAX_PLAN];
    int copy_back = 0, rc;
    const int ns = ssp_plan(s->cfg.order, plan, &copy_back);
    const size_t row_elems = (size_t)s->cfg.nx * s->nv;
    const bool py = s->cfg.bc_bottom == HYPE_BC_PERIODIC && b.n > 1;
    cudaStream_t on_stage[4] = {s->stream, s->stream2, s->stream3, s->stream4};
    bool done[MAX_PLAN][hype_solver::MAX_BANDS] = {};
    int next[MAX_PLAN] = {};   // per stage: the position in b.order of its next band
    int uploaded = U_in ? 0 : b.n;
    auto nbrs = [&](int k, int *nb) -> int {   // bands whose rows band k's stencils read
        int m = 0;
        nb[m++] = k;
        if (k > 0) nb[m++] = k - 1; else if (py) nb[m++] = b.n - 1;
        if (k + 1 < b.n) nb[m++] = k + 1; else if (py) nb[m++] = 0;
        return m;
    };
    auto ready = [&](int st, int k) -> bool {
        int nb[3];
        const int m = nbrs(k, nb);
        for (int j = 0; j < m; ++j)
            if (st == 0 ? nb[j] >= uploaded : !done[st - 1][nb[j]]) return false;
        return true;
    };
    auto launch = [&](int st, int k) -> int {
        const PlanStage &q = plan[st];
        cudaStream_t on = on_stage[st % 4];
        int nb[3];
        const int m = nbrs(k, nb);
        for (int j = 0; j < m; ++j) {
            if (st == 0 && U_in) CUDA_TRY(s, cudaStreamWaitEvent(on, s->ev_in[nb[j]], 0));
            if (st > 0) CUDA_TRY(s, cudaStreamWaitEvent(on, s->ev_sb[(st - 1) * hype_solver::MAX_BANDS + nb[j]], 0));
        }
        CUDA_TRY(s, stage_band(s, b, k, q, 0, nullptr, on));
        cudaEvent_t ev = s->ev_sb[st * hype_solver::MAX_BANDS + k];
        CUDA_TRY(s, cudaEventRecord(ev, on));
        done[st][k] = true;
        if (st == ns - 1 && U_out) {   // band k of the result: to the host while later bands compute
            const int r0 = b.row[k], nr = b.row[k + 1] - r0;
            CUDA_TRY(s, cudaStreamWaitEvent(s->cvout, ev, 0));
            CUDA_TRY(s, state_to_rows(s, q.out, r0, nr, s->cvout));
            CUDA_TRY(s, cudaEventRecord(s->ev_dc[k], s->cvout));
            CUDA_TRY(s, cudaStreamWaitEvent(s->cout, s->ev_dc[k], 0));
            return download_rows(s, io, k, U_out, r0 * row_elems, row_elems * nr);
        }
        return HYPE_OK;
    };
    CUDA_TRY(s, launch_begin_step(s->dSc, s->stream));
    CUDA_TRY(s, cudaEventRecord(s->ev_fence, s->stream));   // the other compute streams start behind begin_step
    for (int j = 1; j < 4; ++j) CUDA_TRY(s, cudaStreamWaitEvent(on_stage[j], s->ev_fence, 0));
    for (int u = 0;; ++u) {
        if (u < b.n && U_in) {
            if ((rc = upload_band(s, b, u, U_in, plan[0].in, io))) return rc;
            uploaded = u + 1;
        }
        for (int st = 0; st < ns; ++st)
            while (next[st] < b.n && ready(st, b.order[next[st]])) {
                if ((rc = launch(st, b.order[next[st]]))) return rc;
                ++next[st];
            }
        if (uploaded >= b.n) break;
    }
    for (int st = 0; st < ns; ++st)
        if (next[st] < b.n) return fail(s, HYPE_ERR_CUDA, "banded step: stage %d band %d never became ready", st, b.order[next[st]]);
    for (int k = 0; k < b.n; ++k)   // end_step and everything after it behind every compute stream
        for (int st = ns - 4 > 0 ? ns - 4 : 0; st < ns; ++st)
            CUDA_TRY(s, cudaStreamWaitEvent(s->stream, s->ev_sb[st * hype_solver::MAX_BANDS + k], 0));
    CUDA_TRY(s, launch_end_step(s->dSc, s->cfl_h, s->stream));
    return HYPE_OK;
}

int hype_advance_host(hype_solver *s, const double *U_in, double *U_out, int nsteps, int *steps_done, double *t_end,
                      double *dt_next)
{
    if (!s || !U_in || !U_out || nsteps < 1) return fail(s, HYPE_ERR_INVALID, "bad argument");
    if (!s->began) return fail(s, HYPE_ERR_INVALID, "hype_begin not called");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    int rc;
    const bool banded = s->cfg.order != 0;   // forward Euler's last write is a copy, not a stage
    if (!banded) {
        if ((rc = hype_set_state(s, U_in)) || (rc = hype_advance(s, nsteps))) return rc;
        rc = hype_wait(s, steps_done, t_end, dt_next);
        if (rc && rc != HYPE_ERR_INADMISSIBLE) return rc;
        const int rc2 = hype_get_state(s, U_out);
        return rc ? rc : rc2;
    }
    if ((rc = ensure_step_graph(s))) return rc;
    const Bands b = host_bands(s);
    if ((rc = fence_copy_streams(s))) return rc;
    HostIO io = host_io(s, U_in, U_out);
    CUDA_TRY(s, cudaEventRecord(s->ev0, s->stream));
    if ((rc = enqueue_step_banded(s, b, U_in, nsteps == 1 ? U_out : nullptr, io))) return rc;
    for (int k = 1; k + 1 < nsteps; ++k) CUDA_TRY(s, cudaGraphLaunch(s->step_exec, s->stream));
    if (nsteps > 1 && (rc = enqueue_step_banded(s, b, nullptr, U_out, io))) return rc;
    CUDA_TRY(s, cudaEventRecord(s->ev1, s->stream));
    if ((rc = finish_downloads(s, io, U_out))) return rc;
    return hype_wait(s, steps_done, t_end, dt_next);
}

int hype_wait(hype_solver *s, int *steps_done, double *t_end, double *dt_next)
{
    if (!s) return HYPE_ERR_INVALID;
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    int rc = read_scalars(s);
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s->ev0, s->ev1) == cudaSuccess) s->last_ms = ms;
    if (steps_done) *steps_done = s->hSc->steps;
    if (t_end) *t_end = s->hSc->t;
    if (dt_next) *dt_next = s->hSc->time_step;
    return rc;
}

int hype_solve(hype_solver *s, double t0, double t_final, int max_steps, int *steps_done, double *t_end, double *dt_next)
{
    int rc = hype_begin(s, t0, t_final, max_steps);
    if (rc) return rc;
    // Each replay checks the stop condition on the device; replays after the
    // end return at once.  Poll between chunks so a t_final stop costs little.
    int launched = 0;
    const int chunk = 64;
    for (;;) {
        const int n = (max_steps - launched) < chunk ? (max_steps - launched) : chunk;
        if (n > 0) { if ((rc = hype_advance(s, n))) return rc; launched += n; }
        if ((rc = hype_wait(s, steps_done, t_end, dt_next))) return rc;
        if (s->hSc->done || launched >= max_steps) break;
    }
    // the loop above leaves done unset when it stopped exactly at max_steps
    return HYPE_OK;
}

int hype_totals(hype_solver *s, int scaled, double *totals, double *amin, double *amax)
{
    if (!s || !totals) return fail(s, HYPE_ERR_INVALID, "null argument");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    std::vector<double> h((size_t)s->nv + 2);
    if (s->mixed) {   // the mixed state widened to FP64 planes in the S0 buffer first
        CUDA_TRY(s, store_state(s, 0, s->dAosOut));
        CUDA_TRY(s, launch_aos_to_planes(s->dAosOut, s->dS0, s->cfg.nx, s->cfg.ny, s->nv, s->pitch, s->plane, s->stream));
    }
    CUDA_TRY(s, launch_totals(s->mixed ? s->dS0 : s->dU, s->dRed, s->cfg.nx, s->cfg.ny, s->nv, s->pitch, s->plane,
                              s->cfg.system == HYPE_EULER ? -1 : (s->cfg.system == HYPE_KAPILA_5EQN ? 5 : 8), s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(h.data(), s->dRed, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    const double area = scaled ? s->h * s->h : 1.0;
    for (int c = 0; c < s->nv; ++c) totals[c] = h[c] * area;
    if (amin) *amin = h[s->nv];
    if (amax) *amax = h[s->nv + 1];
    return HYPE_OK;
}

int hype_launch_info(const hype_solver *s, int *gx, int *gy, int *threads, size_t *smem, int *bps)
{
    if (!s) return HYPE_ERR_INVALID;
    if (gx) *gx = s->strips;
    if (gy) *gy = s->runs;
    if (threads) *threads = stage_threads(s->cells);
    if (smem) *smem = s->mixed ? mixed_smem_bytes(s->cfg.system, s->cells) : stage_smem_bytes(s->cfg.system, s->cfg.order, s->cells);
    if (bps) *bps = s->bps;
    return HYPE_OK;
}

int hype_time_stage(hype_solver *s, int reps, double *ms_per_launch)
{
    if (!s || reps < 1 || !ms_per_launch) return fail(s, HYPE_ERR_INVALID, "bad argument");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    int rc;
    // keep the time loop's scalars (t, dt, step count) for the caller
    DevScalars saved;
    CUDA_TRY(s, cudaMemcpyAsync(&saved, s->dSc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    if ((rc = reset_scalars(s))) return rc;
    s->hSc->dt = 1e-30;   // a representative AXPY stage S0 -> S1 with a negligible step
    CUDA_TRY(s, cudaMemcpyAsync(s->dSc, s->hSc, sizeof(DevScalars), cudaMemcpyHostToDevice, s->stream));
    auto one = [&]() -> cudaError_t {
        if (s->mixed) return stage_m(s, 1, 2, OUT_AXPY, 0, 2.0, 0, -1, 1);
        return stage(s, s->dS0, s->dS1, OUT_AXPY, 0, 2.0, 0, nullptr, nullptr, 1);
    };
    if (s->mixed) {
        const long long moff = (long long)s->row_off * s->pitch;   // whole planes, halo rows included
        const MixedLayout L = mixed_layout(s->cfg.system);
        CUDA_TRY(s, cudaMemcpyAsync(s->mf[1] - moff, s->mf[0] - moff, sizeof(float) * L.nf * (size_t)s->plane, cudaMemcpyDeviceToDevice,
                                    s->stream));
        CUDA_TRY(s, cudaMemcpyAsync(s->md[1] - moff, s->md[0] - moff, sizeof(double) * L.nd * (size_t)s->plane, cudaMemcpyDeviceToDevice,
                                    s->stream));
    } else {
        CUDA_TRY(s, cudaMemcpyAsync(solver_alloc_base(s, s->dS0), solver_alloc_base(s, s->dU), sizeof(double) * (size_t)s->plane * s->nv,
                                    cudaMemcpyDeviceToDevice, s->stream));
    }
    CUDA_TRY(s, one());   // warm
    CUDA_TRY(s, cudaEventRecord(s->ev0, s->stream));
    for (int k = 0; k < reps; ++k) CUDA_TRY(s, one());
    CUDA_TRY(s, cudaEventRecord(s->ev1, s->stream));
    if ((rc = read_scalars(s)) && rc != HYPE_ERR_INADMISSIBLE) return rc;
    float ms = 0.f;
    CUDA_TRY(s, cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    *ms_per_launch = (double)ms / reps;
    *s->hSc = saved;
    CUDA_TRY(s, cudaMemcpyAsync(s->dSc, s->hSc, sizeof(DevScalars), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return HYPE_OK;
}

int hype_autotune(hype_solver *s, int reps, int *cells_out, int *waves_out)
{
    if (!s) return HYPE_ERR_INVALID;
    if (reps < 1) reps = 3;
    static const int cand_cells[2] = {64, 128};
    static const int cand_waves[3] = {1, 2, 4};
    int best_c = s->cells, best_w = s->waves, rc;
    double best = 1e300;
    for (int c : cand_cells)
        for (int w : cand_waves) {
            if ((rc = set_tiling(s, c, w))) return rc;

            double ms = 0.0;
            if ((rc = hype_time_stage(s, reps, &ms))) return rc;
            if (ms < best) { best = ms; best_c = c; best_w = w; }
        }
    if ((rc = set_tiling(s, best_c, best_w))) return rc;
    if (cells_out) *cells_out = best_c;
    if (waves_out) *waves_out = best_w;
    return HYPE_OK;
}

int hype_solver_config(const hype_solver *s, hype_config *cfg)
{
    if (!s || !cfg) return HYPE_ERR_INVALID;
    *cfg = s->cfg;
    return HYPE_OK;
}

int hype_get_primitive(hype_solver *s, double *W)
{
    if (!s || !W) return fail(s, HYPE_ERR_INVALID, "null argument");
    CUDA_TRY(s, cudaSetDevice(s->cfg.device));
    const double *planes = s->dU;
    if (s->mixed) {   // widened to FP64 planes in S0 first
        CUDA_TRY(s, store_state(s, 0, s->dAosOut));
        CUDA_TRY(s, launch_aos_to_planes(s->dAosOut, s->dS0, s->cfg.nx, s->cfg.ny, s->nv, s->pitch, s->plane, s->stream));
        planes = s->dS0;
    }
    const StageParams p = base_params(s);
    CUDA_TRY(s, launch_cons2prim(s->cfg.system, p.eos, planes, s->dAosOut, s->cfg.nx, s->cfg.ny, s->pitch, s->plane, s->stream));
    CUDA_TRY(s, cudaMemcpyAsync(W, s->dAosOut, sizeof(double) * (size_t)s->cfg.nx * s->cfg.ny * s->nv, cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));
    return HYPE_OK;
}

int hype_last_elapsed_ms(const hype_solver *s, double *ms)
{
    if (!s || !ms) return HYPE_ERR_INVALID;
    *ms = s->last_ms;
    return HYPE_OK;
}

int hype_test_skip_row_loads(hype_solver *s, int row)
{
    if (!s) return HYPE_ERR_INVALID;
    CUDA_TRY(s, cudaStreamSynchronize(s->stream));   // no captured step of the old setting is in flight
    s->test_skip_row = row < 0 ? -1 : row;
    if (s->step_exec) { cudaGraphExecDestroy(s->step_exec); s->step_exec = nullptr; }
    return HYPE_OK;
}

}  // extern "C"

int hype::solver_reset_scalars(hype_solver *s) { return reset_scalars(s); }
int hype::solver_read_scalars(hype_solver *s) { return read_scalars(s); }
