// hype_group.cu -- one grid as y-slabs on one or more GPUs of one process
// (include/hype_group.h): HyPE-2D's DMDA decomposition (hype.c:108-122), its
// ghost-row refresh (rhs_function_prim.c:44-45) and the global minimum of dt
// (rhs_function_prim.c:620-623), done with the stage kernels' own stores into the
// neighbours' halo rows, events between the slabs' streams, and one reduction
// kernel per step.
#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>
#include "../../include/hype_group.h"
#include "hype_solver.h"

using namespace hype;

namespace {

constexpr int MAX_SLABS = 64;

struct GroupScalars {
    DevScalars *sc[MAX_SLABS];
    int n;
};

// The slabs' reductions made common: the largest wave speeds (the global minimum
// of dt, rhs_function_prim.c:620-623) and the union of the error bits, so that
// every slab takes the same dt and stops at the same step.  Each slab keeps its
// own first erring cell.  One thread; the slabs' DevScalars may be on other GPUs
// (peer loads and stores).
__global__ void group_reduce_kernel(GroupScalars g)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long smax = 0ull, smaxv = 0ull;
    unsigned err = 0u;
    for (int k = 0; k < g.n; ++k) {
        const DevScalars *s = g.sc[k];
        // non-negative doubles order as their bit patterns
        smax = s->smax > smax ? s->smax : smax;
        smaxv = s->smax_v > smaxv ? s->smax_v : smaxv;
        err |= s->err;
    }
    for (int k = 0; k < g.n; ++k) {
        DevScalars *s = g.sc[k];
        s->smax = smax;
        s->smax_v = smaxv;
        s->err = err;
    }
}

}  // namespace

struct hype_group {
    hype_config cfg;
    int n = 0;
    std::vector<hype_solver *> slab;
    std::vector<int> row0, rows, dev;
    std::vector<cudaEvent_t> ev;   // per slab, on its device: its last enqueued stage
    cudaEvent_t ev_red = nullptr, ev_fork = nullptr, ev0 = nullptr, ev1 = nullptr;   // slab 0's device
    cudaGraphExec_t exec = nullptr;
    GroupScalars gs;
    bool began = false;
    double last_ms = 0.0;
    char err[512] = {0};
};

static int gfail(hype_group *g, int code, const char *fmt, ...)
{
    if (g) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(g->err, sizeof(g->err), fmt, ap);
        va_end(ap);
    }
    return code;
}
#define G_TRY(g, expr)                                                                                     \
    do {                                                                                                   \
        cudaError_t e_ = (expr);                                                                           \
        if (e_ != cudaSuccess) return gfail((g), HYPE_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)
// a slab call's status, with the slab's message
#define G_SLAB(g, k, expr)                                                                                 \
    do {                                                                                                   \
        const int rc_ = (expr);                                                                            \
        if (rc_ != HYPE_OK) return gfail((g), rc_, "slab %d: %s", (k), hype_last_error((g)->slab[(k)])); \
    } while (0)

static int lo_of(const hype_group *g, int k) { return k > 0 ? k - 1 : (g->cfg.bc_bottom == HYPE_BC_PERIODIC ? g->n - 1 : -1); }
static int hi_of(const hype_group *g, int k) { return k + 1 < g->n ? k + 1 : (g->cfg.bc_top == HYPE_BC_PERIODIC ? 0 : -1); }

// stream k waits for the neighbours' last recorded stage
static cudaError_t wait_neighbours(hype_group *g, int k)
{
    cudaError_t e;
    const int nb[2] = {lo_of(g, k), hi_of(g, k)};
    for (int j : nb)
        if (j >= 0 && j != k && (e = cudaStreamWaitEvent(g->slab[k]->stream, g->ev[j], 0)) != cudaSuccess) return e;
    return cudaSuccess;
}

// after each slab's last enqueued work: the common maxima on slab 0's stream,
// every stream behind it
static cudaError_t reduce_all(hype_group *g)
{
    cudaError_t e;
    for (int k = 0; k < g->n; ++k) {
        if ((e = cudaSetDevice(g->dev[k])) != cudaSuccess || (e = cudaEventRecord(g->ev[k], g->slab[k]->stream)) != cudaSuccess) return e;
    }
    if ((e = cudaSetDevice(g->dev[0])) != cudaSuccess) return e;
    cudaStream_t lead = g->slab[0]->stream;
    for (int k = 1; k < g->n; ++k)
        if ((e = cudaStreamWaitEvent(lead, g->ev[k], 0)) != cudaSuccess) return e;
    group_reduce_kernel<<<1, 32, 0, lead>>>(g->gs);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaEventRecord(g->ev_red, lead)) != cudaSuccess) return e;
    for (int k = 1; k < g->n; ++k) {
        if ((e = cudaSetDevice(g->dev[k])) != cudaSuccess || (e = cudaStreamWaitEvent(g->slab[k]->stream, g->ev_red, 0)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

// One SSP-RK step over all slabs (ssp_plan's stages between begin_step and end_step).
// Stage st of slab k reads halo rows that stage st-1 of its neighbours stored, and
// stores into their halo rows of a buffer that their stage st-1 may still read: it
// waits for both neighbours' stage st-1.  Stage 0 follows the previous step's
// reduction, which follows every slab's last stage.
static cudaError_t enqueue_group_step(hype_group *g)
{
    cudaError_t e;
    PlanStage plan[MAX_PLAN];
    int copy_back = 0;
    const int ns = ssp_plan(g->cfg.order, plan, &copy_back);
    for (int k = 0; k < g->n; ++k) {
        if ((e = cudaSetDevice(g->dev[k])) != cudaSuccess || (e = launch_begin_step(g->slab[k]->dSc, g->slab[k]->stream)) != cudaSuccess)
            return e;
    }
    for (int st = 0; st < ns; ++st) {
        for (int k = 0; k < g->n; ++k) {
            if ((e = cudaSetDevice(g->dev[k])) != cudaSuccess) return e;
            if (st > 0 && (e = wait_neighbours(g, k)) != cudaSuccess) return e;
            if ((e = solver_stage(g->slab[k], plan[st])) != cudaSuccess) return e;
        }
        for (int k = 0; k < g->n; ++k)
            if ((e = cudaSetDevice(g->dev[k])) != cudaSuccess || (e = cudaEventRecord(g->ev[k], g->slab[k]->stream)) != cudaSuccess) return e;
    }
    if (copy_back) {   // forward Euler: u = S0, halo rows included (the neighbours' stores into S0 are done)
        for (int k = 0; k < g->n; ++k) {
            hype_solver *s = g->slab[k];
            if ((e = cudaSetDevice(g->dev[k])) != cudaSuccess || (e = wait_neighbours(g, k)) != cudaSuccess) return e;
            if ((e = cudaMemcpyAsync(solver_alloc_base(s, s->dU), solver_alloc_base(s, s->dS0), sizeof(double) * (size_t)s->plane * s->nv,
                                     cudaMemcpyDeviceToDevice, s->stream)) != cudaSuccess)
                return e;
        }
    }
    if ((e = reduce_all(g)) != cudaSuccess) return e;
    for (int k = 0; k < g->n; ++k) {
        if ((e = cudaSetDevice(g->dev[k])) != cudaSuccess || (e = launch_end_step(g->slab[k]->dSc, g->slab[k]->cfl_h, g->slab[k]->stream)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

// the step captured once as one graph over all slabs' streams
static int ensure_graph(hype_group *g)
{
    if (g->exec) return HYPE_OK;
    G_TRY(g, cudaSetDevice(g->dev[0]));
    cudaStream_t lead = g->slab[0]->stream;
    cudaGraph_t graph;
    G_TRY(g, cudaStreamBeginCapture(lead, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaEventRecord(g->ev_fork, lead);
    for (int k = 1; k < g->n && e == cudaSuccess; ++k) {
        if ((e = cudaSetDevice(g->dev[k])) == cudaSuccess) e = cudaStreamWaitEvent(g->slab[k]->stream, g->ev_fork, 0);
    }
    if (e == cudaSuccess) e = enqueue_group_step(g);
    // join every slab's stream back into the capturing one
    for (int k = 1; k < g->n && e == cudaSuccess; ++k) {
        if ((e = cudaSetDevice(g->dev[k])) == cudaSuccess) e = cudaEventRecord(g->ev[k], g->slab[k]->stream);
        if (e == cudaSuccess && (e = cudaSetDevice(g->dev[0])) == cudaSuccess) e = cudaStreamWaitEvent(lead, g->ev[k], 0);
    }
    cudaSetDevice(g->dev[0]);
    const cudaError_t e2 = cudaStreamEndCapture(lead, &graph);
    if (e != cudaSuccess) {
        if (e2 == cudaSuccess) cudaGraphDestroy(graph);
        return gfail(g, HYPE_ERR_CUDA, "step capture: %s", cudaGetErrorString(e));
    }
    if (e2 != cudaSuccess) return gfail(g, HYPE_ERR_CUDA, "step capture end: %s", cudaGetErrorString(e2));
    e = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return gfail(g, HYPE_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return HYPE_OK;
}

static int sync_all(hype_group *g)
{
    for (int k = 0; k < g->n; ++k) {
        G_TRY(g, cudaSetDevice(g->dev[k]));
        G_TRY(g, cudaStreamSynchronize(g->slab[k]->stream));
    }
    return HYPE_OK;
}

extern "C" {

int hype_group_create(const hype_config *cfg, int nslabs, const int *devices, hype_group **out)
{
    if (!out) return HYPE_ERR_INVALID;
    *out = nullptr;
    hype_group *g = new (std::nothrow) hype_group();
    if (!g) return HYPE_ERR_NOMEM;
    *out = g;
    int rc = validate_config(cfg, g->err, sizeof(g->err));
    if (rc) return rc;
    g->cfg = *cfg;
    if (nslabs < 1 || nslabs > MAX_SLABS || nslabs > cfg->ny / 3)
        return gfail(g, HYPE_ERR_INVALID, "nslabs must be 1..min(%d, ny/3 = %d) (got %d)", MAX_SLABS, cfg->ny / 3, nslabs);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return gfail(g, HYPE_ERR_NO_DEVICE, "no CUDA device");
    g->n = nslabs;
    g->slab.assign(nslabs, nullptr);
    g->ev.assign(nslabs, nullptr);
    g->row0.resize(nslabs);
    g->rows.resize(nslabs);
    g->dev.resize(nslabs);
    // PETSc's split of ny rows over n ranks: the first ny % n get one row more
    for (int k = 0, r = 0; k < nslabs; ++k) {
        g->row0[k] = r;
        g->rows[k] = cfg->ny / nslabs + (k < cfg->ny % nslabs ? 1 : 0);
        g->dev[k] = devices ? devices[k] : cfg->device;
        r += g->rows[k];
        if (g->dev[k] < 0 || g->dev[k] >= ndev) return gfail(g, HYPE_ERR_NO_DEVICE, "CUDA device %d not available", g->dev[k]);
    }
    // peer access between every two devices in use (neighbours' halo stores, the reduction)
    for (int a = 0; a < nslabs; ++a)
        for (int b = 0; b < nslabs; ++b) {
            const int da = g->dev[a], db = g->dev[b];
            if (da == db) continue;
            int can = 0;
            if (cudaDeviceCanAccessPeer(&can, da, db) != cudaSuccess || !can)
                return gfail(g, HYPE_ERR_INVALID, "device %d has no peer access to device %d", da, db);
            G_TRY(g, cudaSetDevice(da));
            const cudaError_t e = cudaDeviceEnablePeerAccess(db, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
            else if (e != cudaSuccess) return gfail(g, HYPE_ERR_CUDA, "cudaDeviceEnablePeerAccess(%d -> %d): %s", da, db, cudaGetErrorString(e));
        }
    const bool periodic = cfg->bc_bottom == HYPE_BC_PERIODIC;
    for (int k = 0; k < nslabs; ++k) {
        hype_config c = *cfg;
        c.device = g->dev[k];
        const bool halo_lo = nslabs > 1 && (k > 0 || periodic);
        const bool halo_hi = nslabs > 1 && (k + 1 < nslabs || periodic);
        rc = create_slab(&c, g->row0[k], g->rows[k], halo_lo, halo_hi, &g->slab[k]);
        if (rc) return gfail(g, rc, "slab %d: %s", k, g->slab[k] ? hype_last_error(g->slab[k]) : hype_status_string(rc));
        G_TRY(g, cudaSetDevice(g->dev[k]));
        G_TRY(g, cudaEventCreateWithFlags(&g->ev[k], cudaEventDisableTiming));
    }
    // neighbour planes by buffer role; row r of slab k is row r + rows[lo] of its lower
    // neighbour (that one's top halo) and row r - rows[k] of its upper neighbour
    for (int k = 0; k < nslabs; ++k) {
        hype_solver *s = g->slab[k];
        const int lo = lo_of(g, k), hi = hi_of(g, k);
        for (int role = B_U; role <= B_S2; ++role) {
            if (lo >= 0 && nslabs > 1) s->nb_lo[role] = solver_buf(g->slab[lo], role);
            if (hi >= 0 && nslabs > 1) s->nb_hi[role] = solver_buf(g->slab[hi], role);
        }
        for (int k3 = 0; k3 < 3 && s->mixed && nslabs > 1; ++k3) {   // mixed states U, S0, S1
            if (lo >= 0) { s->nbf_lo[k3] = g->slab[lo]->mf[k3]; s->nbd_lo[k3] = g->slab[lo]->md[k3]; }
            if (hi >= 0) { s->nbf_hi[k3] = g->slab[hi]->mf[k3]; s->nbd_hi[k3] = g->slab[hi]->md[k3]; }
        }
        if (lo >= 0) { s->nb_plane_lo = g->slab[lo]->plane; s->nb_shift_lo = g->rows[lo]; }
        if (hi >= 0) { s->nb_plane_hi = g->slab[hi]->plane; s->nb_shift_hi = -g->rows[k]; }
        g->gs.sc[k] = s->dSc;
    }
    g->gs.n = nslabs;
    G_TRY(g, cudaSetDevice(g->dev[0]));
    G_TRY(g, cudaEventCreateWithFlags(&g->ev_red, cudaEventDisableTiming));
    G_TRY(g, cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming));
    G_TRY(g, cudaEventCreate(&g->ev0));
    G_TRY(g, cudaEventCreate(&g->ev1));
    return HYPE_OK;
}

int hype_group_destroy(hype_group *g)
{
    if (!g) return HYPE_OK;
    for (int k = 0; k < g->n; ++k)
        if (g->slab[k] && g->slab[k]->stream) { cudaSetDevice(g->dev[k]); cudaStreamSynchronize(g->slab[k]->stream); }
    if (g->n > 0) cudaSetDevice(g->dev[0]);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    cudaEvent_t evs[] = {g->ev_red, g->ev_fork, g->ev0, g->ev1};
    for (cudaEvent_t e : evs) if (e) cudaEventDestroy(e);
    for (int k = 0; k < g->n; ++k) {
        cudaSetDevice(g->dev[k]);
        if (g->ev[k]) cudaEventDestroy(g->ev[k]);
        hype_destroy(g->slab[k]);
    }
    delete g;
    return HYPE_OK;
}

const char *hype_group_last_error(const hype_group *g) { return g ? g->err : "null group"; }

int hype_group_slab(const hype_group *g, int k, int *row0, int *rows, int *device)
{
    if (!g || k < 0 || k >= g->n) return HYPE_ERR_INVALID;
    if (row0) *row0 = g->row0[k];
    if (rows) *rows = g->rows[k];
    if (device) *device = g->dev[k];
    return HYPE_OK;
}

// Each slab takes its rows and, where it has a neighbour, the 3 rows beyond each
// edge (wrapping on a periodic y axis), so that its halo rows hold the state too.
int hype_group_set_state(hype_group *g, const double *U)
{
    if (!g || !U) return gfail(g, HYPE_ERR_INVALID, "null argument");
    if (g->n == 0) return gfail(g, HYPE_ERR_INVALID, "group not created");
    const int nx = g->cfg.nx, ny = g->cfg.ny, nv = hype_nvar(g->cfg.system);
    const size_t row_elems = (size_t)nx * nv;
    for (int k = 0; k < g->n; ++k) {
        hype_solver *s = g->slab[k];
        G_TRY(g, cudaSetDevice(g->dev[k]));
        const int lo = s->nb_lo[B_U] ? 3 : 0, hi = s->nb_hi[B_U] ? 3 : 0;
        // dAosIn holds local rows -3 .. rows+2 from its start
        for (int r = -lo; r < g->rows[k] + hi;) {
            const int gr = ((g->row0[k] + r) % ny + ny) % ny;
            int len = 1;   // a run of consecutive grid rows
            while (r + len < g->rows[k] + hi && gr + len < ny) ++len;
            G_TRY(g, cudaMemcpyAsync(s->dAosIn + (size_t)(r + 3) * row_elems, U + (size_t)gr * row_elems, sizeof(double) * row_elems * len,
                                     cudaMemcpyHostToDevice, s->stream));
            r += len;
        }
        if (s->mixed)
            G_TRY(g, launch_aos_to_mixed(s->cfg.system, s->dAosIn + (size_t)(3 - lo) * row_elems, s->mf[0] - (long long)lo * s->pitch,
                                         s->md[0] - (long long)lo * s->pitch, nx, g->rows[k] + lo + hi, s->pitch, s->plane, s->stream));
        else
            G_TRY(g, launch_aos_to_planes_rows(s->dAosIn, solver_alloc_base(s, s->dU), nx, 3 - lo, g->rows[k] + lo + hi, nv, s->pitch,
                                               s->plane, s->stream));
    }
    return sync_all(g);
}

int hype_group_get_state(hype_group *g, double *U)
{
    if (!g || !U) return gfail(g, HYPE_ERR_INVALID, "null argument");
    if (g->n == 0) return gfail(g, HYPE_ERR_INVALID, "group not created");
    const int nx = g->cfg.nx, nv = hype_nvar(g->cfg.system);
    const size_t row_elems = (size_t)nx * nv;
    for (int k = 0; k < g->n; ++k) {
        hype_solver *s = g->slab[k];
        G_TRY(g, cudaSetDevice(g->dev[k]));
        if (s->mixed) G_TRY(g, launch_mixed_to_aos(s->cfg.system, s->mf[0], s->md[0], s->dAosOut, nx, g->rows[k], s->pitch, s->plane, s->stream));
        else G_TRY(g, launch_planes_to_aos(s->dU, s->dAosOut, nx, g->rows[k], nv, s->pitch, s->plane, s->stream));
        G_TRY(g, cudaMemcpyAsync(U + (size_t)g->row0[k] * row_elems, s->dAosOut, sizeof(double) * row_elems * g->rows[k],
                                 cudaMemcpyDeviceToHost, s->stream));
    }
    return sync_all(g);
}

int hype_group_begin(hype_group *g, double t0, double t_final, int max_steps)
{
    if (!g || g->n == 0) return gfail(g, HYPE_ERR_INVALID, "group not created");
    if (max_steps < 0) return gfail(g, HYPE_ERR_INVALID, "max_steps < 0");
    for (int k = 0; k < g->n; ++k) {
        hype_solver *s = g->slab[k];
        G_TRY(g, cudaSetDevice(g->dev[k]));
        G_SLAB(g, k, solver_reset_scalars(s));
        s->hSc->t = t0; s->hSc->t_final = t_final; s->hSc->max_steps = max_steps;
        G_TRY(g, cudaMemcpyAsync(s->dSc, s->hSc, sizeof(DevScalars), cudaMemcpyHostToDevice, s->stream));
        // hype.c:343: one RHS evaluation of the initial state seeds Ctx.dt
        G_TRY(g, solver_seed_rhs(s));
    }
    G_TRY(g, reduce_all(g));
    for (int k = 0; k < g->n; ++k) {
        G_TRY(g, cudaSetDevice(g->dev[k]));
        G_TRY(g, launch_seed_dt(g->slab[k]->dSc, g->slab[k]->cfl_h, g->slab[k]->stream));
    }
    const int rc = ensure_graph(g);
    if (rc) return rc;
    g->began = true;
    return HYPE_OK;
}

int hype_group_advance(hype_group *g, int nsteps)
{
    if (!g || g->n == 0) return gfail(g, HYPE_ERR_INVALID, "group not created");
    if (!g->began) return gfail(g, HYPE_ERR_INVALID, "hype_group_begin not called");
    const int rc = ensure_graph(g);
    if (rc) return rc;
    G_TRY(g, cudaSetDevice(g->dev[0]));
    cudaStream_t lead = g->slab[0]->stream;
    // the graph starts behind every slab's enqueued work (it forks from slab 0's stream)
    for (int k = 1; k < g->n; ++k) {
        G_TRY(g, cudaSetDevice(g->dev[k]));
        G_TRY(g, cudaEventRecord(g->ev[k], g->slab[k]->stream));
        G_TRY(g, cudaSetDevice(g->dev[0]));
        G_TRY(g, cudaStreamWaitEvent(lead, g->ev[k], 0));
    }
    G_TRY(g, cudaEventRecord(g->ev0, lead));
    for (int k = 0; k < nsteps; ++k) G_TRY(g, cudaGraphLaunch(g->exec, lead));
    G_TRY(g, cudaEventRecord(g->ev1, lead));
    // and every slab's later work behind the graphs
    for (int k = 1; k < g->n; ++k) {
        G_TRY(g, cudaSetDevice(g->dev[k]));
        G_TRY(g, cudaStreamWaitEvent(g->slab[k]->stream, g->ev1, 0));
    }
    return HYPE_OK;
}

int hype_group_wait(hype_group *g, int *steps_done, double *t_end, double *dt_next)
{
    if (!g || g->n == 0) return gfail(g, HYPE_ERR_INVALID, "group not created");
    int rc = sync_all(g);
    if (rc) return rc;
    G_TRY(g, cudaSetDevice(g->dev[0]));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, g->ev0, g->ev1) == cudaSuccess) g->last_ms = ms;
    // every slab carries the common t, step count, dt and error bits (the reduction);
    // the first erring cell of the grid is the least of the slabs' own, shifted
    rc = HYPE_OK;
    unsigned long long cell = ~0ull;
    for (int k = 0; k < g->n; ++k) {
        hype_solver *sk = g->slab[k];
        G_TRY(g, cudaSetDevice(g->dev[k]));
        const int rk = solver_read_scalars(sk);
        if (rk && !rc) { rc = rk; gfail(g, rk, "%s", hype_last_error(sk)); }
        if (sk->hSc->err_cell != 0xffffffffu)
            cell = std::min(cell, (unsigned long long)g->row0[k] * g->cfg.nx + sk->hSc->err_cell);
    }
    if (rc == HYPE_ERR_INADMISSIBLE && cell != ~0ull)
        gfail(g, rc, "inadmissible face state near cell (i=%llu, j=%llu)", cell % (unsigned)g->cfg.nx, cell / (unsigned)g->cfg.nx);
    hype_solver *s = g->slab[0];
    if (steps_done) *steps_done = s->hSc->steps;
    if (t_end) *t_end = s->hSc->t;
    if (dt_next) *dt_next = s->hSc->time_step;
    return rc;
}

int hype_group_solve(hype_group *g, double t0, double t_final, int max_steps, int *steps_done, double *t_end, double *dt_next)
{
    int rc = hype_group_begin(g, t0, t_final, max_steps);
    if (rc) return rc;
    int launched = 0;
    const int chunk = 64;
    for (;;) {
        const int n = (max_steps - launched) < chunk ? (max_steps - launched) : chunk;
        if (n > 0) { if ((rc = hype_group_advance(g, n))) return rc; launched += n; }
        if ((rc = hype_group_wait(g, steps_done, t_end, dt_next))) return rc;
        if (g->slab[0]->hSc->done || launched >= max_steps) break;
    }
    return HYPE_OK;
}

int hype_group_last_elapsed_ms(const hype_group *g, double *ms)
{
    if (!g || !ms) return HYPE_ERR_INVALID;
    *ms = g->last_ms;
    return HYPE_OK;
}

}  // extern "C"
