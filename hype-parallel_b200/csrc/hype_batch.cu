// hype_batch.cu -- the C ABI of include/hype_batch.h: many independent
// instances (grid, state, time loop) advanced together.
//
// Instances are grouped by kind -- (system, order) in FP64, or the mixed
// Kapila N = 2 form -- because a kind fixes the stage kernel's template.  Per
// kind the device holds, indexed by instance slot:
//   params[stage][slot]   StageParams / MixedParams of each stage of the step
//   maps[buffer][slot]    TMA descriptors of the slot's U, S0, S1 buffers
//   work[]                (slot, tile) items of every member, longest first
//   members[]             count, then the member slots (step control)
//   sched[3]              item count and the persistent kernel's counters
// A step of the batch is one CUDA graph: per kind, on its own branch,
// begin-step, one persistent launch per stage, end-step.  Joins and leaves
// rewrite these arrays with stream-ordered copies; the graph is re-captured
// only when the set of non-empty kinds or a tile shape changes.
#include <cuda.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>
#include "../../include/hype_gpu.h"
#include "../../include/hype_batch.h"
#include "hype_internal.h"

using namespace hype;

namespace {

// kinds: FP64 primitive path 0..11 (3 systems x 4 orders), 12 = mixed Kapila N = 2,
// conservative path 13..24 (3 systems x 4 orders), viscous Kapila N = 1..3: primitive
// 25..27, conservative 28..30; mixed Baer-Nunziato and Euler N = 2: 31, 32
constexpr int NKIND = 33;
constexpr int KIND_MIXED = 12;
constexpr int KIND_CONS0 = 13, KIND_VISC0 = 25, KIND_VISC_CONS0 = 28;
constexpr int KIND_MIXED_BN = 31, KIND_MIXED_EULER = 32;
bool kind_is_mixed(int id) { return id == KIND_MIXED || id == KIND_MIXED_BN || id == KIND_MIXED_EULER; }
constexpr int NBUF = 4;                // U, S0, S1, S2
constexpr int MAX_SUBSTEPS = 16;       // steps an instance may take per batch step

int kind_of(const hype_config &c)
{
    if (c.precision == HYPE_PREC_MIXED)
        return c.system == HYPE_BAER_NUNZIATO ? KIND_MIXED_BN : c.system == HYPE_EULER ? KIND_MIXED_EULER : KIND_MIXED;
    const bool cons = (c.flags & HYPE_FLAG_CONSERVATIVE) != 0;
    if (c.flags & HYPE_FLAG_VISCOUS) return (cons ? KIND_VISC_CONS0 : KIND_VISC0) + c.order - 1;
    return (cons ? KIND_CONS0 : 0) + c.system * 4 + c.order;
}

// the persistent kernel family of a kind: -1 the primitive path's, else BATCH_PATH_*
int path_of_kind(int id)
{
    if (id >= KIND_VISC_CONS0) return BATCH_PATH_VISC_CONS;
    if (id >= KIND_VISC0) return BATCH_PATH_VISC;
    if (id >= KIND_CONS0) return BATCH_PATH_CONS;
    return -1;
}

struct Inst {
    bool used = false;
    int kind = -1;
    hype_config cfg;
    int nv = 0, pitch = 0;
    long long plane = 0;
    double h = 0.0, cfl_h = 0.0;
    double *buf[NBUF] = {nullptr, nullptr, nullptr, nullptr};   // FP64 planes
    float *mf[3] = {nullptr, nullptr, nullptr};                  // mixed: FP32 planes of U, S0, S1
    double *md[3] = {nullptr, nullptr, nullptr};                 //        FP64 planes
    double *inlet = nullptr;
    size_t bytes = 0;
    int strips = 1, runs = 1;
    int substeps = 1;                  // steps per batch step (hype_batch_set_substeps)
};

// The members taking sub-step j of a batch step (those with substeps > j):
// their step-control list and the (slot, tile) work-list of the stage launches.
struct SubList {
    int2 *dWork = nullptr;
    int work_cap = 0, nwork = 0;
    int *dSched = nullptr;             // [4]: item count, next item, blocks finished
    int *dMembers = nullptr;           // [1 + M]
};

struct Kind {
    int system = 0, order = 0;
    bool mixed = false;
    int path = -1;                     // BATCH_PATH_* for the conservative and viscous kinds (128-column tiles)
    bool ready = false;
    int nstage = 0, copy_back = 0;
    PlanStage plan[MAX_PLAN];
    int cells = STAGE_CELLS, rows = 64, bps = 0;
    std::vector<int> members;
    StageParams *dParams = nullptr;    // [MAX_PLAN][M]
    MixedParams *dMParams = nullptr;   // [MAX_PLAN][M]
    CUtensorMap *dMaps = nullptr;      // [3][M]
    MixedMaps *dMMaps = nullptr;       // [3][M]
    SubList sub[MAX_SUBSTEPS];
    int nsub = 1;                      // sub-steps in the captured step (max substeps of the members)
    long long cost = 0;                // cells of all members (autotune report)
    double **dCopyDst = nullptr, **dCopySrc = nullptr;   // forward Euler u = S0, [M]
    long long *dCopyN = nullptr;
};

}  // namespace

struct hype_batch {
    hype_batch_config cfg;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side[NKIND] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[NKIND] = {};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaMemPool_t pool = nullptr;
    std::vector<Inst> inst;
    DevScalars *dSc = nullptr;
    DevScalars *hSc = nullptr;        // pinned mirror, [M]
    int *dHold = nullptr;             // per-slot hold flags read by begin-step, [M]
    int *hHold = nullptr;             // pinned host copy
    bool hold_dirty = false;
    cudaEvent_t hold_ev = nullptr;    // completion of the last hold upload
    double *dStage = nullptr;         // Vec-layout staging, max_cells * 9 doubles
    Kind kinds[NKIND];
    cudaGraphExec_t exec = nullptr;
    bool dirty = true;
    size_t budget = 0, in_use = 0;
    double last_ms = 0.0;
    bool timed = false;
    char err[512] = {0};
};

static int bfail(hype_batch *b, int code, const char *fmt, ...)
{
    if (b) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(b->err, sizeof(b->err), fmt, ap);
        va_end(ap);
    }
    return code;
}
#define BCUDA(b, expr)                                                                                      \
    do {                                                                                                    \
        cudaError_t e_ = (expr);                                                                            \
        if (e_ != cudaSuccess) return bfail((b), HYPE_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

template <typename T>
static cudaError_t pool_alloc(hype_batch *b, T **p, size_t bytes)
{
    void *v = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&v, bytes, b->pool, b->stream);
    *p = static_cast<T *>(v);
    return e;
}
template <typename T>
static void pool_free(hype_batch *b, T *&p)
{
    if (p) cudaFreeAsync(p, b->stream);
    p = nullptr;
}

static int inst_pitch(const hype_config &c)
{
    return c.precision == HYPE_PREC_MIXED ? ((c.nx + 31) & ~31) : ((c.nx + 15) & ~15);
}

// state buffers of an instance, in bytes (what admission charges)
static size_t state_bytes(const hype_config &c)
{
    const long long plane = (long long)inst_pitch(c) * c.ny;
    if (c.precision == HYPE_PREC_MIXED) {
        const MixedLayout L = mixed_layout(c.system);
        return (size_t)3 * plane * (L.nf * sizeof(float) + L.nd * sizeof(double));
    }
    const int nbuf = c.order == 3 ? 4 : 3;
    size_t s = (size_t)nbuf * plane * hype_nvar(c.system) * sizeof(double);
    if (c.bc_left == HYPE_BC_INLET) s += sizeof(double) * 3 * (size_t)(c.ny + 6) * hype_nvar(c.system);
    return s;
}

// ---------------------------------------------------------------------------
// kinds: device arrays, tile shape, per-instance parameters, work-list
// ---------------------------------------------------------------------------
static int kind_blocks_per_sm(const Kind &k, int cells)
{
    if (k.path >= 0) return cells == STAGE_CELLS ? path_batch_blocks_per_sm(k.path, k.system, k.order) : 0;
    return k.mixed ? mixed_batch_blocks_per_sm(k.system, cells) : stage_batch_blocks_per_sm(k.system, k.order, cells);
}

static int sub_init(hype_batch *b, SubList &l)
{
    if (l.dSched) return HYPE_OK;
    const int M = b->cfg.max_instances;
    BCUDA(b, pool_alloc(b, &l.dSched, sizeof(int) * 4));
    BCUDA(b, cudaMemsetAsync(l.dSched, 0, sizeof(int) * 4, b->stream));
    BCUDA(b, pool_alloc(b, &l.dMembers, sizeof(int) * (1 + M)));
    BCUDA(b, cudaMemsetAsync(l.dMembers, 0, sizeof(int) * (1 + M), b->stream));
    return HYPE_OK;
}

static int kind_init(hype_batch *b, int id, const hype_config &c)
{
    Kind &k = b->kinds[id];
    if (k.ready) return HYPE_OK;
    const int M = b->cfg.max_instances;
    k.system = c.system;
    k.order = c.order;
    k.mixed = kind_is_mixed(id);
    k.path = path_of_kind(id);
    k.nstage = ssp_plan(c.order, k.plan, &k.copy_back);
    // the grid form of a path kind's kernel seeds each instance's dt
    if (k.path == BATCH_PATH_CONS) BCUDA(b, stage_cons_configure(c.system, c.order));
    else if (k.path >= 0) BCUDA(b, stage_visc_configure(c.order, k.path == BATCH_PATH_VISC_CONS));
    k.cells = k.mixed ? MIXED_CELLS : STAGE_CELLS;
    k.rows = 64;
    k.bps = kind_blocks_per_sm(k, k.cells);
    if (k.bps < 1) return bfail(b, HYPE_ERR_CUDA, "stage kernel of kind %d does not fit on an SM", id);
    if (k.mixed) {
        BCUDA(b, pool_alloc(b, &k.dMParams, sizeof(MixedParams) * MAX_PLAN * M));
        BCUDA(b, pool_alloc(b, &k.dMMaps, sizeof(MixedMaps) * 3 * M));
    } else {
        BCUDA(b, pool_alloc(b, &k.dParams, sizeof(StageParams) * MAX_PLAN * M));
        BCUDA(b, pool_alloc(b, &k.dMaps, sizeof(CUtensorMap) * 3 * M));
    }
    int rc;
    if ((rc = sub_init(b, k.sub[0]))) return rc;
    if (k.copy_back) {
        BCUDA(b, pool_alloc(b, &k.dCopyDst, sizeof(double *) * M));
        BCUDA(b, pool_alloc(b, &k.dCopySrc, sizeof(double *) * M));
        BCUDA(b, pool_alloc(b, &k.dCopyN, sizeof(long long) * M));
    }
    k.ready = true;
    return HYPE_OK;
}

// Tile decomposition of one instance for the kind's tile shape: strips of the
// stage kernel's column tiling, runs of about `rows` rows (at least 8 each).
static void inst_tiling(const Kind &k, Inst &in)
{
    const int nx = in.cfg.nx, ny = in.cfg.ny;
    in.strips = k.mixed ? mixed_strips(nx, k.cells) : stage_strips(nx, k.cells);
    int runs = (ny + k.rows / 2) / k.rows;
    const int cap = ny / 8 > 0 ? ny / 8 : 1;
    if (runs > cap) runs = cap;
    if (runs < 1) runs = 1;
    in.runs = runs;
}

static StageParams inst_params(hype_batch *b, const Inst &in, const PlanStage &q)
{
    StageParams p;
    std::memset(&p, 0, sizeof(p));
    const hype_config &c = in.cfg;
    p.nx = c.nx; p.ny = c.ny; p.pitch = in.pitch; p.plane = in.plane;
    p.strips = in.strips; p.runs = in.runs;
    p.bc[0] = c.bc_left; p.bc[1] = c.bc_right; p.bc[2] = c.bc_bottom; p.bc[3] = c.bc_top;
    p.eos.g1 = c.gamma1; p.eos.g2 = c.gamma2; p.eos.pi1 = c.pi1; p.eos.pi2 = c.pi2;
    p.eos.fix_p2 = (c.flags & HYPE_FLAG_BN_FIX_P2) ? 1 : 0;
    p.r1_h = 1. / in.h;
    p.cfl_h = in.cfl_h;
    p.sc = b->dSc + (&in - b->inst.data());
    p.inlet = in.inlet;
    p.in = q.in >= 0 ? in.buf[q.in] : nullptr;
    p.out = q.out >= 0 ? in.buf[q.out] : nullptr;
    p.xn = q.x >= 0 ? in.buf[q.x] : nullptr;
    p.out2 = q.out2 >= 0 ? in.buf[q.out2] : nullptr;
    p.mode = q.mode; p.ka = q.ka; p.kb = q.kb; p.kc = q.kc;
    p.reduce_smax = q.reduce;
    p.mu1 = c.mu1; p.mu2 = c.mu2;
    return p;
}

static MixedParams inst_mparams(hype_batch *b, const Inst &in, const PlanStage &q)
{
    MixedParams p;
    std::memset(&p, 0, sizeof(p));
    const hype_config &c = in.cfg;
    p.nx = c.nx; p.ny = c.ny; p.pitch = in.pitch; p.plane = in.plane;
    p.bc[0] = c.bc_left; p.bc[1] = c.bc_right; p.bc[2] = c.bc_bottom; p.bc[3] = c.bc_top;
    p.eos.g1 = c.gamma1; p.eos.g2 = c.gamma2; p.eos.pi1 = c.pi1; p.eos.pi2 = c.pi2;
    p.eos.fix_p2 = (c.flags & HYPE_FLAG_BN_FIX_P2) ? 1 : 0;
    p.r1_h = 1. / in.h; p.cfl_h = in.cfl_h;
    p.in_f = in.mf[q.in]; p.in_d = in.md[q.in];
    if (q.x >= 0) { p.xn_f = in.mf[q.x]; p.xn_d = in.md[q.x]; }
    if (q.out >= 0) { p.out_f = in.mf[q.out]; p.out_d = in.md[q.out]; }
    p.mode = q.mode; p.ka = q.ka; p.kb = q.kb; p.kc = q.kc;
    p.sc = b->dSc + (&in - b->inst.data());
    p.reduce_smax = q.reduce;
    p.strips = in.strips; p.runs = in.runs;
    return p;
}

// TMA descriptors of the instance's U, S0, S1 for the kind's tile width
static int inst_maps(hype_batch *b, const Kind &k, const Inst &in, CUtensorMap *maps, MixedMaps *mmaps)
{
    const hype_config &c = in.cfg;
    for (int q = 0; q < 3; ++q) {
        CUresult r;
        if (k.mixed) {
            const int bw = mixed_box_width(k.cells);
            const MixedLayout L = mixed_layout(c.system);
            r = encode_planes_map(&mmaps[q].f, in.mf[q], true, c.nx, c.ny, L.nf, in.pitch, in.plane, bw);
            if (r == CUDA_SUCCESS) r = encode_planes_map(&mmaps[q].d, in.md[q], false, c.nx, c.ny, L.nd, in.pitch, in.plane, bw);
        } else {
            r = encode_planes_map(&maps[q], in.buf[q], false, c.nx, c.ny, in.nv, in.pitch, in.plane, stage_box_width(k.cells, in.nv));
        }
        if (r != CUDA_SUCCESS) return bfail(b, HYPE_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    }
    return HYPE_OK;
}

// Uploads slot `s`'s stage parameters and descriptors into the kind's arrays.
static int upload_inst(hype_batch *b, int s)
{
    Inst &in = b->inst[s];
    Kind &k = b->kinds[in.kind];
    const int M = b->cfg.max_instances;
    inst_tiling(k, in);
    int rc;
    if (k.mixed) {
        MixedMaps mm[3];
        if ((rc = inst_maps(b, k, in, nullptr, mm))) return rc;
        for (int q = 0; q < 3; ++q)
            BCUDA(b, cudaMemcpyAsync(&k.dMMaps[q * M + s], &mm[q], sizeof(MixedMaps), cudaMemcpyHostToDevice, b->stream));
        for (int st = 0; st < k.nstage; ++st) {
            const MixedParams p = inst_mparams(b, in, k.plan[st]);
            BCUDA(b, cudaMemcpyAsync(&k.dMParams[st * M + s], &p, sizeof(p), cudaMemcpyHostToDevice, b->stream));
        }
    } else {
        CUtensorMap tm[3];
        if ((rc = inst_maps(b, k, in, tm, nullptr))) return rc;
        for (int q = 0; q < 3; ++q)
            BCUDA(b, cudaMemcpyAsync(&k.dMaps[q * M + s], &tm[q], sizeof(CUtensorMap), cudaMemcpyHostToDevice, b->stream));
        for (int st = 0; st < k.nstage; ++st) {
            const StageParams p = inst_params(b, in, k.plan[st]);
            BCUDA(b, cudaMemcpyAsync(&k.dParams[st * M + s], &p, sizeof(p), cudaMemcpyHostToDevice, b->stream));
        }
    }
    if (k.copy_back) {
        double *dst = in.buf[B_U], *src = in.buf[B_S0];
        const long long n = in.plane * in.nv;
        BCUDA(b, cudaMemcpyAsync(&k.dCopyDst[s], &dst, sizeof(dst), cudaMemcpyHostToDevice, b->stream));
        BCUDA(b, cudaMemcpyAsync(&k.dCopySrc[s], &src, sizeof(src), cudaMemcpyHostToDevice, b->stream));
        BCUDA(b, cudaMemcpyAsync(&k.dCopyN[s], &n, sizeof(n), cudaMemcpyHostToDevice, b->stream));
    }
    return HYPE_OK;
}

// Rebuilds the kind's member lists and work-lists, one per sub-step j (the
// members with substeps > j): every (slot, tile) of those members, sorted by
// estimated tile cost (columns x rows, halos included), longest first, so the
// persistent blocks finish together.
static int rebuild_work(hype_batch *b, int id)
{
    Kind &k = b->kinds[id];
    struct Item { long long cost; int2 it; int H, run, st, strips; };
    int K = 1;
    k.cost = 0;
    for (int s : k.members) {
        const Inst &in = b->inst[s];
        k.cost += (long long)in.cfg.nx * in.cfg.ny;
        if (in.substeps > K) K = in.substeps;
    }
    if (K != k.nsub) {
        k.nsub = K;
        b->dirty = true;
    }
    int rc;
    for (int j = 0; j < K; ++j) {
        SubList &l = k.sub[j];
        if ((rc = sub_init(b, l))) return rc;
        std::vector<Item> items;
        std::vector<int> mem(1, 0);
        for (int s : k.members) {
            const Inst &in = b->inst[s];
            if (in.substeps <= j) continue;
            mem.push_back(s);
            const int halo = k.mixed ? 8 : 6;
            for (int run = 0; run < in.runs; ++run) {
                const int H = (int)(((long long)(run + 1) * in.cfg.ny) / in.runs) - (int)(((long long)run * in.cfg.ny) / in.runs);
                for (int st = 0; st < in.strips; ++st) {
                    const int w = in.cfg.nx / in.strips + 1;
                    items.push_back(Item{(long long)(w + halo) * (H + 6), make_int2(s, run * in.strips + st), H, run, st, in.strips});
                }
            }
        }
        mem[0] = (int)mem.size() - 1;
        auto longest_first = [](const Item &x, const Item &y) { return x.cost > y.cost; };
        std::stable_sort(items.begin(), items.end(), longest_first);
        // The last wave of the list (half the resident blocks' worth of items) decides
        // when the launch ends: its tiles of 32 rows or more are split into two runs of
        // the instance's decomposition refined twice (item_refine), so the blocks finish
        // closer together.  The list is sorted again.
        const int tail = std::min((int)items.size(), std::max(1, b->sms * k.bps / 2));
        const int split_from = (int)items.size() - tail;
        for (int i = (int)items.size() - 1; i >= split_from; --i) {
            Item &x = items[i];
            if (x.H < 32) continue;
            const int w = (int)(x.cost / (x.H + 6));
            const int s = x.it.x, st = x.st, S = x.strips, r = x.run;
            const Inst &in = b->inst[s];
            const long long R2 = 2LL * in.runs;
            int h2[2];
            for (int q = 0; q < 2; ++q)
                h2[q] = (int)(((long long)(2 * r + q + 1) * in.cfg.ny) / R2) - (int)(((long long)(2 * r + q) * in.cfg.ny) / R2);
            x = Item{(long long)w * (h2[0] + 6), make_int2(s, (1 << 28) | ((2 * r) * S + st)), h2[0], 2 * r, st, S};
            items.push_back(Item{(long long)w * (h2[1] + 6), make_int2(s, (1 << 28) | ((2 * r + 1) * S + st)), h2[1], 2 * r + 1, st, S});
        }
        std::stable_sort(items.begin(), items.end(), longest_first);
        const int n = (int)items.size();
        if (n > l.work_cap) {
            int cap = l.work_cap > 0 ? l.work_cap : 1024;
            while (cap < n) cap *= 2;
            if (b->exec) {   // the captured graph holds the old pointer
                BCUDA(b, cudaStreamSynchronize(b->stream));
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
            }
            pool_free(b, l.dWork);
            BCUDA(b, pool_alloc(b, &l.dWork, sizeof(int2) * cap));
            l.work_cap = cap;
            b->dirty = true;
        }
        std::vector<int2> w(n);
        for (int i = 0; i < n; ++i) w[i] = items[i].it;
        if (n) BCUDA(b, cudaMemcpyAsync(l.dWork, w.data(), sizeof(int2) * n, cudaMemcpyHostToDevice, b->stream));
        BCUDA(b, cudaMemcpyAsync(l.dSched, &n, sizeof(int), cudaMemcpyHostToDevice, b->stream));
        BCUDA(b, cudaMemcpyAsync(l.dMembers, mem.data(), sizeof(int) * mem.size(), cudaMemcpyHostToDevice, b->stream));
        l.nwork = n;
    }
    return HYPE_OK;
}

// New tile shape for a kind: every member's decomposition, descriptors and
// parameters, then the work-list.
static int kind_set_tiling(hype_batch *b, int id, int cells, int rows)
{
    Kind &k = b->kinds[id];
    if (!k.ready) return HYPE_OK;
    if (k.path >= 0) cells = STAGE_CELLS;   // the conservative and viscous kernels come in 128-column tiles
    const int bps = kind_blocks_per_sm(k, cells);
    if (bps < 1) return bfail(b, HYPE_ERR_CUDA, "stage kernel does not fit on an SM with %d-column tiles", cells);
    if (k.cells != cells) b->dirty = true;
    k.cells = cells;
    k.rows = rows;
    k.bps = bps;
    int rc;
    for (int s : k.members)
        if ((rc = upload_inst(b, s))) return rc;
    if ((rc = rebuild_work(b, id))) return rc;
    b->dirty = true;
    return HYPE_OK;
}

// ---------------------------------------------------------------------------
// the step graph
// ---------------------------------------------------------------------------
static cudaError_t enqueue_kind_stage(hype_batch *b, int id, int st, cudaStream_t s, int j = 0)
{
    Kind &k = b->kinds[id];
    SubList &l = k.sub[j];
    const int M = b->cfg.max_instances;
    const int blocks = b->sms * k.bps;
    const PlanStage &q = k.plan[st];
    if (k.mixed) return launch_mixed_batch(k.system, k.cells, k.dMParams + st * M, k.dMMaps + q.in * M, l.dWork, l.dSched, blocks, s);
    if (k.path >= 0) return launch_path_batch(k.path, k.system, k.order, k.dParams + st * M, k.dMaps + q.in * M, l.dWork, l.dSched, blocks, s);
    return launch_stage_batch(k.system, k.order, k.cells, k.dParams + st * M, k.dMaps + q.in * M, l.dWork, l.dSched, blocks, s);
}

// One batch step of a kind: sub-step j steps the members with substeps > j.
static cudaError_t enqueue_kind_step(hype_batch *b, int id, cudaStream_t s)
{
    Kind &k = b->kinds[id];
    const int M = b->cfg.max_instances;
    cudaError_t e;
    for (int j = 0; j < k.nsub; ++j) {
        const int *mem = k.sub[j].dMembers;
        if ((e = launch_begin_step_batch(b->dSc, mem, b->dHold, M, s)) != cudaSuccess) return e;
        for (int st = 0; st < k.nstage; ++st)
            if ((e = enqueue_kind_stage(b, id, st, s, j)) != cudaSuccess) return e;
        if (k.copy_back && (e = launch_copy_batch(k.dCopyDst, k.dCopySrc, k.dCopyN, mem, M, b->dSc, s)) != cudaSuccess) return e;
        if ((e = launch_end_step_batch(b->dSc, mem, M, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Captures one step of every non-empty kind; kinds run on parallel branches.
static int capture_step(hype_batch *b)
{
    if (b->exec) {
        BCUDA(b, cudaStreamSynchronize(b->stream));
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    std::vector<int> live;
    for (int id = 0; id < NKIND; ++id)
        if (b->kinds[id].ready && !b->kinds[id].members.empty()) live.push_back(id);
    b->dirty = false;
    if (live.empty()) return HYPE_OK;
    cudaGraph_t g;
    BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    if (live.size() == 1) {
        e = enqueue_kind_step(b, live[0], b->stream);
    } else {
        e = cudaEventRecord(b->fork, b->stream);
        for (int id : live) {
            if (e == cudaSuccess) e = cudaStreamWaitEvent(b->side[id], b->fork, 0);
            if (e == cudaSuccess) e = enqueue_kind_step(b, id, b->side[id]);
            if (e == cudaSuccess) e = cudaEventRecord(b->join[id], b->side[id]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[id], 0);
        }
    }
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) {
        if (e2 == cudaSuccess) cudaGraphDestroy(g);
        return bfail(b, HYPE_ERR_CUDA, "batch step capture: %s", cudaGetErrorString(e));
    }
    if (e2 != cudaSuccess) return bfail(b, HYPE_ERR_CUDA, "batch step capture end: %s", cudaGetErrorString(e2));
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->dirty = true; return bfail(b, HYPE_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e)); }
    return HYPE_OK;
}

static int inst_status(const hype_batch *b, int s)
{
    const DevScalars &d = b->hSc[s];
    if (d.err & ERR_TMA_TIMEOUT) return HYPE_ERR_TIMEOUT;
    if (d.err & ERR_BAD_LAUNCH) return HYPE_ERR_CUDA;
    if (d.err & ERR_INADMISSIBLE_FACE) return HYPE_ERR_INADMISSIBLE;
    return HYPE_OK;
}

static void free_inst(hype_batch *b, Inst &in)
{
    for (int q = 0; q < NBUF; ++q) pool_free(b, in.buf[q]);
    for (int q = 0; q < 3; ++q) { pool_free(b, in.mf[q]); pool_free(b, in.md[q]); }
    pool_free(b, in.inlet);
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void hype_batch_config_default(hype_batch_config *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->device = 0;
    c->max_instances = 256;
    c->hbm_budget = 0;
    c->max_cells = 2048LL * 2048LL;
}

const char *hype_batch_last_error(const hype_batch *b) { return b ? b->err : "null batch"; }

size_t hype_batch_instance_bytes(const hype_config *cfg)
{
    if (!cfg || validate_config(cfg, nullptr, 0) != HYPE_OK) return 0;
    return state_bytes(*cfg);
}

int hype_batch_destroy(hype_batch *b)
{
    if (!b) return HYPE_OK;
    cudaSetDevice(b->cfg.device);
    if (b->stream) {
        cudaStreamSynchronize(b->stream);
        if (b->exec) cudaGraphExecDestroy(b->exec);
        for (Inst &in : b->inst)
            if (in.used) free_inst(b, in);
        for (Kind &k : b->kinds) {
            pool_free(b, k.dParams); pool_free(b, k.dMParams); pool_free(b, k.dMaps); pool_free(b, k.dMMaps);
            for (SubList &l : k.sub) { pool_free(b, l.dWork); pool_free(b, l.dSched); pool_free(b, l.dMembers); }
            pool_free(b, k.dCopyDst); pool_free(b, k.dCopySrc); pool_free(b, k.dCopyN);
        }
        cudaStreamSynchronize(b->stream);
    }
    if (b->pool) cudaMemPoolDestroy(b->pool);
    if (b->dSc) cudaFree(b->dSc);
    if (b->hSc) cudaFreeHost(b->hSc);
    if (b->dHold) cudaFree(b->dHold);
    if (b->hHold) cudaFreeHost(b->hHold);
    if (b->hold_ev) cudaEventDestroy(b->hold_ev);
    if (b->dStage) cudaFree(b->dStage);
    for (int k = 0; k < NKIND; ++k) {
        if (b->side[k]) cudaStreamDestroy(b->side[k]);
        if (b->join[k]) cudaEventDestroy(b->join[k]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return HYPE_OK;
}

int hype_batch_create(const hype_batch_config *c, hype_batch **out)
{
    if (!out) return HYPE_ERR_INVALID;
    *out = nullptr;
    hype_batch *b = new (std::nothrow) hype_batch();
    if (!b) return HYPE_ERR_NOMEM;
    *out = b;   // on failure the caller reads hype_batch_last_error, then destroys
    if (!c) return bfail(b, HYPE_ERR_INVALID, "null config");
    b->cfg = *c;
    if (c->max_instances < 1 || c->max_instances > 65536) return bfail(b, HYPE_ERR_INVALID, "max_instances must be 1..65536");
    if (c->max_cells < 9) return bfail(b, HYPE_ERR_INVALID, "max_cells must be at least 9");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || c->device < 0 || c->device >= ndev)
        return bfail(b, HYPE_ERR_NO_DEVICE, "CUDA device %d not available", c->device);
    BCUDA(b, cudaSetDevice(c->device));
    cudaDeviceProp prop;
    BCUDA(b, cudaGetDeviceProperties(&prop, c->device));
    if (prop.major != 10) return bfail(b, HYPE_ERR_NO_DEVICE, "device %d is sm_%d%d; the library is built for sm_100a", c->device, prop.major, prop.minor);
    b->sms = prop.multiProcessorCount;
    BCUDA(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    for (int k = 0; k < NKIND; ++k) {
        BCUDA(b, cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking));
        BCUDA(b, cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming));
    }
    BCUDA(b, cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    BCUDA(b, cudaEventCreate(&b->ev0));
    BCUDA(b, cudaEventCreate(&b->ev1));
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = c->device;
    BCUDA(b, cudaMemPoolCreate(&b->pool, &props));
    unsigned long long keep = ~0ull;   // freed instances' memory stays in the pool for the next joins
    BCUDA(b, cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    const int M = c->max_instances;
    BCUDA(b, cudaMalloc(&b->dSc, sizeof(DevScalars) * M));
    BCUDA(b, cudaMemset(b->dSc, 0, sizeof(DevScalars) * M));
    BCUDA(b, cudaMallocHost(&b->hSc, sizeof(DevScalars) * M));
    std::memset(b->hSc, 0, sizeof(DevScalars) * M);
    BCUDA(b, cudaMalloc(&b->dHold, sizeof(int) * M));
    BCUDA(b, cudaMemset(b->dHold, 0, sizeof(int) * M));
    BCUDA(b, cudaMallocHost(&b->hHold, sizeof(int) * M));
    std::memset(b->hHold, 0, sizeof(int) * M);
    BCUDA(b, cudaEventCreateWithFlags(&b->hold_ev, cudaEventDisableTiming));
    if (cudaMalloc(&b->dStage, sizeof(double) * 9 * (size_t)c->max_cells) != cudaSuccess)
        return bfail(b, HYPE_ERR_NOMEM, "staging buffer of %lld cells", (long long)c->max_cells);
    b->inst.resize(M);
    size_t fr = 0, tot = 0;
    BCUDA(b, cudaMemGetInfo(&fr, &tot));
    b->budget = c->hbm_budget ? c->hbm_budget : (size_t)(0.8 * (double)fr);
    return HYPE_OK;
}

int hype_batch_add(hype_batch *b, const hype_config *cfg, const double *U0, double t0, double t_final, int max_steps, int *id)
{
    if (!b || !cfg || !U0 || !id) return bfail(b, HYPE_ERR_INVALID, "null argument");
    if (!b->dSc) return bfail(b, HYPE_ERR_INVALID, "batch not created");
    if (max_steps < 0) return bfail(b, HYPE_ERR_INVALID, "max_steps < 0");
    char msg[256];
    int rc = validate_config(cfg, msg, sizeof(msg));
    if (rc) return bfail(b, rc, "%s", msg);
    if (cfg->precision == HYPE_PREC_FP64_FAST)
        return bfail(b, HYPE_ERR_INVALID, "the FP64 performance form runs in single solvers and slab groups, not in batches");
    if ((long long)cfg->nx * cfg->ny > b->cfg.max_cells)
        return bfail(b, HYPE_ERR_INVALID, "grid %dx%d exceeds the batch's max_cells (%lld)", cfg->nx, cfg->ny, (long long)b->cfg.max_cells);
    int s = -1;
    for (int k = 0; k < (int)b->inst.size(); ++k)
        if (!b->inst[k].used) { s = k; break; }
    if (s < 0) return bfail(b, HYPE_ERR_BUSY, "all %d instance slots are taken", (int)b->inst.size());
    const size_t bytes = state_bytes(*cfg);
    if (b->in_use + bytes > b->budget)
        return bfail(b, HYPE_ERR_NOMEM, "admission: %zu bytes in use + %zu exceed the HBM budget of %zu", b->in_use, bytes, b->budget);
    BCUDA(b, cudaSetDevice(b->cfg.device));
    BCUDA(b, cudaStreamSynchronize(b->stream));

    Inst &in = b->inst[s];
    in = Inst();
    in.cfg = *cfg;
    in.cfg.device = b->cfg.device;
    in.kind = kind_of(*cfg);
    in.nv = hype_nvar(cfg->system);
    in.pitch = inst_pitch(*cfg);
    in.plane = (long long)in.pitch * cfg->ny;
    in.h = (cfg->x_max - cfg->x_min) / (double)cfg->nx;   // hype.c:57
    in.cfl_h = cfg->cfl * in.h;                           // rhs_function_prim.c:620
    const bool mixed = kind_is_mixed(in.kind);
    bool ok = true;
    if (mixed) {
        const MixedLayout L = mixed_layout(cfg->system);
        for (int q = 0; q < 3 && ok; ++q)
            ok = pool_alloc(b, &in.mf[q], sizeof(float) * L.nf * (size_t)in.plane) == cudaSuccess &&
                 pool_alloc(b, &in.md[q], sizeof(double) * L.nd * (size_t)in.plane) == cudaSuccess;
    } else {
        const int nbuf = cfg->order == 3 ? 4 : 3;
        for (int q = 0; q < nbuf && ok; ++q) ok = pool_alloc(b, &in.buf[q], sizeof(double) * in.nv * (size_t)in.plane) == cudaSuccess;
    }
    std::vector<double> tab;
    if (ok && cfg->bc_left == HYPE_BC_INLET) {
        inlet_table(*cfg, in.h, tab);
        if (cfg->flags & HYPE_FLAG_CONSERVATIVE) inlet_to_conserved(*cfg, tab);
        ok = pool_alloc(b, &in.inlet, sizeof(double) * tab.size()) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        free_inst(b, in);
        return bfail(b, HYPE_ERR_NOMEM, "device pool allocation of %zu bytes failed", bytes);
    }
    if ((rc = kind_init(b, in.kind, *cfg))) { free_inst(b, in); return rc; }
    Kind &k = b->kinds[in.kind];
    if (!tab.empty()) BCUDA(b, cudaMemcpyAsync(in.inlet, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, b->stream));
    const size_t aos_bytes = sizeof(double) * (size_t)cfg->nx * cfg->ny * in.nv;
    BCUDA(b, cudaMemcpyAsync(b->dStage, U0, aos_bytes, cudaMemcpyHostToDevice, b->stream));
    if (mixed) BCUDA(b, launch_aos_to_mixed(cfg->system, b->dStage, in.mf[0], in.md[0], cfg->nx, cfg->ny, in.pitch, in.plane, b->stream));
    else BCUDA(b, launch_aos_to_planes(b->dStage, in.buf[B_U], cfg->nx, cfg->ny, in.nv, in.pitch, in.plane, b->stream));
    // time loop of this instance (hype_begin): t0, t_final, max_steps, dt from the RHS of U0
    DevScalars &h = b->hSc[s];
    std::memset(&h, 0, sizeof(h));
    h.err_cell = 0xffffffffu;
    h.t = t0; h.t_final = t_final; h.max_steps = max_steps;
    h.cfl_h = in.cfl_h;
    h.r1h_v = (cfg->flags & HYPE_FLAG_VISCOUS) ? 1. / in.h : 0.0;   // the viscous dt term (rhs_function_prim.c:617)
    BCUDA(b, cudaMemcpyAsync(&b->dSc[s], &h, sizeof(h), cudaMemcpyHostToDevice, b->stream));
    in.used = true;
    in.bytes = bytes;
    b->in_use += bytes;
    if (b->hHold[s]) {
        BCUDA(b, cudaEventSynchronize(b->hold_ev));
        b->hHold[s] = 0;
        b->hold_dirty = true;
    }
    k.members.push_back(s);
    if (k.members.size() == 1) b->dirty = true;
    if ((rc = upload_inst(b, s)) || (rc = rebuild_work(b, in.kind))) return rc;
    // hype.c:343: one RHS evaluation of the initial state seeds Ctx.dt
    const PlanStage seed{B_U, mixed ? B_NONE : B_S1, OUT_RHS, 0.0, 1.0, 0.0, B_NONE, B_NONE, 1};
    if (mixed) {
        MixedMaps mm[3];
        if ((rc = inst_maps(b, k, in, nullptr, mm))) return rc;
        MixedParams p = inst_mparams(b, in, seed);
        p.out_rhs = b->dStage;
        BCUDA(b, launch_mixed(cfg->system, k.cells, mm[0], p, b->stream));
    } else {
        CUtensorMap tm[3];
        if ((rc = inst_maps(b, k, in, tm, nullptr))) return rc;
        const StageParams sp = inst_params(b, in, seed);
        if (k.path == BATCH_PATH_CONS) BCUDA(b, launch_stage_cons(k.system, k.order, tm[0], sp, b->stream));
        else if (k.path >= 0) BCUDA(b, launch_stage_visc(k.order, k.path == BATCH_PATH_VISC_CONS, tm[0], sp, b->stream));
        else BCUDA(b, launch_stage(k.system, k.order, k.cells, tm[0], sp, b->stream));
    }
    BCUDA(b, launch_seed_dt(&b->dSc[s], in.cfl_h, b->stream));
    BCUDA(b, cudaMemcpyAsync(&b->hSc[s], &b->dSc[s], sizeof(DevScalars), cudaMemcpyDeviceToHost, b->stream));
    BCUDA(b, cudaStreamSynchronize(b->stream));
    *id = s;
    return HYPE_OK;
}

int hype_batch_remove(hype_batch *b, int id)
{
    if (!b || id < 0 || id >= (int)b->inst.size() || !b->inst[id].used) return bfail(b, HYPE_ERR_INVALID, "no instance %d", id);
    BCUDA(b, cudaSetDevice(b->cfg.device));
    Inst &in = b->inst[id];
    Kind &k = b->kinds[in.kind];
    k.members.erase(std::find(k.members.begin(), k.members.end(), id));
    if (k.members.empty()) b->dirty = true;
    int rc = rebuild_work(b, in.kind);   // ordered before the next step on the stream
    free_inst(b, in);                     // after the steps already queued
    b->in_use -= in.bytes;
    in.used = false;
    std::memset(&b->hSc[id], 0, sizeof(DevScalars));
    return rc;
}

int hype_batch_advance(hype_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return bfail(b, HYPE_ERR_INVALID, "bad argument");
    BCUDA(b, cudaSetDevice(b->cfg.device));
    int rc;
    if (b->dirty && (rc = capture_step(b))) return rc;
    if (!b->exec) { b->timed = false; return HYPE_OK; }
    if (b->hold_dirty) {
        BCUDA(b, cudaMemcpyAsync(b->dHold, b->hHold, sizeof(int) * b->inst.size(), cudaMemcpyHostToDevice, b->stream));
        BCUDA(b, cudaEventRecord(b->hold_ev, b->stream));
        b->hold_dirty = false;
    }
    BCUDA(b, cudaEventRecord(b->ev0, b->stream));
    for (int k = 0; k < nsteps; ++k) BCUDA(b, cudaGraphLaunch(b->exec, b->stream));
    BCUDA(b, cudaEventRecord(b->ev1, b->stream));
    b->timed = true;
    return HYPE_OK;
}

int hype_batch_sync(hype_batch *b)
{
    if (!b) return HYPE_ERR_INVALID;
    BCUDA(b, cudaSetDevice(b->cfg.device));
    BCUDA(b, cudaMemcpyAsync(b->hSc, b->dSc, sizeof(DevScalars) * b->inst.size(), cudaMemcpyDeviceToHost, b->stream));
    BCUDA(b, cudaStreamSynchronize(b->stream));
    for (size_t s = 0; s < b->inst.size(); ++s)
        if (!b->inst[s].used) std::memset(&b->hSc[s], 0, sizeof(DevScalars));
    if (b->timed) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) b->last_ms = ms;
        b->timed = false;
    }
    return HYPE_OK;
}

int hype_batch_status(const hype_batch *b, int id, hype_instance_status *st)
{
    if (!b || !st || id < 0 || id >= (int)b->inst.size()) return HYPE_ERR_INVALID;
    std::memset(st, 0, sizeof(*st));
    if (!b->inst[id].used) return HYPE_OK;
    const DevScalars &d = b->hSc[id];
    st->active = 1;
    st->done = d.done;
    st->steps = d.steps;
    st->status = inst_status(b, id);
    st->t = d.t;
    st->dt_next = d.time_step;
    st->held = b->hHold[id];
    st->substeps = b->inst[id].substeps;
    return HYPE_OK;
}

int hype_batch_set_substeps(hype_batch *b, int id, int substeps)
{
    if (!b || id < 0 || id >= (int)b->inst.size() || !b->inst[id].used) return bfail(b, HYPE_ERR_INVALID, "no instance %d", id);
    if (substeps < 1 || substeps > MAX_SUBSTEPS) return bfail(b, HYPE_ERR_INVALID, "substeps must be 1..%d", MAX_SUBSTEPS);
    Inst &in = b->inst[id];
    if (in.substeps == substeps) return HYPE_OK;
    BCUDA(b, cudaSetDevice(b->cfg.device));
    in.substeps = substeps;
    return rebuild_work(b, in.kind);
}

int hype_batch_hold(hype_batch *b, int id, int hold)
{
    if (!b || id < 0 || id >= (int)b->inst.size() || !b->inst[id].used) return bfail(b, HYPE_ERR_INVALID, "no instance %d", id);
    const int v = hold ? 1 : 0;
    if (b->hHold[id] == v) return HYPE_OK;
    BCUDA(b, cudaSetDevice(b->cfg.device));
    BCUDA(b, cudaEventSynchronize(b->hold_ev));   // the last upload has read the host array
    b->hHold[id] = v;
    b->hold_dirty = true;
    return HYPE_OK;
}

int hype_batch_get_state(hype_batch *b, int id, double *U)
{
    if (!b || !U || id < 0 || id >= (int)b->inst.size() || !b->inst[id].used) return bfail(b, HYPE_ERR_INVALID, "no instance %d", id);
    BCUDA(b, cudaSetDevice(b->cfg.device));
    const Inst &in = b->inst[id];
    const hype_config &c = in.cfg;
    if (kind_is_mixed(in.kind)) BCUDA(b, launch_mixed_to_aos(c.system, in.mf[0], in.md[0], b->dStage, c.nx, c.ny, in.pitch, in.plane, b->stream));
    else BCUDA(b, launch_planes_to_aos(in.buf[B_U], b->dStage, c.nx, c.ny, in.nv, in.pitch, in.plane, b->stream));
    BCUDA(b, cudaMemcpyAsync(U, b->dStage, sizeof(double) * (size_t)c.nx * c.ny * in.nv, cudaMemcpyDeviceToHost, b->stream));
    BCUDA(b, cudaStreamSynchronize(b->stream));
    return HYPE_OK;
}

int hype_batch_set_tiling(hype_batch *b, int cells, int rows)
{
    if (!b) return HYPE_ERR_INVALID;
    if ((cells != 64 && cells != 128) || rows < 16 || rows > 1024)
        return bfail(b, HYPE_ERR_INVALID, "tile shape must be 64 or 128 columns and 16..1024 rows");
    BCUDA(b, cudaSetDevice(b->cfg.device));
    int rc;
    for (int id = 0; id < NKIND; ++id)
        if ((rc = kind_set_tiling(b, id, cells, rows))) return rc;
    return HYPE_OK;
}

int hype_batch_autotune(hype_batch *b, int reps, int *cells_out, int *rows_out)
{
    if (!b) return HYPE_ERR_INVALID;
    if (reps < 1) reps = 3;
    BCUDA(b, cudaSetDevice(b->cfg.device));
    static const int cand_cells[2] = {64, 128};
    static const int cand_rows[4] = {16, 32, 64, 128};
    long long most = -1;
    int rc;
    for (int id = 0; id < NKIND; ++id) {
        Kind &k = b->kinds[id];
        if (!k.ready || k.members.empty()) continue;
        int bc = k.cells, br = k.rows;
        double best = 1e300;
        for (int c : cand_cells)
            for (int r : cand_rows) {
                if (k.path >= 0 && c != STAGE_CELLS) continue;
                if ((rc = kind_set_tiling(b, id, c, r))) return rc;
                BCUDA(b, enqueue_kind_stage(b, id, 0, b->stream));   // warm
                BCUDA(b, cudaEventRecord(b->ev0, b->stream));
                for (int i = 0; i < reps; ++i) BCUDA(b, enqueue_kind_stage(b, id, 0, b->stream));
                BCUDA(b, cudaEventRecord(b->ev1, b->stream));
                BCUDA(b, cudaStreamSynchronize(b->stream));
                float ms = 0.f;
                BCUDA(b, cudaEventElapsedTime(&ms, b->ev0, b->ev1));
                if (ms < best) { best = ms; bc = c; br = r; }
            }
        if ((rc = kind_set_tiling(b, id, bc, br))) return rc;
        if (k.cost > most) {
            most = k.cost;
            if (cells_out) *cells_out = bc;
            if (rows_out) *rows_out = br;
        }
    }
    b->timed = false;
    return HYPE_OK;
}

int hype_batch_info(const hype_batch *b, int *instances, int *work_items, size_t *bytes_in_use, size_t *budget)
{
    if (!b) return HYPE_ERR_INVALID;
    int n = 0, w = 0;
    for (const Inst &in : b->inst) n += in.used ? 1 : 0;
    for (const Kind &k : b->kinds) w += k.ready ? k.sub[0].nwork : 0;
    if (instances) *instances = n;
    if (work_items) *work_items = w;
    if (bytes_in_use) *bytes_in_use = b->in_use;
    if (budget) *budget = b->budget;
    return HYPE_OK;
}

int hype_batch_last_elapsed_ms(const hype_batch *b, double *ms)
{
    if (!b || !ms) return HYPE_ERR_INVALID;
    *ms = b->last_ms;
    return HYPE_OK;
}

}  // extern "C"
