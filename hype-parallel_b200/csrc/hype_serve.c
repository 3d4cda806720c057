/*
 * hype_serve.c -- the request loop of include/hype_serve.h, in C over the
 * batch ABI (include/hype_batch.h).
 *
 * Initial states are built by a host thread (the stager) into a ring of
 * pinned buffers, each request from its arrival on and in arrival order, its
 * cells filled on several threads (hype_ic.c), while the GPU steps the
 * resident requests; a fill callback (HYPE_IC_CALLBACK) is therefore called
 * from that thread.  One iteration of the loop:
 *   1. admit, in arrival order, every request whose initial state is built
 *      while the batch has a free slot and HBM budget for it (the state is
 *      uploaded and its dt seeded by one RHS evaluation); a request that does
 *      not fit waits at the head of the queue until finished instances free
 *      their memory; the loop waits for the stager only when nothing is
 *      resident;
 *   2. choose which resident requests step (least remaining work first, up
 *      to active_cells cells; the others are held; a small grid takes up to
 *      substep_cells / cells steps per batch step), enqueue k steps of the
 *      batch (k graph replays, k sized so that they take about poll_ms of GPU
 *      time) and wait for them;
 *   3. retire every instance whose time loop ended: copy its state out, hand
 *      it to the sink, free its slot and memory.
 * Instances stop on the device at their own t_final / max_steps, so the k
 * steps of step 2 never overrun a request.
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <cuda_runtime_api.h>
#include "../../include/hype_batch.h"
#include "../../include/hype_ic.h"
#include "../../include/hype_serve.h"

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void sleep_s(double s)
{
    if (s <= 0.0) return;
    struct timespec ts;
    ts.tv_sec = (time_t)s;
    ts.tv_nsec = (long)((s - (double)ts.tv_sec) * 1e9);
    nanosleep(&ts, NULL);
}

static int cmp_double(const void *a, const void *b)
{
    const double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* nearest-rank percentile of sorted v[0..n-1] */
static double pct(const double *v, int n, double p)
{
    if (n <= 0) return 0.0;
    int k = (int)ceil(p / 100.0 * (double)n) - 1;
    if (k < 0) k = 0;
    if (k >= n) k = n - 1;
    return v[k];
}

void hype_serve_config_default(hype_serve_config *c)
{
    if (!c) return;
    memset(c, 0, sizeof(*c));
    c->device = 0;
    c->max_instances = 256;
    c->hbm_budget = 0;
    c->max_cells = 2048LL * 2048LL;
    c->poll_ms = 10.0;
    c->realtime = 1;
    c->autotune = 1;
    c->fetch_results = 1;
    c->active_cells = 4LL << 20;
    c->substep_cells = 0;
}

/* steps per batch step for a grid of `cells` cells: the largest power of two
 * k <= 16 with k * cells <= substep_cells (at least 1) */
static int substeps_for(long long cells, long long substep_cells)
{
    int k = 1;
    while (k < 16 && 2LL * k * cells <= substep_cells) k *= 2;
    return k;
}

typedef struct {
    double work;     /* cells x remaining steps */
    int slot;
    int order;       /* request index: ties go to the earlier arrival */
    long long cells; /* cells stepped per batch step (grid cells x substeps) */
} pick_t;

static int cmp_pick(const void *a, const void *b)
{
    const pick_t *x = (const pick_t *)a, *y = (const pick_t *)b;
    if (x->work != y->work) return x->work < y->work ? -1 : 1;
    return x->order - y->order;
}

/* Least-remaining-work-first: release the resident requests with the least
 * work left until the cells they step per batch step reach `budget`, hold
 * the others. */
static void schedule(hype_batch *b, const hype_request *req, const int *req_of, int M, long long budget, pick_t *tmp)
{
    int n = 0;
    for (int s = 0; s < M; ++s) {
        if (req_of[s] < 0) continue;
        const hype_request *r = &req[req_of[s]];
        hype_instance_status st;
        hype_batch_status(b, s, &st);
        double rem = (double)(r->max_steps - st.steps);
        if (r->t_final < 1e300 && st.dt_next > 0.0) {
            const double by_t = ceil((r->t_final - st.t) / st.dt_next);
            if (by_t < rem) rem = by_t;
        }
        if (rem < 1.0) rem = 1.0;
        const long long cells = (long long)r->cfg.nx * r->cfg.ny;
        tmp[n].cells = cells * (st.substeps > 0 ? st.substeps : 1);
        tmp[n].work = rem * (double)cells;
        tmp[n].slot = s;
        tmp[n].order = req_of[s];
        ++n;
    }
    qsort(tmp, (size_t)n, sizeof(pick_t), cmp_pick);
    long long acc = 0;
    for (int k = 0; k < n; ++k) {
        const int run = (k == 0) || acc < budget;
        if (run) acc += tmp[k].cells;
        hype_batch_hold(b, tmp[k].slot, !run);
    }
}

static int make_initial(const hype_request *r, int index, hype_fill_fn fill, void *ctx, double *U)
{
    switch (r->ic) {
    case HYPE_IC_CALLBACK: return fill ? (fill(ctx, index, r, U) == 0 ? HYPE_OK : HYPE_ERR_INVALID) : HYPE_ERR_INVALID;
    case HYPE_IC_SHOCK_BUBBLE: return hype_ic_shock_bubble(&r->cfg, r->ic_seed, r->ic_param, U);
    case HYPE_IC_BN_DISCS: return hype_ic_bn_discs(&r->cfg, r->ic_seed, U);
    case HYPE_IC_EULER_QUADRANTS: return hype_ic_euler_quadrants(&r->cfg, r->ic_seed, U);
    case HYPE_IC_SMOOTH_VORTEX: return hype_ic_smooth_vortex(&r->cfg, U);
    default: return HYPE_ERR_INVALID;
    }
}

/* the stager: initial states of the requests, in order, from each one's arrival on */
#define NSTAGE 3
typedef struct {
    pthread_t th;
    int started;
    pthread_mutex_t mu;
    pthread_cond_t cv;
    const hype_request *req;
    int n;
    hype_fill_fn fill;
    void *ctx;
    int realtime;
    double t_start;
    long long max_cells;
    double *buf[NSTAGE];
    int req_of[NSTAGE];   /* request index built (or being built) in the buffer; -1: free */
    int ready[NSTAGE];    /* 1: built, status in rc[] */
    int rc[NSTAGE];
    int next;             /* next request to build */
    int stop;
} stager_t;

static void *stager_main(void *a)
{
    stager_t *g = (stager_t *)a;
    pthread_mutex_lock(&g->mu);
    while (!g->stop && g->next < g->n) {
        int k = -1;
        for (int q = 0; q < NSTAGE; ++q)
            if (g->req_of[q] < 0) { k = q; break; }
        const hype_request *r = &g->req[g->next];
        const double wait = g->realtime ? r->arrival_s - (now_s() - g->t_start) : 0.0;
        if (k < 0) {   /* every buffer holds a request not yet admitted */
            pthread_cond_wait(&g->cv, &g->mu);
            continue;
        }
        if (wait > 0.0) {   /* not arrived yet */
            struct timespec ts;
            clock_gettime(CLOCK_REALTIME, &ts);
            const double until = (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec + (wait < 0.05 ? wait : 0.05);
            ts.tv_sec = (time_t)until;
            ts.tv_nsec = (long)((until - (double)ts.tv_sec) * 1e9);
            pthread_cond_timedwait(&g->cv, &g->mu, &ts);
            continue;
        }
        const int i = g->next++;
        g->req_of[k] = i;
        g->ready[k] = 0;
        pthread_mutex_unlock(&g->mu);
        int rc = HYPE_OK;
        if (hype_batch_instance_bytes(&r->cfg) == 0 || (long long)r->cfg.nx * r->cfg.ny > g->max_cells) rc = HYPE_ERR_INVALID;
        else rc = make_initial(r, i, g->fill, g->ctx, g->buf[k]);
        pthread_mutex_lock(&g->mu);
        g->rc[k] = rc;
        g->ready[k] = 1;
        pthread_cond_broadcast(&g->cv);
    }
    pthread_mutex_unlock(&g->mu);
    return NULL;
}

/* the buffer holding request i: -1 if the stager has not reached it; *ready set */
static int stager_find(stager_t *g, int i, int *ready)
{
    for (int q = 0; q < NSTAGE; ++q)
        if (g->req_of[q] == i) { *ready = g->ready[q]; return q; }
    *ready = 0;
    return -1;
}

static void stager_release(stager_t *g, int k)
{
    pthread_mutex_lock(&g->mu);
    g->req_of[k] = -1;
    g->ready[k] = 0;
    pthread_cond_broadcast(&g->cv);
    pthread_mutex_unlock(&g->mu);
}

int hype_serve_run(const hype_serve_config *c, const hype_request *req, int n, hype_fill_fn fill, hype_sink_fn sink,
                   void *ctx, hype_request_result *res, hype_serve_stats *stats)
{
    if (!c || (n > 0 && (!req || !res)) || n < 0 || !stats) return HYPE_ERR_INVALID;
    if (c->max_instances < 1 || c->max_cells < 9 || !(c->poll_ms > 0.0)) return HYPE_ERR_INVALID;
    for (int i = 1; i < n; ++i)
        if (req[i].arrival_s < req[i - 1].arrival_s) return HYPE_ERR_INVALID;
    memset(stats, 0, sizeof(*stats));
    memset(res, 0, sizeof(*res) * (size_t)n);

    hype_batch_config bc;
    hype_batch_config_default(&bc);
    bc.device = c->device;
    bc.max_instances = c->max_instances;
    bc.hbm_budget = c->hbm_budget;
    bc.max_cells = c->max_cells;
    hype_batch *b = NULL;
    int rc = hype_batch_create(&bc, &b);
    if (rc) { hype_batch_destroy(b); return rc; }

    const int M = c->max_instances;
    size_t budget = 0;
    hype_batch_info(b, NULL, NULL, NULL, &budget);
    int *req_of = (int *)malloc(sizeof(int) * (size_t)M);
    pick_t *picks = (pick_t *)malloc(sizeof(pick_t) * (size_t)M);
    /* pinned host staging: initial states in (the stager's ring), final states out */
    stager_t g;
    memset(&g, 0, sizeof(g));
    double *host_out = NULL;
    const size_t hbytes = sizeof(double) * 9 * (size_t)c->max_cells;
    int alloc_ok = req_of && picks && cudaMallocHost((void **)&host_out, hbytes) == cudaSuccess;
    for (int q = 0; q < NSTAGE && alloc_ok; ++q) alloc_ok = cudaMallocHost((void **)&g.buf[q], hbytes) == cudaSuccess;
    if (!alloc_ok) {
        free(req_of);
        free(picks);
        if (host_out) cudaFreeHost(host_out);
        for (int q = 0; q < NSTAGE; ++q)
            if (g.buf[q]) cudaFreeHost(g.buf[q]);
        hype_batch_destroy(b);
        return HYPE_ERR_NOMEM;
    }
    for (int s = 0; s < M; ++s) req_of[s] = -1;

    int next = 0, finished = 0, running = 0;
    int steps_per_poll = 1, tuned_at = 0;
    double ms_per_step = -1.0;
    const double t_start = now_s();
    rc = HYPE_OK;
    g.req = req; g.n = n; g.fill = fill; g.ctx = ctx; g.realtime = c->realtime; g.t_start = t_start;
    g.max_cells = c->max_cells;
    for (int q = 0; q < NSTAGE; ++q) g.req_of[q] = -1;
    pthread_mutex_init(&g.mu, NULL);
    pthread_cond_init(&g.cv, NULL);
    g.started = pthread_create(&g.th, NULL, stager_main, &g) == 0;
    if (!g.started) rc = HYPE_ERR_NOMEM;

    while (rc == HYPE_OK && finished < n) {
        double t = now_s() - t_start;
        /* 1. admission, in arrival order, of requests whose initial state is built */
        int admitted = 0;
        while (next < n && (!c->realtime || req[next].arrival_s <= t)) {
            const hype_request *r = &req[next];
            hype_request_result *o = &res[next];
            const size_t need = hype_batch_instance_bytes(&r->cfg);
            const long long cells = (long long)r->cfg.nx * r->cfg.ny;
            int kbuf = -1, built = 0;
            pthread_mutex_lock(&g.mu);
            kbuf = stager_find(&g, next, &built);
            while (!built && running == 0) {   /* nothing to step meanwhile: wait for the stager */
                pthread_cond_wait(&g.cv, &g.mu);
                kbuf = stager_find(&g, next, &built);
            }
            pthread_mutex_unlock(&g.mu);
            if (!built) break;   /* step the resident requests meanwhile */
            if (need == 0 || cells > c->max_cells) {
                o->status = HYPE_ERR_INVALID;
            } else if (need > budget) {
                o->status = HYPE_ERR_NOMEM;   /* can never be admitted */
            } else {
                int st = g.rc[kbuf];
                int id = -1;
                if (st == HYPE_OK) st = hype_batch_add(b, &r->cfg, g.buf[kbuf], r->t0, r->t_final, r->max_steps, &id);
                if (st == HYPE_ERR_NOMEM || st == HYPE_ERR_BUSY) {
                    if (running > 0) break;   /* wait for retirements; the built state stays staged */
                    st = HYPE_ERR_NOMEM;      /* nothing to wait for: it can never fit */
                }
                if (st == HYPE_OK && c->substep_cells > 0) {
                    const int k = substeps_for(cells, c->substep_cells);
                    if (k > 1) st = hype_batch_set_substeps(b, id, k);
                    if (st != HYPE_OK) hype_batch_remove(b, id);
                }
                if (st == HYPE_OK) {
                    stager_release(&g, kbuf);   /* hype_batch_add has copied it to the device */
                    req_of[id] = next;
                    o->admit_s = now_s() - t_start;
                    ++running;
                    ++admitted;
                    ++next;
                    t = now_s() - t_start;
                    continue;
                }
                o->status = st;
            }
            stager_release(&g, kbuf);
            /* rejected request: finished with an error */
            o->admit_s = o->done_s = now_s() - t_start;
            o->latency_s = o->done_s - (c->realtime ? r->arrival_s : 0.0);
            ++finished;
            ++next;
        }
        if (running == 0) {
            if (next < n && c->realtime) sleep_s(req[next].arrival_s - (now_s() - t_start));
            continue;
        }
        if (admitted) {
            int ninst = 0, nwork = 0;
            size_t bytes = 0;
            hype_batch_info(b, &ninst, &nwork, &bytes, NULL);
            if (ninst > stats->peak_instances) stats->peak_instances = ninst;
            if (bytes > stats->peak_bytes) stats->peak_bytes = bytes;
            if (c->autotune && ninst >= 2 && 2 * ninst >= 3 * (tuned_at > 0 ? tuned_at : 1)) {
                if ((rc = hype_batch_autotune(b, 2, NULL, NULL))) break;
                tuned_at = ninst;
                ms_per_step = -1.0;
            }
            if (ms_per_step < 0.0) steps_per_poll = 1;   /* re-measure the step time */
        }
        if (c->active_cells > 0) schedule(b, req, req_of, M, c->active_cells, picks);
        /* 2. k steps of every released instance */
        if ((rc = hype_batch_advance(b, steps_per_poll))) break;
        if ((rc = hype_batch_sync(b))) break;
        stats->polls++;
        stats->steps_replayed += steps_per_poll;
        double ms = 0.0;
        hype_batch_last_elapsed_ms(b, &ms);
        if (ms > 0.0) {
            const double per = ms / steps_per_poll;
            ms_per_step = ms_per_step < 0.0 ? per : 0.5 * (ms_per_step + per);
            int k = (int)(c->poll_ms / ms_per_step + 0.5);
            steps_per_poll = k < 1 ? 1 : (k > 64 ? 64 : k);
        }
        /* 3. retire finished instances */
        for (int s = 0; s < M; ++s) {
            if (req_of[s] < 0) continue;
            hype_instance_status is;
            hype_batch_status(b, s, &is);
            if (!is.done && is.status == HYPE_OK) continue;
            const int i = req_of[s];
            hype_request_result *o = &res[i];
            o->status = is.status;
            o->steps = is.steps;
            o->t_end = is.t;
            if (c->fetch_results || sink) {
                const int st = hype_batch_get_state(b, s, host_out);
                if (st != HYPE_OK && o->status == HYPE_OK) o->status = st;
            }
            o->done_s = now_s() - t_start;
            o->latency_s = o->done_s - (c->realtime ? req[i].arrival_s : 0.0);
            if (sink) sink(ctx, i, &req[i], host_out, o);
            if (o->status == HYPE_OK) stats->cell_updates += (double)req[i].cfg.nx * req[i].cfg.ny * is.steps;
            hype_batch_remove(b, s);
            req_of[s] = -1;
            --running;
            ++finished;
        }
    }
    const double t_end = now_s() - t_start;
    if (g.started) {
        pthread_mutex_lock(&g.mu);
        g.stop = 1;
        pthread_cond_broadcast(&g.cv);
        pthread_mutex_unlock(&g.mu);
        pthread_join(g.th, NULL);
    }
    pthread_cond_destroy(&g.cv);
    pthread_mutex_destroy(&g.mu);

    /* statistics over the finished requests */
    double *lat = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *que = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    int m = 0;
    double sum = 0.0, first = n > 0 && c->realtime ? req[0].arrival_s : 0.0;
    for (int i = 0; i < n && lat && que; ++i) {
        if (res[i].status == HYPE_OK) stats->completed++;
        else stats->failed++;
        if (res[i].done_s <= 0.0 && res[i].status == HYPE_OK) continue;   /* never ran (loop stopped) */
        lat[m] = res[i].latency_s;
        que[m] = res[i].admit_s - (c->realtime ? req[i].arrival_s : 0.0);
        sum += lat[m];
        ++m;
    }
    if (lat && que && m > 0) {
        qsort(lat, (size_t)m, sizeof(double), cmp_double);
        qsort(que, (size_t)m, sizeof(double), cmp_double);
        stats->p50_s = pct(lat, m, 50);
        stats->p90_s = pct(lat, m, 90);
        stats->p99_s = pct(lat, m, 99);
        stats->max_s = lat[m - 1];
        stats->mean_s = sum / m;
        stats->queue_p50_s = pct(que, m, 50);
        stats->queue_p99_s = pct(que, m, 99);
    }
    stats->wall_s = t_end - first;
    stats->cell_updates_per_s = stats->wall_s > 0.0 ? stats->cell_updates / stats->wall_s : 0.0;
    free(lat);
    free(que);
    free(req_of);
    free(picks);
    for (int q = 0; q < NSTAGE; ++q) cudaFreeHost(g.buf[q]);
    cudaFreeHost(host_out);
    hype_batch_destroy(b);
    return rc;
}
