/*
 * hype_serve.h -- a request loop over a batch (hype_batch.h): solves arrive
 * over time, are admitted while slots and the HBM budget allow, run together
 * with everything else resident on the GPU (continuous batching: a request
 * that arrives while others are stepping joins them between two steps), and
 * leave the moment their own time loop ends.  Reports per-request
 * time-to-solution and the run's p50/p99 and aggregate cell-updates/s.
 *
 * No counterpart in the reference (HyPE-2D solves one problem per job).
 * Plain C.  The loop runs on the calling thread and returns when every
 * request has finished or failed.
 */
#ifndef HYPE_SERVE_H
#define HYPE_SERVE_H

#include <stddef.h>
#include <stdint.h>
#include "hype_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Built-in seeded initial states (hype_ic.h); HYPE_IC_CALLBACK asks fill(). */
#define HYPE_IC_CALLBACK         0
#define HYPE_IC_SHOCK_BUBBLE     1   /* Kapila; ic_param = bubble count */
#define HYPE_IC_BN_DISCS         2   /* Baer-Nunziato */
#define HYPE_IC_EULER_QUADRANTS  3   /* Euler */
#define HYPE_IC_SMOOTH_VORTEX    4   /* Kapila (kapila_5eqn.c:527-562) */

typedef struct {
    double arrival_s;        /* seconds after the start of the run; non-decreasing */
    hype_config cfg;         /* system, order, grid, EOS, boundaries, precision   */
    double t0, t_final;      /* time interval of the solve                          */
    int max_steps;           /* step limit of the solve                             */
    int ic;                  /* HYPE_IC_*                                           */
    uint64_t ic_seed;
    int ic_param;
} hype_request;

typedef struct {
    int status;              /* HYPE_OK, or why the request failed                  */
    int steps;               /* steps taken                                         */
    double t_end;            /* time reached                                        */
    double admit_s;          /* when it joined the batch (run clock)                */
    double done_s;           /* when its result was on the host (run clock)         */
    double latency_s;        /* time-to-solution: done_s - arrival_s                */
} hype_request_result;

typedef struct {
    int device;
    int max_instances;       /* slots of the batch                                  */
    size_t hbm_budget;       /* device bytes of resident state; 0 = 80% of free    */
    long long max_cells;     /* largest grid accepted                               */
    double poll_ms;          /* target GPU time between two polls of the batch      */
    int realtime;            /* 1: a request is visible from its arrival time on;
                                0: every request is queued at the start             */
    int autotune;            /* 1: retune the tile shape when the batch has grown
                                by half since the last tuning                        */
    int fetch_results;       /* 1: copy each final state to the host (sink or not)  */
    long long active_cells;  /* scheduling: each poll, resident requests step in order
                                of least remaining work (cells x steps left) until
                                their cells reach this many; the rest are held.
                                0 = every resident request steps (processor sharing) */
    long long substep_cells; /* a request of c cells takes up to substep_cells / c steps
                                (a power of two, 1..16) per batch step, so small grids
                                are not paced by large ones; 0 = one step each        */
} hype_serve_config;

typedef struct {
    int completed;           /* finished with HYPE_OK                                */
    int failed;
    double wall_s;           /* first arrival .. last result                         */
    double p50_s, p90_s, p99_s, max_s, mean_s;   /* time-to-solution, all requests    */
    double queue_p50_s, queue_p99_s;             /* arrival .. admission              */
    double cell_updates;     /* sum of nx * ny * steps                                */
    double cell_updates_per_s;                   /* cell_updates / wall_s             */
    int peak_instances;
    size_t peak_bytes;
    long long polls;
    long long steps_replayed;                    /* batch steps (graph replays)       */
} hype_serve_stats;

/* Fills U0 (Vec layout, nx*ny*nvar doubles) for request `index`; returns 0 on success. */
typedef int (*hype_fill_fn)(void *ctx, int index, const hype_request *req, double *U0);
/* Receives request `index`'s final state (valid during the call only). */
typedef void (*hype_sink_fn)(void *ctx, int index, const hype_request *req, const double *U, const hype_request_result *res);

/* device 0, 256 slots, budget 0, max_cells 2048*2048, poll 10 ms, realtime, autotune, fetch,
 * active_cells 4*2^20, substep_cells 0 */
HYPE_API void hype_serve_config_default(hype_serve_config *c);

/*
 * Runs the requests.  res (n entries) and stats are written; fill is needed
 * only for HYPE_IC_CALLBACK requests; sink may be NULL.  Returns HYPE_OK when
 * the loop ran (individual failures are in res[i].status), or an error that
 * stopped it.
 */
HYPE_API int hype_serve_run(const hype_serve_config *c, const hype_request *req, int n, hype_fill_fn fill,
                            hype_sink_fn sink, void *ctx, hype_request_result *res, hype_serve_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
