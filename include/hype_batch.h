/*
 * hype_batch.h -- many independent HyPE-2D runs stepped together on one GPU.
 *
 * No counterpart in the reference: HyPE-2D runs one grid per MPI job (one
 * DMDA, one TS; hype.c:56-396).  A batch holds instances -- each one a grid,
 * a state and its own time loop (t, dt, t_final, max_steps, step count) with
 * exactly the arithmetic of a lone hype_solver of the same configuration --
 * and advances all of them with one persistent stage-kernel launch per RK
 * stage and per kind of instance, over a device work-list of (instance, tile)
 * items sorted longest first.  A whole step of the batch is one CUDA graph;
 * in it an instance takes one step, or several (hype_batch_set_substeps).
 * Every configuration a solver takes is an instance kind: the FP64 primitive
 * and conservative paths (HYPE_FLAG_CONSERVATIVE), the VISCOUS build
 * (HYPE_FLAG_VISCOUS) and mixed precision.
 *
 * Instances join and leave between steps (continuous batching): the work-list,
 * member lists and per-instance parameters live in device memory, so adding or
 * removing an instance re-captures nothing unless the set of instance kinds
 * changes.  Each instance stops on its own at its t_final or max_steps; its
 * tiles then cost one flag read per stage until it is removed.
 *
 * Admission is bounded by an HBM budget: hype_batch_add refuses with
 * HYPE_ERR_NOMEM (nothing changed) when the instance's device bytes would
 * take the batch over the budget, and with HYPE_ERR_BUSY when every slot is
 * taken.  Device memory comes from a stream-ordered pool owned by the batch,
 * so joins and leaves never synchronise the device.
 *
 * All calls on one batch must come from one thread at a time.
 */
#ifndef HYPE_BATCH_H
#define HYPE_BATCH_H

#include <stddef.h>
#include "hype_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hype_batch hype_batch;

typedef struct {
    int device;             /* CUDA device ordinal                                        */
    int max_instances;      /* slots; instance ids are 0 .. max_instances-1                */
    size_t hbm_budget;      /* device bytes the instances may hold; 0 = 80% of the free
                               memory at creation                                         */
    long long max_cells;    /* largest nx*ny of an instance (sizes the staging buffer)    */
} hype_batch_config;

typedef struct {
    int active;             /* slot holds an instance                                     */
    int done;               /* the instance reached t_final or max_steps                  */
    int steps;              /* steps taken                                                */
    int status;             /* HYPE_OK, or HYPE_ERR_INADMISSIBLE / HYPE_ERR_TIMEOUT raised
                               by this instance's stages                                  */
    double t;               /* time reached                                               */
    double dt_next;         /* dt the last RHS proposed (Ctx->dt)                         */
    int held;               /* hype_batch_hold is in force                                */
    int substeps;           /* steps it takes per batch step                              */
} hype_instance_status;

/* max_instances 256, budget 0 (80% of free), max_cells 2048*2048, device 0 */
HYPE_API void hype_batch_config_default(hype_batch_config *c);

HYPE_API int hype_batch_create(const hype_batch_config *c, hype_batch **out);
HYPE_API int hype_batch_destroy(hype_batch *b);
HYPE_API const char *hype_batch_last_error(const hype_batch *b);

/* Device bytes an instance of this configuration holds in a batch (what the
 * admission test charges); 0 for an invalid configuration. */
HYPE_API size_t hype_batch_instance_bytes(const hype_config *cfg);

/*
 * Adds an instance: validates cfg as hype_create does, copies the initial
 * state U0 (host, Vec layout of hype_gpu.h), evaluates the RHS of U0 once to
 * seed dt (hype.c:343) and sets its time loop to (t0, t_final, max_steps).
 * cfg->device is ignored (the batch's device is used).  On success *id is the
 * instance's slot.  Waits for the batch's queued work first.
 */
HYPE_API int hype_batch_add(hype_batch *b, const hype_config *cfg, const double *U0, double t0, double t_final,
                            int max_steps, int *id);

/* Frees an instance's slot and device memory (stream-ordered). */
HYPE_API int hype_batch_remove(hype_batch *b, int id);

/* Enqueues nsteps steps of every instance (nsteps graph replays); returns
 * without waiting.  Instances that are done are skipped on the device. */
HYPE_API int hype_batch_advance(hype_batch *b, int nsteps);

/* Waits for the queued steps and reads every instance's time-loop scalars
 * (one device-to-host copy); the wall time of the last hype_batch_advance
 * span is then available from hype_batch_last_elapsed_ms. */
HYPE_API int hype_batch_sync(hype_batch *b);

/* Status of an instance as of the last hype_batch_sync (or add). */
HYPE_API int hype_batch_status(const hype_batch *b, int id, hype_instance_status *st);

/* Holds (hold = 1) or releases an instance: a held instance keeps its state
 * and time loop but takes no steps, and its tiles cost one flag read per
 * stage -- a scheduler's way to give the GPU to other instances first.  Takes
 * effect from the next hype_batch_advance. */
HYPE_API int hype_batch_hold(hype_batch *b, int id, int hold);

/* Steps an instance takes per batch step (1..16, default 1): a small grid
 * can take several steps while a large one takes one, so that small, long
 * runs are not paced by the largest member.  Each step is still the
 * instance's own step, with its own dt and stop tests (an instance never
 * overruns its t_final or max_steps).  Takes effect from the next advance. */
HYPE_API int hype_batch_set_substeps(hype_batch *b, int id, int substeps);

/* Copies an instance's state out (host, Vec layout); waits for queued work. */
HYPE_API int hype_batch_get_state(hype_batch *b, int id, double *U);

/*
 * Tile shape of the persistent launches: tile width `cells` (64 or 128
 * columns) and about `rows` rows per tile (16..1024), applied to every
 * instance kind (the conservative and viscous kinds keep 128 columns).
 * Rebuilds the work-list and the step graph.
 */
HYPE_API int hype_batch_set_tiling(hype_batch *b, int cells, int rows);

/*
 * Autotuner: times the first stage of a step over the current instances
 * (inputs untouched, reps launches per candidate) for every tile width in
 * {64, 128} and rows per tile in {16, 32, 64, 128}, per instance kind, and
 * keeps the fastest; reports the choice of the kind with the most work.
 */
HYPE_API int hype_batch_autotune(hype_batch *b, int reps, int *cells, int *rows);

/* Instances held, work items per stage launch (all kinds), device bytes held,
 * the admission budget. */
HYPE_API int hype_batch_info(const hype_batch *b, int *instances, int *work_items, size_t *bytes_in_use, size_t *budget);

HYPE_API int hype_batch_last_elapsed_ms(const hype_batch *b, double *ms);

#ifdef __cplusplus
}
#endif
#endif
