/*
 * hype_group.h -- one grid split into y-slabs on one or more GPUs of one process.
 *
 * This replaces HyPE-2D's DMDA domain decomposition across MPI ranks.  The
 * reference creates the grid with DMDACreate2d (hype.c:108-122, ghost width 3,
 * BOX stencil, PETSC_DECIDE ranks), refreshes the ghost rows of every rank with
 * DMGlobalToLocalBegin/End before each RHS (rhs_function_prim.c:44-45), and takes
 * the time step as the MPI_Allreduce(MIN) of the ranks' dt
 * (rhs_function_prim.c:620-623).
 *
 * Here slab k holds global rows row0_k .. row0_k+rows_k-1.  Like PETSc's split,
 * the first ny % nslabs slabs get one row more.  Each slab keeps 3 halo rows on
 * each side where it has a neighbour.  The stage kernel that produces a state
 * stores the slab's 3 edge rows into its neighbours' halo rows in the same
 * launch; these are peer stores over NVLink when the neighbour is on another
 * GPU.  Per-stage event dependencies on the two neighbours replace the halo
 * exchange.  After each step's last stage, one kernel takes the maximum wave
 * speed over all slabs and gives every slab the same dt.  The result equals a
 * single solver's on the same grid bit for bit: t, the step count and the state.
 * Every form of the single solver: FP64 (primitive, conservative and viscous
 * paths, N = 0..3) and mixed precision, whose stage kernel stores the edge rows
 * into the neighbours' FP32 and FP64 planes the same way.
 *
 * Calls return HYPE_OK or an HYPE_ERR_* code of hype_gpu.h, with the message in
 * hype_group_last_error.
 */
#ifndef HYPE_GROUP_H
#define HYPE_GROUP_H

#include "hype_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hype_group hype_group;

/* `cfg` describes the whole grid.  nslabs is 1..ny/3 (a slab has at least the
 * 3 rows a neighbour's stencil reads).  Slab k runs on devices[k]; with
 * devices NULL, every slab runs on cfg->device.  Slabs on different GPUs need
 * peer access between them.  On error *out may still be set: read the message
 * with hype_group_last_error, then destroy it. */
HYPE_API int hype_group_create(const hype_config *cfg, int nslabs, const int *devices, hype_group **out);
HYPE_API int hype_group_destroy(hype_group *g);
HYPE_API const char *hype_group_last_error(const hype_group *g);
/* rows of slab k: global rows *row0 .. *row0 + *rows - 1, on *device */
HYPE_API int hype_group_slab(const hype_group *g, int k, int *row0, int *rows, int *device);

/* the whole grid's interleaved state (hype_gpu.h layout), to and from the slabs */
HYPE_API int hype_group_set_state(hype_group *g, const double *U);
HYPE_API int hype_group_get_state(hype_group *g, double *U);

/* The time loop, as hype_begin / hype_advance / hype_wait / hype_solve. One
 * step is one CUDA graph over all slabs. */
HYPE_API int hype_group_begin(hype_group *g, double t0, double t_final, int max_steps);
HYPE_API int hype_group_advance(hype_group *g, int nsteps);
HYPE_API int hype_group_wait(hype_group *g, int *steps_done, double *t_end, double *dt_next);
HYPE_API int hype_group_solve(hype_group *g, double t0, double t_final, int max_steps, int *steps_done, double *t_end,
                     double *dt_next);
/* device time of the last hype_group_advance, in ms, from events on slab 0's stream */
HYPE_API int hype_group_last_elapsed_ms(const hype_group *g, double *ms);

#ifdef __cplusplus
}
#endif
#endif
