/*
 * hype_gpu.h -- C ABI of hype-parallel_b200, a B200 (sm_100a) implementation of
 * HyPE-2D's right-hand-side evaluation and explicit SSP-RK time step for the
 * Euler, Kapila five-equation and Baer-Nunziato systems.
 *
 * Plain C: pointers, sizes and status codes only; no PETSc and no CUDA types.
 * Every entry point returns HYPE_OK (0) or a HYPE_ERR_* code; hype_last_error()
 * gives the message of the last failure on a solver.
 *
 * State arrays crossing this boundary have the layout of the reference's
 * global Vec (HyPE-2D/hype.h:68-70, Field{comp[nVar]} indexed u[j][i]):
 * nx*ny cells, row-major (i fastest), nvar doubles interleaved per cell.
 * Component orders are the reference's:
 *   Euler   [rho, rho u, rho v, E]                                  euler.c:14-38
 *   Kapila  [a1 rho1, a2 rho2, rho u, rho v, E, a1]                  kapila_5eqn.c:14-61
 *   BN      [a1 r1, a1 r1 u1, a1 r1 v1, a1 E1, a2 r2, a2 r2 u2,
 *            a2 r2 v2, a2 E2, a1]                                    baer_nunziato.c:14-60
 */
#ifndef HYPE_GPU_H
#define HYPE_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define HYPE_API __attribute__((visibility("default")))
#else
#define HYPE_API
#endif

/* ---- status codes -------------------------------------------------------- */
#define HYPE_OK                0
#define HYPE_ERR_INVALID       1   /* bad argument or unsupported configuration            */
#define HYPE_ERR_CUDA          2   /* CUDA runtime or driver error                          */
#define HYPE_ERR_INADMISSIBLE  3   /* a face state failed the flux admissibility test; the
                                      reference calls MPI_Abort there (kapila_5eqn.c:353-357,
                                      baer_nunziato.c:281-303, euler.c:212-222)              */
#define HYPE_ERR_TIMEOUT       4   /* a bounded device wait expired                          */
#define HYPE_ERR_NOMEM         5   /* device memory (or the admission budget) exhausted      */
#define HYPE_ERR_NO_DEVICE     6   /* no CUDA device / not an sm_100 device                  */
#define HYPE_ERR_BUSY          7   /* operation needs the solver idle                        */

/* ---- PDE systems: the compile-time #define of HyPE-2D/hype.h:33-35 --------- */
#define HYPE_EULER          0
#define HYPE_KAPILA_5EQN    1
#define HYPE_BAER_NUNZIATO  2

/* ---- boundary types: values of HyPE-2D/hype.h:76 enum bndry_type ------------ */
#define HYPE_BC_WALL          0   /* rejected: the reference never fills its ghosts      */
#define HYPE_BC_INLET         1   /* left boundary, Kapila only (InletBCPrim)            */
#define HYPE_BC_PERIODIC      2
#define HYPE_BC_REFLECTIVE    3
#define HYPE_BC_TRANSMISSIVE  4

/* ---- arithmetic ---------------------------------------------------------- */
#define HYPE_PREC_FP64   0    /* bit-compatible with the reference's C          */
#define HYPE_PREC_MIXED  1    /* FP32 state/reconstruction/flux, FP64 EOS and totals */
#define HYPE_PREC_FP64_FAST 2 /* FP64 with fused multiply-adds and shared reciprocals:
                                 within 1e-12 relative L-infinity (per field, of the
                                 field's largest value) of the reference per RHS call;
                                 primitive inviscid path (no HYPE_FLAG_CONSERVATIVE or
                                 HYPE_FLAG_VISCOUS), single solvers and slab groups    */

/* ---- flags --------------------------------------------------------------- */
#define HYPE_FLAG_BN_FIX_P2   1u  /* Baer-Nunziato: take the phase-2 flux pressure from V[7]
                                     instead of V[8] (baer_nunziato.c:271 reads alpha_1)   */
#define HYPE_FLAG_CONSERVATIVE 2u /* reconstruct conserved variables: the RHS is HyPE-2D's
                                     RHSFunction (rhs_function.c:12-625), which hype.c uses
                                     when Ctx.ReconsPrimitive is false (hype.c:341-352).
                                     FP64 solvers only (not mixed, batch or no-alloc).      */
#define HYPE_FLAG_VISCOUS     4u  /* the reference's VISCOUS build (hype.h:36, off there by
                                     default): viscous face fluxes with viscosities mu1/mu2
                                     (rhs_function_prim.c:356-374, riemann.c:146-186,
                                     kapila_5eqn.c:119-158, 377-411) and the viscous dt.
                                     Kapila, N = 1..3, FP64 solvers only.                    */

/*
 * Run-time form of the reference's compile-time and AppCtx parameters:
 *   system                 hype.h:33-35 (#define KAPILA_5EQN ...)
 *   order                  AppCtx.N (hype.c:32): 0..3; selects WENO degree,
 *                          quadrature and SSP scheme (hype.c:59-68, 362-382)
 *   nx, ny, x/y min/max    AppCtx.N_x, N_y, x_min ... (hype.c:33-38); h = (x_max-x_min)/nx
 *   cfl                    AppCtx.CFL
 *   bc_*                   AppCtx.LeftBoundary ... (hype.c:46-49)
 *   gamma1..pi2            GAMMA_1, GAMMA_2, PI_1, PI_2 (hype.h:42-45)
 *   mu1, mu2               MU_1, MU_2 (hype.h:46-47), with HYPE_FLAG_VISCOUS
 */
typedef struct {
    int system;
    int order;
    int nx, ny;
    double x_min, x_max, y_min, y_max;
    double cfl;
    int bc_left, bc_right, bc_bottom, bc_top;
    double gamma1, gamma2, pi1, pi2;
    int precision;
    unsigned flags;
    int device;           /* CUDA device ordinal */
    double mu1, mu2;      /* MU_1, MU_2 (hype.h:46-47): phase viscosities, read with HYPE_FLAG_VISCOUS */
} hype_config;

typedef struct hype_solver hype_solver;

/* Fills *cfg with the defaults of HyPE-2D/hype.c:32-50 and hype.h:42-45. */
HYPE_API void hype_config_default(hype_config *cfg);

/* Number of conserved variables of a system (nVar, hype.h:37): 4, 6 or 9; 0 if unknown. */
HYPE_API int hype_nvar(int system);

/* Human-readable name of a status code. */
HYPE_API const char *hype_status_string(int status);

/*
 * Creates a solver: validates cfg, allocates the device state (three stage
 * buffers of nx*ny*nvar doubles plus staging), builds the TMA descriptors.
 * Replaces the set-up half of HyPE-2D/hype.c:56-309 (DMDA, work Vecs, scratch
 * arrays u_bnd/F/G/D/E, quadrature and basis tables).
 */
HYPE_API int hype_create(const hype_config *cfg, hype_solver **out);
HYPE_API int hype_destroy(hype_solver *s);
HYPE_API const char *hype_last_error(const hype_solver *s);

/*
 * Drop-in for RHSFunctionPrim (HyPE-2D/rhs_function_prim.c:12-626, declared at
 * hype.h:306): RHS = L(U) over all cells and *dt = CFL*h/(2*s_max), the value
 * the reference leaves in Ctx->dt (rhs_function_prim.c:620-623).  U and RHS are
 * host arrays in the Vec layout above.  t is accepted for the TS signature (the
 * inlet profile is time independent).  Thread-compatible, not reentrant on one
 * solver (as the reference, which shares AppCtx scratch).  The copies overlap the
 * launch, band of rows by band of rows.  Pinned (page-locked) U and RHS go to the
 * copy engines directly; pageable ones (PETSc's Vec arrays) are staged through
 * two pinned buffers of the state's size that the solver allocates on first use
 * (direct copies if that allocation fails), copied by the calling thread and a
 * pool of three host threads that the library starts on the first such copy (one
 * pool per process; the threads idle between copies and end with the process).
 * The same holds for hype_rhs_prim_slab, hype_advance_host, hype_set_state and
 * hype_get_state.
 */
HYPE_API int hype_rhs_prim(hype_solver *s, double t, const double *U, double *RHS, double *dt);

/* Same with U and RHS in device memory of the solver's device (e.g. a PETSc
 * VECCUDA array); the call is synchronous. */
HYPE_API int hype_rhs_prim_device(hype_solver *s, double t, const double *dU, double *dRHS, double *dt);

/* One MPI rank's share of a grid decomposed over ranks in y: HyPE-2D's DMDA
 * (hype.c:108-122) with one rank across x.  The solver owns global rows
 * row0 .. row0+rows-1 of the grid `cfg` describes (nx, ny, domain and boundaries of
 * the whole grid).  A side with a neighbouring rank (row0 > 0, row0+rows < ny, or a
 * periodic y axis when the slab is not the whole grid) takes its 3 ghost rows from
 * the caller instead of a boundary condition.  FP64 or mixed precision. */
HYPE_API int hype_create_slab(const hype_config *cfg, int row0, int rows, hype_solver **out);

/* One MPI rank's block of a grid decomposed over ranks in x and y: HyPE-2D's DMDA
 * as hype.c:108-122 creates it (PETSC_DECIDE x PETSC_DECIDE ranks, BOX stencil,
 * ghost width 3).  The solver owns global columns col0 .. col0+cols-1 and rows
 * row0 .. row0+rows-1 of the grid `cfg` describes (the whole grid's nx, ny, domain
 * and boundaries); cols, rows >= 3.  A side with a neighbouring rank (an inner
 * edge, or a periodic axis the block does not span) takes its 3 ghost rows or
 * columns, corners included, from the caller instead of a boundary condition.
 * With cols == nx this is hype_create_slab.  A block split in x takes an FP64
 * precision (HYPE_ERR_INVALID for mixed precision). */
HYPE_API int hype_create_block(const hype_config *cfg, int col0, int cols, int row0, int rows, hype_solver **out);

/* RHSFunctionPrim (or RHSFunction) on a slab or block: rhs_function_prim.c:12-626
 * for one rank.  U points at the block's cell (0, 0) in a host array whose rows
 * are row_stride doubles apart: cols*nvar for a compact array, or the ghosted width
 * times nvar for a DMDA local vector after DMGlobalToLocal.  Rows -3..-1 and
 * rows..rows+2, and columns -3..-1 and cols..cols+2, are read on the sides with a
 * neighbour; other ghost cells are never read.  RHS receives the block's cells,
 * compact.  *dt is this block's CFL h / (2 s_max); the caller takes the minimum
 * over ranks, as rhs_function_prim.c:620-623 does with MPI_Allreduce(MIN). */
HYPE_API int hype_rhs_prim_slab(hype_solver *s, double t, const double *U, long long row_stride, double *RHS, double *dt);

/*
 * RHSFunctionPrim for callers that cannot allocate device memory -- for
 * example a plug-in running inside an application or framework whose memory
 * pool already owns the GPU, or a time loop that must not pay the device-wide
 * synchronisation of cudaMalloc/cudaFree.  No counterpart in the reference
 * (HyPE-2D allocates its scratch in main, hype.c:237-251); it has the meaning
 * of hype_rhs_prim_device but needs no solver object and calls no allocator.
 *
 * dU and dRHS are device arrays in the Vec layout (caller-owned).  All working
 * memory is one static device array of HYPE_NOALLOC_MAX_BYTES, held by every
 * GPU that loads this library until the process exits: the grid must satisfy
 * 256 + ceil16(nx) * ny * nvar * 8 <= HYPE_NOALLOC_MAX_BYTES (Kapila up to
 * about 590 x 590 cells), else HYPE_ERR_NOMEM is returned before any device
 * work.  FP64 only; periodic, reflective and transmissive boundaries only
 * (HYPE_ERR_INVALID otherwise).  Runs on the legacy default stream and returns
 * when the result is in dRHS; a dU written on a stream created with
 * cudaStreamNonBlocking is not ordered before that stream, so synchronise such
 * a stream first.  Each call looks up the array's device address (no
 * allocation); the first call on a device loads the module there and should
 * come before any stream capture.  Calls share the array: calls that overlap
 * on the GPU race and must be serialised by the caller.
 */
#define HYPE_NOALLOC_MAX_BYTES (16u * 1024u * 1024u)
HYPE_API int hype_rhs_prim_noalloc(const hype_config *cfg, double t, const double *dU, double *dRHS, double *dt);

/* Device-resident state: copy in / out (Vec layout, host memory).  Setting the
 * state keeps the time-loop scalars (t, dt, step count) of hype_begin; call
 * hype_begin again to restart the loop from a new initial state. */
HYPE_API int hype_set_state(hype_solver *s, const double *U);
HYPE_API int hype_get_state(hype_solver *s, double *U);

/* Primitive variables of the device state (Vec layout, host memory): what
 * ComputePrimitiveVariables leaves in Ctx->W (post_process.c:165-200). */
HYPE_API int hype_get_primitive(hype_solver *s, double *W);

/* The solver's configuration. */
HYPE_API int hype_solver_config(const hype_solver *s, hype_config *cfg);

/*
 * The reference's files, from and into the device state:
 *   hype_write_restart  PETSc binary Vec of the conserved state -- big-endian
 *                       class id 1211214, length, the doubles in Vec order --
 *                       as VecView(U) writes restart1/2.bin (post_process.c:47-64),
 *                       plus the viewer's "<path>.info" (-vecload_block_size nVar);
 *   hype_read_restart   VecLoad of such a file into the state (hype.c:316-325);
 *                       the grid must match (HYPE_ERR_INVALID otherwise);
 *   hype_write_vts      VTK XML structured grid of the primitive variables with
 *                       the DMDA's cell-centre coordinates and field names, as
 *                       sol-%08d.vts (post_process.c:25-45, hype.c:388-399), the
 *                       file HyPE-2D/plot.py reads.
 */
HYPE_API int hype_write_restart(hype_solver *s, const char *path);
HYPE_API int hype_read_restart(hype_solver *s, const char *path);
HYPE_API int hype_write_vts(hype_solver *s, const char *path);

/*
 * hype_solve with the reference's output schedule: the files MonitorFunction
 * writes (post_process.c:12-64) -- sol-%08d.vts every write_interval steps
 * (step 0 included), restart1.bin when step % restart_interval == 0 and
 * restart2.bin when (step + 7) % restart_interval == 0 -- and the final
 * sol-%08d.vts of hype.c:386-399, into directory `dir` (NULL: the current
 * one).  An interval of 0 writes nothing of that kind.
 */
HYPE_API int hype_solve_monitored(hype_solver *s, double t0, double t_final, int max_steps, int write_interval,
                                  int restart_interval, const char *dir, int *steps_done, double *t_end, double *dt_next);

/*
 * The time loop of HyPE-2D/hype.c:337-384 on the device-resident state: one
 * RHS call at t0 seeds dt (hype.c:343, 356), then SSP-RK steps (N=0 forward
 * Euler, N=1 SSPRKS2 two stages, N=2 SSPRKS3 four stages, N=3 SSPRK(10,4);
 * hype.c:362-382) until t_final (last step clipped, TS_EXACTFINALTIME_MATCHSTEP)
 * or max_steps; each step's dt is the CFL dt of the previous step's last RHS
 * call (MonitorFunction, post_process.c:19).  Outputs may be NULL.
 */
HYPE_API int hype_solve(hype_solver *s, double t0, double t_final, int max_steps,
               int *steps_done, double *t_end, double *dt_next);

/* Split form of hype_solve for callers that overlap host work:
 * hype_begin seeds dt; hype_advance enqueues up to nsteps steps (CUDA graph
 * replays, asynchronous); hype_wait blocks and reports progress and errors. */
HYPE_API int hype_begin(hype_solver *s, double t0, double t_final, int max_steps);
HYPE_API int hype_advance(hype_solver *s, int nsteps);
HYPE_API int hype_wait(hype_solver *s, int *steps_done, double *t_end, double *dt_next);

/*
 * Host state in, n steps, host state out: hype_set_state(U_in) +
 * hype_advance(nsteps) + hype_wait + hype_get_state(U_out), with the copies
 * overlapped by the computation -- the rows of U_in stream in while the first
 * step's stages run, band of rows by band of rows, on the rows already there,
 * and the rows of U_out stream out while the last step finishes the rows after
 * them.  Needs hype_begin.  U_in
 * and U_out may be the same array; pinned (page-locked) host memory gives the
 * overlap its full effect (pageable arrays: see hype_rhs_prim).  Returns what
 * hype_wait returns.
 */
HYPE_API int hype_advance_host(hype_solver *s, const double *U_in, double *U_out, int nsteps, int *steps_done, double *t_end,
                               double *dt_next);

/* Sums of each conserved variable over the cells (times h^2 when scaled != 0),
 * computed on the device in FP64 with a fixed reduction order; totals has nvar
 * entries.  Also reports min/max of the volume fraction (Kapila, BN). */
HYPE_API int hype_totals(hype_solver *s, int scaled, double *totals, double *alpha_min, double *alpha_max);

/* Launch geometry of the stage kernel chosen for this grid (for reports). */
HYPE_API int hype_launch_info(const hype_solver *s, int *grid_x, int *grid_y, int *threads, size_t *smem_bytes,
                     int *blocks_per_sm);

/* Average device time of one stage-kernel launch (an SSP-RK stage u + dt/2 L(u)
 * over the device state, dt negligible so the state is unchanged to rounding),
 * over `reps` launches timed with CUDA events on the solver's stream. */
HYPE_API int hype_time_stage(hype_solver *s, int reps, double *ms_per_launch);

/* Autotuner: times the stage kernel (hype_time_stage, `reps` launches each) for
 * every tile shape -- tile width 64 or 128 columns, 1, 2 or 4 waves of row runs
 * -- on the solver's current state and keeps the fastest.  Results are
 * unchanged by the choice (bit for bit).  Call before hype_begin or between
 * steps; reports the chosen width and wave count. */
HYPE_API int hype_autotune(hype_solver *s, int reps, int *cells, int *waves);

/* Device time of the last hype_solve/hype_wait interval, in milliseconds
 * (CUDA events around the step replays). */
HYPE_API int hype_last_elapsed_ms(const hype_solver *s, double *ms);

/* The FP64 roofline of the bit-exact kernels, measured on `device`: the rate of
 * separately rounded FP64 multiplies and adds (the kernels are built without
 * FMA contraction), from a short kernel of independent multiply-add chains on
 * every SM, best of `reps` launches timed with CUDA events.  *ops_per_s counts
 * one per multiply and one per add. */
HYPE_API int hype_fp64_rate(int device, int reps, double *ops_per_s);

/* The FP64 roofline of the performance form (HYPE_PREC_FP64_FAST), which fuses
 * multiplies and adds: the same measurement with one fused multiply-add per
 * chain link, counted as two FLOPs. */
HYPE_API int hype_fp64_fma_rate(int device, int reps, double *flops_per_s);

/*
 * Test hook for the error path of the bounded device waits; no counterpart in
 * the reference.  With row >= 0 the stage kernels of this solver issue no TMA
 * row load for rows >= row, so the wait for that row runs out (after about 2 s
 * of GPU time per wave of blocks): the block waits for the loads it did issue,
 * raises the timeout bit and returns, and the call reports HYPE_ERR_TIMEOUT
 * with the context still usable.  row < 0 restores normal operation.  Waits
 * for the solver's stream first and drops its captured step graph.
 */
HYPE_API int hype_test_skip_row_loads(hype_solver *s, int row);

/*
 * Test hook for the branch-free correctly rounded FP64 division the bit-exact
 * Baer-Nunziato reconstruction uses (csrc/hype_div.cuh); no counterpart in the
 * reference.  On device `device`, n operand pairs drawn from `seed` -- random
 * bit patterns (zeros, subnormals, infinities and NaNs included), random
 * operands of every exponent, near-midpoint quotients and divisors with an
 * all-ones significand -- are divided both ways.  *mismatches counts pairs whose
 * result differs from IEEE division bit for bit although the function reported
 * them in range, *specials the pairs it reported out of range (where its caller
 * uses IEEE division).
 */
HYPE_API int hype_test_division(int device, long long n, unsigned long long seed, long long *mismatches, long long *specials);

#ifdef __cplusplus
}
#endif
#endif /* HYPE_GPU_H */
