/*
 * glue_driver.c -- TEST INFRASTRUCTURE.  Calls the product's PETSc-signature
 * RHSFunctionPrim (hype-parallel_b200/csrc/petsc_glue.c) the way HyPE-2D's
 * hype.c does (an AppCtx filled as hype.c:32-68 fills it, a DMDA global Vec,
 * hype.c:343; TSSolve with the RHS registered and dt reset every step,
 * hype.c:337-384 and post_process.c:19), on the PETSc stand-in of
 * oracle/petsc_mini, and hands the RHS, the state and Ctx.dt back to the Python
 * test.  With live ranks (glue_live_join) the process is one MPI rank of a DMDA
 * split over several processes; state arrays stay whole grids and each rank
 * reads and writes its own block of them.  Built by tests/glue/Makefile
 * with -include oracle/petsc_mini/hype_ref_cfg.h (AppCtx, bndry_type) and
 * -D<SYSTEM> -DHYPE_REF_NVAR=<nVar>.
 */
#include <string.h>

PetscReal GAMMA_1 = 1.4, GAMMA_2 = 1.4, PI_1 = 0.0, PI_2 = 0.0;
PetscReal MU_1 = 1.0e-2, MU_2 = 0.0;   /* hype.h:46-47; read by the VISCOUS build */

void glue_set_mu(double mu1, double mu2) { MU_1 = mu1; MU_2 = mu2; }

PetscErrorCode RHSFunctionPrim(TS ts, PetscReal t, Vec U, Vec RHS, void *ctx);
PetscErrorCode RHSFunction(TS ts, PetscReal t, Vec U, Vec RHS, void *ctx);
void RHSFunctionPrimFinalize(void);

int glue_nvar(void) { return nVar; }

/* one rank of a y-split DMDA (petsc_mini's emulation): rank `rank` of `size` owns rows
 * ys .. ys+ym-1; the other ranks' rows come from `full` (the whole grid's state) */
void glue_emulate(int rank, int size, int ys, int ym, const double *full) { petsc_mini_emulate_rank(rank, size, ys, ym, full); }

/* live MPI ranks over a shared segment of glue_live_bytes(grid_doubles) bytes */
size_t glue_live_bytes(long long grid_doubles) { return petsc_mini_live_bytes(grid_doubles); }
int glue_live_join(int rank, int size, int px, int py, void *shm, long long grid_doubles)
{
    return petsc_mini_live_join(rank, size, px, py, shm, grid_doubles);
}
void glue_live_set_wait(double seconds) { petsc_mini_live_set_wait(seconds); }
int glue_corners(int nx, int ny, int *xs, int *ys, int *xm, int *ym)
{
    DM da;
    DMDACreate2d(PETSC_COMM_WORLD, DM_BOUNDARY_GHOSTED, DM_BOUNDARY_GHOSTED, DMDA_STENCIL_BOX, nx, ny, PETSC_DECIDE,
                 PETSC_DECIDE, nVar, 3, NULL, NULL, &da);
    DMSetUp(da);
    PetscInt a, b, c, d;
    DMDAGetCorners(da, &a, &b, NULL, &c, &d, NULL);
    *xs = (int)a; *ys = (int)b; *xm = (int)c; *ym = (int)d;
    DMDestroy(&da);
    return 0;
}

/* this rank's block of a whole-grid array <-> a Vec's local part */
static void block_in(Vec V, DM da, int nx, const double *full)
{
    PetscInt xs, ys, xm, ym;
    DMDAGetCorners(da, &xs, &ys, NULL, &xm, &ym, NULL);
    PetscScalar *a;
    VecGetArray(V, &a);
    for (PetscInt j = 0; j < ym; ++j)
        memcpy(a + (size_t)j * xm * nVar, full + ((size_t)(ys + j) * nx + xs) * nVar, sizeof(double) * xm * nVar);
    VecRestoreArray(V, &a);
}
static void block_out(Vec V, DM da, int nx, double *full)
{
    PetscInt xs, ys, xm, ym;
    DMDAGetCorners(da, &xs, &ys, NULL, &xm, &ym, NULL);
    PetscScalar *a;
    VecGetArray(V, &a);
    for (PetscInt j = 0; j < ym; ++j)
        memcpy(full + ((size_t)(ys + j) * nx + xs) * nVar, a + (size_t)j * xm * nVar, sizeof(double) * xm * nVar);
    VecRestoreArray(V, &a);
}

int glue_rhs(int N, int nx, int ny, const double dom[4], double cfl, const int bc[4], const double eos[4], int conservative,
             const double *Uin, double *Rout, double *dt)
{
    GAMMA_1 = eos[0]; GAMMA_2 = eos[1]; PI_1 = eos[2]; PI_2 = eos[3];
    AppCtx Ctx;
    memset(&Ctx, 0, sizeof(Ctx));
    Ctx.N = N; Ctx.N_x = nx; Ctx.N_y = ny;
    Ctx.x_min = dom[0]; Ctx.x_max = dom[1]; Ctx.y_min = dom[2]; Ctx.y_max = dom[3];
    Ctx.CFL = cfl;
    Ctx.h = (Ctx.x_max - Ctx.x_min) / (PetscReal)Ctx.N_x;
    Ctx.LeftBoundary = (enum bndry_type)bc[0]; Ctx.RightBoundary = (enum bndry_type)bc[1];
    Ctx.BottomBoundary = (enum bndry_type)bc[2]; Ctx.TopBoundary = (enum bndry_type)bc[3];
    Ctx.ReconsPrimitive = conservative ? PETSC_FALSE : PETSC_TRUE;
    const DMBoundaryType bx = (bc[0] == periodic || bc[1] == periodic) ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    const DMBoundaryType by = (bc[2] == periodic || bc[3] == periodic) ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    DM da;
    Vec U, R;
    DMDACreate2d(PETSC_COMM_WORLD, bx, by, DMDA_STENCIL_BOX, nx, ny, PETSC_DECIDE, PETSC_DECIDE, nVar, 3, NULL, NULL, &da);
    DMSetUp(da);
    DMCreateGlobalVector(da, &U);
    VecDuplicate(U, &R);
    DMCreateLocalVector(da, &Ctx.localU);   /* hype.c keeps it in AppCtx */
    block_in(U, da, nx, Uin);   /* this rank's block of the state (all of it on one rank) */
    TS ts;
    TSCreate(PETSC_COMM_WORLD, &ts);
    TSSetDM(ts, da);
    /* hype.c:341-352: ReconsPrimitive picks the RHS function */
    const PetscErrorCode ierr = Ctx.ReconsPrimitive ? RHSFunctionPrim(ts, 0.0, U, R, &Ctx) : RHSFunction(ts, 0.0, U, R, &Ctx);
    block_out(R, da, nx, Rout);
    *dt = Ctx.dt;
    TSDestroy(&ts);
    VecDestroy(&U);
    VecDestroy(&R);
    VecDestroy(&Ctx.localU);
    DMDestroy(&da);
    return (int)ierr;
}

void glue_finalize(void) { RHSFunctionPrimFinalize(); }

/* MonitorFunction's time-step part (post_process.c:19): dt from the last RHS */
static PetscErrorCode glue_monitor(TS ts, PetscInt step, PetscReal time, Vec U, void *ctx)
{
    (void)step; (void)time; (void)U;
    return TSSetTimeStep(ts, ((AppCtx *)ctx)->dt);
}

/* hype.c:337-384 with the glue's RHS: a direct RHS call seeds Ctx.dt (hype.c:343),
 * then TSSolve with the scheme of order N, MATCHSTEP to t_final and at most
 * max_steps steps.  Uio (whole grid) in and out; each rank writes its block. */
int glue_solve(int N, int nx, int ny, const double dom[4], double cfl, const int bc[4], const double eos[4], int conservative,
               double *Uio, double t0, double t_final, int max_steps, int *steps, double *t_end, double *dt_next)
{
    GAMMA_1 = eos[0]; GAMMA_2 = eos[1]; PI_1 = eos[2]; PI_2 = eos[3];
    AppCtx Ctx;
    memset(&Ctx, 0, sizeof(Ctx));
    Ctx.N = N; Ctx.N_x = nx; Ctx.N_y = ny;
    Ctx.x_min = dom[0]; Ctx.x_max = dom[1]; Ctx.y_min = dom[2]; Ctx.y_max = dom[3];
    Ctx.CFL = cfl;
    Ctx.h = (Ctx.x_max - Ctx.x_min) / (PetscReal)Ctx.N_x;
    Ctx.LeftBoundary = (enum bndry_type)bc[0]; Ctx.RightBoundary = (enum bndry_type)bc[1];
    Ctx.BottomBoundary = (enum bndry_type)bc[2]; Ctx.TopBoundary = (enum bndry_type)bc[3];
    Ctx.ReconsPrimitive = conservative ? PETSC_FALSE : PETSC_TRUE;
    Ctx.InitialTime = t0;
    const DMBoundaryType bx = (bc[0] == periodic || bc[1] == periodic) ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    const DMBoundaryType by = (bc[2] == periodic || bc[3] == periodic) ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    DM da;
    Vec U, R;
    DMDACreate2d(PETSC_COMM_WORLD, bx, by, DMDA_STENCIL_BOX, nx, ny, PETSC_DECIDE, PETSC_DECIDE, nVar, 3, NULL, NULL, &da);
    DMSetUp(da);
    DMCreateGlobalVector(da, &U);
    VecDuplicate(U, &R);
    DMCreateLocalVector(da, &Ctx.localU);
    block_in(U, da, nx, Uio);
    PetscErrorCode (*rhs)(TS, PetscReal, Vec, Vec, void *) = Ctx.ReconsPrimitive ? RHSFunctionPrim : RHSFunction;
    TS ts;
    TSCreate(PETSC_COMM_SELF, &ts);
    TSSetProblemType(ts, TS_NONLINEAR);
    TSSetDM(ts, da);
    PetscErrorCode ierr = rhs(ts, Ctx.InitialTime, U, R, &Ctx);
    if (!ierr) {
        TSSetRHSFunction(ts, NULL, rhs, &Ctx);
        TSSetStepNumber(ts, 0);
        TSSetTime(ts, Ctx.InitialTime);
        TSSetTimeStep(ts, Ctx.dt);
        TSMonitorSet(ts, glue_monitor, &Ctx, NULL);
        TSSetMaxTime(ts, t_final);
        TSSetExactFinalTime(ts, TS_EXACTFINALTIME_MATCHSTEP);
        TSSetMaxSteps(ts, max_steps);
        if (N == 0) TSSetType(ts, TSEULER);
        else {
            TSSetType(ts, TSSSP);
            if (N == 1) { TSSSPSetType(ts, TSSSPRKS2); TSSSPSetNumStages(ts, 2); }
            else if (N == 2) { TSSSPSetType(ts, TSSSPRKS3); TSSSPSetNumStages(ts, 4); }
            else TSSSPSetType(ts, TSSSPRK104);
        }
        ierr = TSSolve(ts, U);
    }
    PetscInt n = 0;
    PetscReal tt = 0.0;
    TSGetStepNumber(ts, &n);
    TSGetTime(ts, &tt);
    *steps = (int)n;
    *t_end = tt;
    *dt_next = Ctx.dt;
    if (!ierr) block_out(U, da, nx, Uio);
    TSDestroy(&ts);
    VecDestroy(&U);
    VecDestroy(&R);
    VecDestroy(&Ctx.localU);
    DMDestroy(&da);
    return (int)ierr;
}
