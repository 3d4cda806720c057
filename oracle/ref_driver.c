/*
 * ref_driver.c -- drives the reference's own (unmodified) HyPE-2D sources,
 * compiled against petsc_mini into oracle/_ref/libhype_ref_<system>.so.
 * TEST INFRASTRUCTURE ONLY: used to pin the C restatement (hype_oracle.c) and
 * to generate the golden fixtures under tests/golden/.
 *
 * ref_setup() mirrors the set-up part of HyPE-2D/hype.c:
 *   nDOF, h, quadrature counts            hype.c:56-68
 *   DMDA (BOX, ghost width 3)             hype.c:95-122
 *   vectors, coordinates                  hype.c:126-135
 *   quadrature points/weights, nodes      hype.c:194-230
 *   scratch arrays and basis tables       hype.c:232-309 (via the reference's
 *                                          basis()/basis_grad(), reconstruction.c:11-100)
 * ref_rhs() calls the reference's RHSFunctionPrim / RHSFunction once.
 * ref_solve() mirrors hype.c:337-384: a direct RHS call seeds Ctx.dt, then
 * TSSolve with the reference's MonitorFunction resetting dt every step;
 * ref_begin() / ref_advance() are the same loop split into chunks of steps.
 *
 * With live ranks (ref_live_join before ref_setup) the process is one MPI rank
 * of a DMDA split over several processes, as under mpiexec: state arrays
 * crossing this file's entry points are then the rank's block (ref_corners),
 * compact, in the Vec layout.
 */
#include <setjmp.h>

PetscReal GAMMA_1 = 1.4, GAMMA_2 = 1.4, PI_1 = 0.0, PI_2 = 0.0;
PetscReal MU_1 = 1.0e-2, MU_2 = 0.0;

/* Symbols that hype.h declares but the chosen PDE file does not define (they
 * are only reached from code paths the oracle does not take: inlet BCs for
 * Euler / Baer-Nunziato, viscous fluxes for Baer-Nunziato, initial data). */
#if defined(EULER) || defined(BAER_NUNZIATO)
static int g_missing_called = 0;
void InletBC(PetscReal x, PetscReal y, PetscReal t, PetscReal *Q)
{ (void)x; (void)y; (void)t; for (int c = 0; c < nVar; ++c) Q[c] = NAN; g_missing_called = 1; }
void InletBCPrim(PetscReal x, PetscReal y, PetscReal t, PetscReal *V)
{ (void)x; (void)y; (void)t; for (int c = 0; c < nVar; ++c) V[c] = NAN; g_missing_called = 1; }
#endif
#if defined(BAER_NUNZIATO)
PetscReal PDEViscFlux(const PetscReal *Q, const PetscReal g[nVar][DIM], PetscReal nx, PetscReal ny, PetscReal *F)
{ (void)Q; (void)g; (void)nx; (void)ny; for (int c = 0; c < nVar; ++c) F[c] = 0.0; g_missing_called = 1; return 0.0; }
PetscReal PDEViscFluxPrim(const PetscReal *V, const PetscReal g[nVar][DIM], PetscReal nx, PetscReal ny, PetscReal *F)
{ (void)V; (void)g; (void)nx; (void)ny; for (int c = 0; c < nVar; ++c) F[c] = 0.0; g_missing_called = 1; return 0.0; }
#endif
void InitialCondition(PetscReal x, PetscReal y, PetscReal *Q0) { (void)x; (void)y; for (int c = 0; c < nVar; ++c) Q0[c] = 0.0; }

typedef struct {
    int N;                    /* degree: 0..3 */
    int nx, ny;
    double x_min, x_max, y_min, y_max;
    double cfl;
    int bc_left, bc_right, bc_bottom, bc_top;   /* enum bndry_type values */
    double gamma1, gamma2, pi1, pi2;
    double mu1, mu2;          /* MU_1, MU_2: read by the VISCOUS build only */
} ref_cfg;

static AppCtx Ctx;
static DM da = NULL;
static Vec U = NULL, RHS = NULL;
static TS ts_rhs = NULL;
static TS ts_run = NULL;      /* the time loop of ref_begin / ref_advance */
static int g_ready = 0;

int ref_nvar(void) { return nVar; }

/* one MPI rank of `size` live processes sharing `shm` (petsc_mini_live_join); call before ref_setup */
size_t ref_live_bytes(long long grid_doubles) { return petsc_mini_live_bytes(grid_doubles); }
int ref_live_join(int rank, int size, int px, int py, void *shm, long long grid_doubles)
{
    return petsc_mini_live_join(rank, size, px, py, shm, grid_doubles);
}
void ref_live_set_wait(double seconds) { petsc_mini_live_set_wait(seconds); }

/* this rank's block of the grid (the whole grid on one rank) */
int ref_corners(int *xs, int *ys, int *xm, int *ym)
{
    if (!g_ready) return -1;
    PetscInt a, b, c, d;
    DMDAGetCorners(da, &a, &b, NULL, &c, &d, NULL);
    *xs = a; *ys = b; *xm = c; *ym = d;
    return 0;
}
static size_t local_doubles(void) { PetscInt n; VecGetLocalSize(U, &n); return (size_t)n; }

void ref_teardown(void)
{
    if (!g_ready) return;
    if (ts_run) TSDestroy(&ts_run);
    VecDestroy(&U); VecDestroy(&RHS); VecDestroy(&Ctx.W); VecDestroy(&Ctx.localU);
    TSDestroy(&ts_rhs);
    free5d(Ctx.u_bnd); free3d(Ctx.F);
#ifdef VISCOUS
    free6d(Ctx.u_bnd_grad);
#endif
    free3d(Ctx.G); free3d(Ctx.D); free3d(Ctx.E);
    free3d(Ctx.phiFace); free2d(Ctx.phiNode); free2d(Ctx.phiVol);
    free2d(Ctx.gradphiVol_x); free2d(Ctx.gradphiVol_y);
    free3d(Ctx.gradphiFace_x); free3d(Ctx.gradphiFace_y);
    PetscFree(Ctx.xGP_Face); PetscFree(Ctx.wGP_Face); PetscFree(Ctx.xGP_Vol);
    PetscFree(Ctx.yGP_Vol); PetscFree(Ctx.wGP_Vol); PetscFree(Ctx.x_node); PetscFree(Ctx.y_node);
    DMDestroy(&da);
    g_ready = 0;
}

int ref_setup(const ref_cfg *cfg)
{
    ref_teardown();
    GAMMA_1 = cfg->gamma1; GAMMA_2 = cfg->gamma2; PI_1 = cfg->pi1; PI_2 = cfg->pi2;
    MU_1 = cfg->mu1; MU_2 = cfg->mu2;
    memset(&Ctx, 0, sizeof(Ctx));
    Ctx.N = cfg->N;
    Ctx.x_min = cfg->x_min; Ctx.x_max = cfg->x_max; Ctx.y_min = cfg->y_min; Ctx.y_max = cfg->y_max;
    Ctx.N_x = cfg->nx; Ctx.N_y = cfg->ny; Ctx.CFL = cfg->cfl;
    Ctx.WriteInterval = 0; Ctx.RestartInterval = 0; Ctx.ReconsPrimitive = PETSC_TRUE;
    Ctx.LeftBoundary = (enum bndry_type)cfg->bc_left; Ctx.RightBoundary = (enum bndry_type)cfg->bc_right;
    Ctx.BottomBoundary = (enum bndry_type)cfg->bc_bottom; Ctx.TopBoundary = (enum bndry_type)cfg->bc_top;

    Ctx.nDOF = (Ctx.N + 1) * (Ctx.N + 2) / 2;
    Ctx.h = (Ctx.x_max - Ctx.x_min) / (PetscReal)(Ctx.N_x);
    if (Ctx.N < 2) { Ctx.Ngp_Face = 1; Ctx.Ngp_Vol = 1; }
    else { Ctx.Ngp_Face = 2; Ctx.Ngp_Vol = 4; }
    Ctx.N_node = 4 * Ctx.Ngp_Face;

    DMBoundaryType bx = (Ctx.LeftBoundary == periodic || Ctx.RightBoundary == periodic) ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    DMBoundaryType by = (Ctx.BottomBoundary == periodic || Ctx.TopBoundary == periodic) ? DM_BOUNDARY_PERIODIC : DM_BOUNDARY_GHOSTED;
    DMDACreate2d(PETSC_COMM_WORLD, bx, by, DMDA_STENCIL_BOX, Ctx.N_x, Ctx.N_y, PETSC_DECIDE, PETSC_DECIDE, nVar, 3, NULL, NULL, &da);
    DMSetUp(da);
    DMCreateGlobalVector(da, &U);
    VecDuplicate(U, &Ctx.W);
    VecDuplicate(U, &RHS);
    DMDASetUniformCoordinates(da, Ctx.x_min + 0.5 * Ctx.h, Ctx.x_max + 0.5 * Ctx.h, Ctx.y_min + 0.5 * Ctx.h, Ctx.y_max + 0.5 * Ctx.h, 0.0, 0.0);

    PetscMalloc1(Ctx.Ngp_Face, &Ctx.xGP_Face); PetscMalloc1(Ctx.Ngp_Face, &Ctx.wGP_Face);
    PetscMalloc1(Ctx.Ngp_Vol, &Ctx.xGP_Vol); PetscMalloc1(Ctx.Ngp_Vol, &Ctx.yGP_Vol); PetscMalloc1(Ctx.Ngp_Vol, &Ctx.wGP_Vol);
    PetscMalloc1(Ctx.N_node, &Ctx.x_node); PetscMalloc1(Ctx.N_node, &Ctx.y_node);
    const PetscReal g = 0.28867513459481287;
    if (Ctx.N < 2) {
        Ctx.xGP_Face[0] = 0.0; Ctx.wGP_Face[0] = 1.0;
        Ctx.xGP_Vol[0] = 0.0; Ctx.yGP_Vol[0] = 0.0; Ctx.wGP_Vol[0] = 1.0;
        Ctx.x_node[0] = 0.5; Ctx.y_node[0] = 0.0; Ctx.x_node[1] = -0.5; Ctx.y_node[1] = 0.0;
        Ctx.x_node[2] = 0.0; Ctx.y_node[2] = 0.5; Ctx.x_node[3] = 0.0; Ctx.y_node[3] = -0.5;
    } else {
        Ctx.xGP_Face[0] = -g; Ctx.wGP_Face[0] = 0.5; Ctx.xGP_Face[1] = g; Ctx.wGP_Face[1] = 0.5;
        const PetscReal vx[4] = {-g, -g, g, g}, vy[4] = {-g, g, -g, g};
        for (int q = 0; q < 4; ++q) { Ctx.xGP_Vol[q] = vx[q]; Ctx.yGP_Vol[q] = vy[q]; Ctx.wGP_Vol[q] = 0.25; }
        const PetscReal nxn[8] = {0.5, 0.5, -0.5, -0.5, -g, g, -g, g};
        const PetscReal nyn[8] = {-g, g, -g, g, 0.5, 0.5, -0.5, -0.5};
        for (int q = 0; q < 8; ++q) { Ctx.x_node[q] = nxn[q]; Ctx.y_node[q] = nyn[q]; }
    }

    PetscInt xs, ys, xm, ym;
    DMDAGetCorners(da, &xs, &ys, NULL, &xm, &ym, NULL);
    Ctx.u_bnd = allocate5d(ym + 2, xm + 2, nVar, 4, Ctx.Ngp_Face);
#ifdef VISCOUS
    Ctx.u_bnd_grad = allocate6d(ym + 2, xm + 2, nVar, 4, Ctx.Ngp_Face, DIM);   /* hype.c:238-240 */
#endif
    Ctx.F = allocate3d(ym, xm + 1, nVar);
    Ctx.G = allocate3d(ym + 1, xm, nVar);
    Ctx.D = allocate3d(ym, xm + 1, nVar);
    Ctx.E = allocate3d(ym + 1, xm, nVar);
    Ctx.phiFace = allocate3d(4, Ctx.Ngp_Face, Ctx.nDOF);
    Ctx.phiNode = allocate2d(Ctx.N_node, Ctx.nDOF);
    Ctx.phiVol = allocate2d(Ctx.Ngp_Vol, Ctx.nDOF);
    Ctx.gradphiVol_x = allocate2d(Ctx.Ngp_Vol, Ctx.nDOF);
    Ctx.gradphiVol_y = allocate2d(Ctx.Ngp_Vol, Ctx.nDOF);
    Ctx.gradphiFace_x = allocate3d(4, Ctx.Ngp_Face, Ctx.nDOF);
    Ctx.gradphiFace_y = allocate3d(4, Ctx.Ngp_Face, Ctx.nDOF);

    PetscReal value, gx, gy;
    for (PetscInt q = 0; q < Ctx.Ngp_Face; ++q)
        for (PetscInt k = 0; k < Ctx.nDOF; ++k) {
            const PetscReal fx[4] = {-0.5, 0.5, Ctx.xGP_Face[q], Ctx.xGP_Face[q]};
            const PetscReal fy[4] = {Ctx.xGP_Face[q], Ctx.xGP_Face[q], -0.5, 0.5};
            for (int f = 0; f < 4; ++f) {
                value = basis(fx[f], fy[f], k);
                basis_grad(fx[f], fy[f], k, &gx, &gy);
                set_element_3d(Ctx.phiFace, f, q, k, value);
                set_element_3d(Ctx.gradphiFace_x, f, q, k, gx);
                set_element_3d(Ctx.gradphiFace_y, f, q, k, gy);
            }
        }
    for (PetscInt q = 0; q < Ctx.N_node; ++q)
        for (PetscInt k = 0; k < Ctx.nDOF; ++k)
            set_element_2d(Ctx.phiNode, q, k, basis(Ctx.x_node[q], Ctx.y_node[q], k));
    for (PetscInt q = 0; q < Ctx.Ngp_Vol; ++q)
        for (PetscInt k = 0; k < Ctx.nDOF; ++k) {
            set_element_2d(Ctx.phiVol, q, k, basis(Ctx.xGP_Vol[q], Ctx.yGP_Vol[q], k));
            basis_grad(Ctx.xGP_Vol[q], Ctx.yGP_Vol[q], k, &gx, &gy);
            set_element_2d(Ctx.gradphiVol_x, q, k, gx);
            set_element_2d(Ctx.gradphiVol_y, q, k, gy);
        }
    DMCreateLocalVector(da, &Ctx.localU);

    TSCreate(PETSC_COMM_SELF, &ts_rhs);
    TSSetDM(ts_rhs, da);
    g_ready = 1;
    return 0;
}

/* One RHS evaluation. prim=1: RHSFunctionPrim (rhs_function_prim.c:12), prim=0:
 * RHSFunction (rhs_function.c:12).  Returns 0, or 1 if the reference aborted
 * (inadmissible face state).  U and RHS are AoS, nx*ny*nVar. */
int ref_rhs(double t, const double *Uin, double *RHSout, double *dt_out, int prim)
{
    if (!g_ready) return -1;
    PetscScalar *a;
    VecGetArray(U, &a); memcpy(a, Uin, sizeof(double) * local_doubles()); VecRestoreArray(U, &a);
    jmp_buf env;
    petsc_mini_set_abort_target(&env);
    if (setjmp(env)) { petsc_mini_set_abort_target(NULL); return 1; }
    PetscErrorCode ierr = prim ? RHSFunctionPrim(ts_rhs, t, U, RHS, &Ctx) : RHSFunction(ts_rhs, t, U, RHS, &Ctx);
    petsc_mini_set_abort_target(NULL);
    if (ierr) return -2;
    VecGetArray(RHS, &a); memcpy(RHSout, a, sizeof(double) * local_doubles()); VecRestoreArray(RHS, &a);
    if (dt_out) *dt_out = Ctx.dt;
    return 0;
}

/* TS set-up of hype.c:337-382 around the state in U: the direct RHS call that seeds
 * Ctx.dt (hype.c:343), then the scheme of order N, MATCHSTEP and the monitor. */
static TS make_ts(int prim, double t_final, int max_steps)
{
    TS ts;
    TSCreate(PETSC_COMM_SELF, &ts);
    TSSetProblemType(ts, TS_NONLINEAR);
    TSSetDM(ts, da);
    if (prim) { RHSFunctionPrim(ts, Ctx.InitialTime, U, RHS, &Ctx); TSSetRHSFunction(ts, NULL, RHSFunctionPrim, &Ctx); }
    else { RHSFunction(ts, Ctx.InitialTime, U, RHS, &Ctx); TSSetRHSFunction(ts, NULL, RHSFunction, &Ctx); }
    TSSetStepNumber(ts, Ctx.InitialStep);
    TSSetTime(ts, Ctx.InitialTime);
    TSSetTimeStep(ts, Ctx.dt);
    TSMonitorSet(ts, MonitorFunction, &Ctx, NULL);
    TSSetMaxTime(ts, t_final);
    TSSetExactFinalTime(ts, TS_EXACTFINALTIME_MATCHSTEP);
    TSSetMaxSteps(ts, max_steps);
    TSSetFromOptions(ts);
    if (Ctx.N == 0) TSSetType(ts, TSEULER);
    else {
        TSSetType(ts, TSSSP);
        if (Ctx.N == 1) { TSSSPSetType(ts, TSSSPRKS2); TSSSPSetNumStages(ts, 2); }
        else if (Ctx.N == 2) { TSSSPSetType(ts, TSSSPRKS3); TSSSPSetNumStages(ts, 4); }
        else TSSSPSetType(ts, TSSSPRK104);
    }
    return ts;
}

/* Time loop as hype.c:337-384, with -ts_max_steps given as max_steps. */
int ref_solve(double *Uio, double t0, double t_final, int max_steps, int prim,
              int *steps_out, double *t_out, double *dt_out)
{
    if (!g_ready) return -1;
    PetscScalar *a;
    VecGetArray(U, &a); memcpy(a, Uio, sizeof(double) * local_doubles()); VecRestoreArray(U, &a);
    Ctx.InitialTime = t0; Ctx.InitialStep = 0; Ctx.FinalTime = t_final;
    TS ts = NULL;
    jmp_buf env;
    petsc_mini_set_abort_target(&env);
    if (setjmp(env)) { petsc_mini_set_abort_target(NULL); if (ts) TSDestroy(&ts); return 1; }
    ts = make_ts(prim, Ctx.FinalTime, max_steps);
    PetscErrorCode ierr = TSSolve(ts, U);
    petsc_mini_set_abort_target(NULL);
    PetscInt n; PetscReal tt;
    TSGetStepNumber(ts, &n); TSGetTime(ts, &tt);
    TSDestroy(&ts);
    if (ierr) return -2;
    VecGetArray(U, &a); memcpy(Uio, a, sizeof(double) * local_doubles()); VecRestoreArray(U, &a);
    if (steps_out) *steps_out = n;
    if (t_out) *t_out = tt;
    if (dt_out) *dt_out = Ctx.dt;
    return 0;
}

/* The same loop in chunks: ref_begin loads the state and seeds dt (hype.c:343);
 * each ref_advance runs up to nsteps more steps of the one TS (TSSolve resumes
 * where the last chunk stopped: its monitor call at the start only sets dt again
 * to Ctx.dt).  Returns 0, 1 where the reference aborted, -1 without a begin. */
int ref_begin(const double *Uin, double t0, double t_final, int prim)
{
    if (!g_ready) return -1;
    if (ts_run) TSDestroy(&ts_run);
    PetscScalar *a;
    VecGetArray(U, &a); memcpy(a, Uin, sizeof(double) * local_doubles()); VecRestoreArray(U, &a);
    Ctx.InitialTime = t0; Ctx.InitialStep = 0; Ctx.FinalTime = t_final;
    jmp_buf env;
    petsc_mini_set_abort_target(&env);
    if (setjmp(env)) { petsc_mini_set_abort_target(NULL); return 1; }
    ts_run = make_ts(prim, t_final, 0);
    petsc_mini_set_abort_target(NULL);
    return 0;
}
int ref_advance(int nsteps, int *steps_out, double *t_out, double *dt_out)
{
    if (!g_ready || !ts_run) return -1;
    PetscInt n0;
    TSGetStepNumber(ts_run, &n0);
    TSSetMaxSteps(ts_run, n0 + nsteps);
    jmp_buf env;
    petsc_mini_set_abort_target(&env);
    if (setjmp(env)) { petsc_mini_set_abort_target(NULL); TSDestroy(&ts_run); return 1; }
    PetscErrorCode ierr = TSSolve(ts_run, U);
    petsc_mini_set_abort_target(NULL);
    if (ierr) return -2;
    PetscInt n; PetscReal tt;
    TSGetStepNumber(ts_run, &n); TSGetTime(ts_run, &tt);
    if (steps_out) *steps_out = n;
    if (t_out) *t_out = tt;
    if (dt_out) *dt_out = Ctx.dt;
    return 0;
}
int ref_get_state(double *Uout);

/* The output schedule of the reference's MonitorFunction (post_process.c:12-64):
 * a solution file every write_interval steps (sol-%08d.vts, primitive variables
 * from ComputePrimitiveVariables), restart1.bin every restart_interval steps and
 * restart2.bin where (step + 7) % restart_interval == 0, written in the current
 * directory.  0 turns a kind of output off (the default after ref_setup). */
void ref_set_output(int write_interval, int restart_interval)
{
    Ctx.WriteInterval = write_interval;
    Ctx.RestartInterval = restart_interval;
}

/* hype.c:389-400 after TSSolve: the primitive variables of U written to
 * sol-<steps>.vts in the current directory. */
int ref_write_final(int steps)
{
    if (!g_ready) return -1;
    ComputePrimitiveVariables(U, Ctx.W, da);
    char filename[20];
    PetscViewer viewer;
    sprintf(filename, "sol-%08d.vts", steps);
    if (PetscViewerVTKOpen(PETSC_COMM_WORLD, filename, FILE_MODE_WRITE, &viewer)) return 1;
    DMView(da, viewer);
    const int rc = VecView(Ctx.W, viewer) != 0;
    PetscViewerDestroy(&viewer);
    return rc;
}

/* hype.c:316-325: the state read from restart1.bin in the current directory with
 * VecLoad, returned in Uout.  Returns 0, or 1 where the file is missing or does
 * not hold a Vec of this grid. */
int ref_load_restart(double *Uout)
{
    if (!g_ready) return -1;
    PetscViewer viewer_binary;
    if (PetscViewerBinaryOpen(PETSC_COMM_WORLD, "restart1.bin", FILE_MODE_READ, &viewer_binary)) return 1;
    const int rc = VecLoad(U, viewer_binary) != 0;
    PetscViewerDestroy(&viewer_binary);
    if (rc) return 1;
    return ref_get_state(Uout);
}

int ref_get_state(double *Uout)
{
    if (!g_ready) return -1;
    PetscScalar *a;
    VecGetArray(U, &a); memcpy(Uout, a, sizeof(double) * local_doubles()); VecRestoreArray(U, &a);
    return 0;
}
