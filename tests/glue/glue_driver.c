/*
 * glue_driver.c -- TEST INFRASTRUCTURE.  Calls the product's PETSc-signature
 * RHSFunctionPrim (hype-parallel_b200/csrc/petsc_glue.c) the way HyPE-2D's
 * hype.c does (an AppCtx filled as hype.c:32-68 fills it, a DMDA global Vec,
 * hype.c:343), on the one-rank PETSc stand-in of oracle/petsc_mini, and hands
 * the RHS and Ctx.dt back to the Python test.  Built by tests/glue/Makefile
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
    /* this rank's rows of the state (all of them on one rank) */
    PetscInt xs, ys, xm, ym;
    DMDAGetCorners(da, &xs, &ys, NULL, &xm, &ym, NULL);
    const size_t row = (size_t)nx * nVar;
    PetscScalar *a;
    VecGetArray(U, &a);
    memcpy(a, Uin + (size_t)ys * row, sizeof(double) * row * ym);
    VecRestoreArray(U, &a);
    TS ts;
    TSCreate(PETSC_COMM_WORLD, &ts);
    TSSetDM(ts, da);
    /* hype.c:341-352: ReconsPrimitive picks the RHS function */
    const PetscErrorCode ierr = Ctx.ReconsPrimitive ? RHSFunctionPrim(ts, 0.0, U, R, &Ctx) : RHSFunction(ts, 0.0, U, R, &Ctx);
    VecGetArray(R, &a);
    memcpy(Rout + (size_t)ys * row, a, sizeof(double) * row * ym);
    VecRestoreArray(R, &a);
    *dt = Ctx.dt;
    TSDestroy(&ts);
    VecDestroy(&U);
    VecDestroy(&R);
    VecDestroy(&Ctx.localU);
    DMDestroy(&da);
    return (int)ierr;
}

void glue_finalize(void) { RHSFunctionPrimFinalize(); }
