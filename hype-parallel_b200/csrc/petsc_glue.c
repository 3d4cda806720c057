/*
 * petsc_glue.c -- RHSFunctionPrim and RHSFunction with the reference's PETSc
 * signatures, forwarding to the C ABI of include/hype_gpu.h.
 *
 * It replaces HyPE-2D/rhs_function_prim.c and rhs_function.c in a HyPE-2D
 * build (RHSFunction: the conservative-variable path that hype.c selects when
 * Ctx.ReconsPrimitive is false, hype.c:341-352): compile it in
 * that tree (it includes the tree's hype.h for AppCtx, the PDE-system #define
 * and the EOS constants GAMMA_1, GAMMA_2, PI_1, PI_2, and the tree's PETSc),
 * link libhype_b200.so, and hype.c's
 *     TSSetRHSFunction(ts, NULL, RHSFunctionPrim, &Ctx);       (hype.c:344)
 *     TSSetRHSFunction(ts, NULL, RHSFunction, &Ctx);           (hype.c:351)
 * and its direct dt-seeding calls (hype.c:343, 350) reach the B200 kernels.
 *
 * Contract kept from rhs_function_prim.c:12-626 / rhs_function.c:12-625 /
 * hype.h:305-306:
 *   - RHS is overwritten for every owned cell; U is not modified;
 *   - Ctx->dt is set to CFL*h/(2*s_max) (rhs_function_prim.c:617-623);
 *   - the scratch of AppCtx (W, localU, u_bnd, F, G, D, E) is not touched:
 *     the kernels need none of it.
 * Differences:
 *   - an inadmissible face state (the reference prints and calls MPI_Abort,
 *     e.g. kapila_5eqn.c:353-357) prints the same kind of message and returns
 *     a non-zero PetscErrorCode, so TS stops through CHKERRQ instead of the
 *     process ending;
 *   - one MPI rank: the whole grid is on this rank's GPU (the DMDA must not
 *     be split); with more ranks the call returns an error.
 * The GPU solver is created on first use and re-created when the AppCtx
 * parameters change (grid, order, CFL, boundaries).  The device is
 * HYPE_DEVICE from the environment, else 0.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "hype.h"
#include "hype_gpu.h"

/* one GPU solver per path: [0] primitive, [1] conservative reconstruction */
static hype_solver *glue_solver[2] = {NULL, NULL};
static hype_config glue_cfg[2];

static int glue_system(void)
{
#if defined(KAPILA_5EQN)
    return HYPE_KAPILA_5EQN;
#elif defined(BAER_NUNZIATO)
    return HYPE_BAER_NUNZIATO;
#else
    return HYPE_EULER;
#endif
}

/* AppCtx (hype.h:203-252) and the compile-time constants -> hype_config.
 * enum bndry_type (hype.h:76) and HYPE_BC_* have the same values. */
static void glue_config(const AppCtx *Ctx, int conservative, hype_config *c)
{
    const char *dev = getenv("HYPE_DEVICE");
    hype_config_default(c);
    c->system = glue_system();
    c->order = (int)Ctx->N;
    c->nx = (int)Ctx->N_x;
    c->ny = (int)Ctx->N_y;
    c->x_min = Ctx->x_min; c->x_max = Ctx->x_max;
    c->y_min = Ctx->y_min; c->y_max = Ctx->y_max;
    c->cfl = Ctx->CFL;
    c->bc_left = (int)Ctx->LeftBoundary;
    c->bc_right = (int)Ctx->RightBoundary;
    c->bc_bottom = (int)Ctx->BottomBoundary;
    c->bc_top = (int)Ctx->TopBoundary;
    c->gamma1 = GAMMA_1; c->gamma2 = GAMMA_2;
    c->pi1 = PI_1; c->pi2 = PI_2;
    c->precision = HYPE_PREC_FP64;
    c->flags = conservative ? HYPE_FLAG_CONSERVATIVE : 0u;
#ifdef VISCOUS
    c->flags |= HYPE_FLAG_VISCOUS;   /* the tree's VISCOUS build (hype.h:36) */
    c->mu1 = MU_1; c->mu2 = MU_2;
#endif
    c->device = dev ? atoi(dev) : 0;
}

/* Frees the GPU solvers (e.g. from the application's clean-up, hype.c:421-451). */
void RHSFunctionPrimFinalize(void)
{
    for (int k = 0; k < 2; ++k) {
        hype_destroy(glue_solver[k]);
        glue_solver[k] = NULL;
    }
}

static PetscErrorCode glue_rhs(int conservative, PetscReal t, Vec U, Vec RHS, AppCtx *Ctx)
{
    int size = 1;
    MPI_Comm_size(PETSC_COMM_WORLD, &size);
    if (size != 1) {
        fprintf(stderr, "RHSFunction (GPU): one MPI rank only, got %d\n", size);
        return 1;
    }
    hype_config c;
    glue_config(Ctx, conservative, &c);
    if (!glue_solver[conservative] || memcmp(&c, &glue_cfg[conservative], sizeof(c)) != 0) {
        hype_destroy(glue_solver[conservative]);
        glue_solver[conservative] = NULL;
        hype_solver *s = NULL;
        const int st = hype_create(&c, &s);
        if (st != HYPE_OK) {
            fprintf(stderr, "RHSFunction (GPU): %s\n", s ? hype_last_error(s) : hype_status_string(st));
            hype_destroy(s);
            return (PetscErrorCode)st;
        }
        glue_solver[conservative] = s;
        glue_cfg[conservative] = c;
    }
    const PetscScalar *u = NULL;
    PetscScalar *r = NULL;
    PetscErrorCode ierr = VecGetArrayRead(U, &u);
    if (ierr) return ierr;
    ierr = VecGetArray(RHS, &r);
    if (ierr) { VecRestoreArrayRead(U, &u); return ierr; }
    double dt = 0.0;
    const int st = hype_rhs_prim(glue_solver[conservative], (double)t, (const double *)u, (double *)r, &dt);
    VecRestoreArray(RHS, &r);
    VecRestoreArrayRead(U, &u);
    if (st != HYPE_OK) {
        fprintf(stderr, "RHSFunction (GPU): %s\n", hype_last_error(glue_solver[conservative]));
        return (PetscErrorCode)st;
    }
    Ctx->dt = dt;   /* rhs_function_prim.c:623, rhs_function.c:622 */
    return 0;
}

PetscErrorCode RHSFunctionPrim(TS ts, PetscReal t, Vec U, Vec RHS, void *ctx)
{
    (void)ts;
    return glue_rhs(0, t, U, RHS, (AppCtx *)ctx);
}

PetscErrorCode RHSFunction(TS ts, PetscReal t, Vec U, Vec RHS, void *ctx)
{
    (void)ts;
    return glue_rhs(1, t, U, RHS, (AppCtx *)ctx);
}
