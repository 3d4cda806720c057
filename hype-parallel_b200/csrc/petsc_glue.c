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
 *   - the scratch of AppCtx (W, u_bnd, F, G, D, E) is not touched: the kernels
 *     need none of it; with several ranks, localU takes the ghosted state, as in
 *     rhs_function_prim.c:44-45.
 Several MPI ranks (the DMDA of hype.c:108-122 split PETSC_DECIDE x PETSC_DECIDE,
 * in x, in y or both): each rank's GPU solver owns its block of cells
 * (hype_create_block); DMGlobalToLocal brings the 3 ghost rows and columns from
 * the neighbouring ranks (corners included, BOX stencil), hype_rhs_prim_slab
 * computes the rank's RHS and dt, and Ctx->dt is the MPI_Allreduce(MIN) of the
 * ranks' dt, as in rhs_function_prim.c:620-623.
 * Differences:
 *   - an inadmissible face state (the reference prints and calls MPI_Abort,
 *     e.g. kapila_5eqn.c:353-357) prints the same kind of message and returns
 *     a non-zero PetscErrorCode, so TS stops through CHKERRQ instead of the
 *     process ending;
 *   - a failed RHS on any rank makes every rank return the error (a reduction of
 *     the status), where the reference's failing rank would MPI_Abort.
 * The GPU solver is created on first use and re-created when the AppCtx
 * parameters change (grid, order, CFL, boundaries).  The device is
 * HYPE_DEVICE from the environment, else 0.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "hype.h"
#include "hype_gpu.h"

/* one GPU solver per path: [0] primitive, [1] conservative reconstruction; with
 * several ranks, for this rank's block: columns col0 .. col0+cols-1, rows row0 ..
 * row0+rows-1 */
static hype_solver *glue_solver[2] = {NULL, NULL};
static hype_config glue_cfg[2];
static int glue_col0[2], glue_cols[2], glue_row0[2], glue_rows[2];

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

static PetscErrorCode glue_rhs(int conservative, TS ts, PetscReal t, Vec U, Vec RHS, AppCtx *Ctx)
{
    int size = 1;
    MPI_Comm_size(PETSC_COMM_WORLD, &size);
    hype_config c;
    glue_config(Ctx, conservative, &c);
    int col0 = 0, cols = c.nx, row0 = 0, rows = c.ny, st = HYPE_OK;
    DM da = NULL;
    PetscInt gxs = 0, gys = 0, gxm = 0, gym = 0;
    if (size > 1) {   /* this rank's block of the DMDA (rhs_function_prim.c:36-53) */
        PetscInt xs, ys, xm, ym;
        TSGetDM(ts, &da);
        DMDAGetCorners(da, &xs, &ys, NULL, &xm, &ym, NULL);
        DMDAGetGhostCorners(da, &gxs, &gys, NULL, &gxm, &gym, NULL);
        col0 = (int)xs;
        cols = (int)xm;
        row0 = (int)ys;
        rows = (int)ym;
    }
    if (st == HYPE_OK && (!glue_solver[conservative] || memcmp(&c, &glue_cfg[conservative], sizeof(c)) != 0 ||
                          glue_col0[conservative] != col0 || glue_cols[conservative] != cols ||
                          glue_row0[conservative] != row0 || glue_rows[conservative] != rows)) {
        hype_destroy(glue_solver[conservative]);
        glue_solver[conservative] = NULL;
        hype_solver *s = NULL;
        st = size > 1 ? hype_create_block(&c, col0, cols, row0, rows, &s) : hype_create(&c, &s);
        if (st != HYPE_OK) {
            fprintf(stderr, "RHSFunction (GPU): %s\n", s ? hype_last_error(s) : hype_status_string(st));
            hype_destroy(s);
        } else {
            glue_solver[conservative] = s;
            glue_cfg[conservative] = c;
            glue_col0[conservative] = col0;
            glue_cols[conservative] = cols;
            glue_row0[conservative] = row0;
            glue_rows[conservative] = rows;
        }
    }
    double dt = 0.0;
    if (st == HYPE_OK) {
        const PetscScalar *u = NULL;
        PetscScalar *r = NULL;
        Vec in = size > 1 ? Ctx->localU : U;
        PetscErrorCode ierr = 0;
        if (size > 1) {   /* the neighbours' ghost rows (rhs_function_prim.c:44-45) */
            ierr = DMGlobalToLocalBegin(da, U, INSERT_VALUES, Ctx->localU);
            if (!ierr) ierr = DMGlobalToLocalEnd(da, U, INSERT_VALUES, Ctx->localU);
        }
        if (!ierr) ierr = VecGetArrayRead(in, &u);
        if (!ierr && (ierr = VecGetArray(RHS, &r)) != 0) VecRestoreArrayRead(in, &u);
        if (ierr) return ierr;
        hype_solver *s = glue_solver[conservative];
        if (size > 1) {
            const int nv = hype_nvar(c.system);
            /* cell (col0, row0) of the ghosted local array; its rows are gxm records apart */
            const double *u0 = (const double *)u + ((size_t)(row0 - gys) * gxm + (size_t)(col0 - gxs)) * nv;
            st = hype_rhs_prim_slab(s, (double)t, u0, (long long)gxm * nv, (double *)r, &dt);
        } else {
            st = hype_rhs_prim(s, (double)t, (const double *)u, (double *)r, &dt);
        }
        VecRestoreArray(RHS, &r);
        VecRestoreArrayRead(in, &u);
        if (st != HYPE_OK) fprintf(stderr, "RHSFunction (GPU): %s\n", hype_last_error(s));
    }
    if (size > 1) {   /* every rank returns the same status; dt is the minimum over ranks */
        const PetscReal mine = (PetscReal)st, dt_mine = dt;
        PetscReal worst = mine, dt_all = dt;
        MPI_Allreduce(&mine, &worst, 1, MPIU_REAL, MPIU_MAX, PETSC_COMM_WORLD);
        MPI_Allreduce(&dt_mine, &dt_all, 1, MPIU_REAL, MPIU_MIN, PETSC_COMM_WORLD);
        st = (int)worst;
        dt = dt_all;
    }
    if (st != HYPE_OK) return (PetscErrorCode)st;
    Ctx->dt = dt;   /* rhs_function_prim.c:623, rhs_function.c:622 */
    return 0;
}

PetscErrorCode RHSFunctionPrim(TS ts, PetscReal t, Vec U, Vec RHS, void *ctx)
{
    return glue_rhs(0, ts, t, U, RHS, (AppCtx *)ctx);
}

PetscErrorCode RHSFunction(TS ts, PetscReal t, Vec U, Vec RHS, void *ctx)
{
    return glue_rhs(1, ts, t, U, RHS, (AppCtx *)ctx);
}
