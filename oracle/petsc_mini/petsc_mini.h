/*
 * petsc_mini.h -- a single-rank stand-in for the part of the PETSc C API that
 * HyPE-2D's hot path (RHSFunctionPrim / RHSFunction and the TS loop that calls
 * them) uses.  TEST INFRASTRUCTURE ONLY: it lets the reference's own .c files
 * compile unmodified (see oracle/Makefile) so their outputs can pin the oracle.
 *
 * PETSc itself (DMDA halo scatter, TS SSP schemes) is not available in this
 * image; what is restated here follows PETSc's published behaviour:
 *   - DMDA 2D, dof per point, stencil width s, DM_BOUNDARY_GHOSTED/PERIODIC,
 *     local vectors carry s ghost layers; one rank owns the whole grid, live
 *     ranks (petsc_mini_live_join) own the blocks of PETSc's process grid.
 *     DMGlobalToLocal copies owned values and fills ghost points whose source
 *     exists (periodic wrap); other ghost points keep their previous contents.
 *   - DMDAVecGetArray returns row pointers offset so that a[j][i] is valid for
 *     j,i in the (ghost) corner range, as PETSc does.
 *   - TSSSP RKS2 / RKS3 / RK104 and TSEULER steppers, TS_EXACTFINALTIME_MATCHSTEP,
 *     monitor called before the first step and after each step.
 * Parity at this boundary (halo, TS) is therefore unpinned: no reference test
 * pins it; it is pinned only by the published scheme definitions.
 */
#ifndef PETSC_MINI_H
#define PETSC_MINI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double PetscReal;
typedef double PetscScalar;
typedef int    PetscInt;
typedef int    PetscMPIInt;
typedef int    PetscErrorCode;
typedef double PetscLogDouble;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;

#define PETSC_PI 3.14159265358979323846264338327950288419716939937510582
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE PETSC_DECIDE

#define PetscSqrtReal(a)  sqrt(a)
#define PetscAbsReal(a)   fabs(a)
#define PetscSinReal(a)   sin(a)
#define PetscCosReal(a)   cos(a)
#define PetscTanhReal(a)  tanh(a)
#define PetscExpReal(a)   exp(a)
#define PetscPowReal(a,b) pow(a,b)
#define PetscMax(a,b) (((a)<(b)) ? (b) : (a))
#define PetscMin(a,b) (((a)<(b)) ? (a) : (b))

#define CHKERRQ(e) do { if (e) return (e); } while (0)

/* ---- MPI on one rank ---------------------------------------------------- */
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define PETSC_COMM_WORLD ((MPI_Comm)0)
#define PETSC_COMM_SELF  ((MPI_Comm)1)
#define MPIU_REAL ((MPI_Datatype)1)
#define MPIU_MIN  ((MPI_Op)1)
#define MPIU_MAX  ((MPI_Op)2)
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Comm_size(MPI_Comm c, int *size);
int MPI_Comm_rank(MPI_Comm c, int *rank);
/* The reference calls MPI_Abort on an inadmissible face state; the stand-in
 * records the event and long-jumps back to the driver (petsc_mini_set_abort_target). */
int MPI_Abort(MPI_Comm c, int code);
/* test hook: emulate rank `rank` of `size` owning rows ys..ys+ym-1 of a y-split DMDA,
 * the other ranks' rows read from `full`; size <= 1 switches it off */
void petsc_mini_emulate_rank(int rank, int size, PetscInt ys, PetscInt ym, const PetscScalar *full);
/* Live ranks: `size` processes (this one is `rank`) share the zero-filled segment
 * `shm` of petsc_mini_live_bytes(grid_doubles) bytes, grid_doubles being at least
 * M*N*dof of the DMDAs they create.  DMDAs created after the join are split over a
 * px x py process grid (0, 0: PETSc's PETSC_DECIDE rule), DMGlobalToLocal passes
 * each rank's edge strips to its neighbours through the segment, MPI_Allreduce
 * reduces over the ranks (MIN, MAX or sum, in rank order) and MPI_Abort in one rank
 * ends the collective calls of all of them.  Returns 0, or 1 for a bad argument.
 * size <= 1 leaves the live mode.  After an abort the segment is spent. */
size_t petsc_mini_live_bytes(long long grid_doubles);
int petsc_mini_live_join(int rank, int size, int px, int py, void *shm, long long grid_doubles);
void petsc_mini_live_set_wait(double seconds);   /* longest barrier wait before an abort (600 s) */

/* ---- objects ------------------------------------------------------------ */
typedef struct _p_Vec         *Vec;
typedef struct _p_DM          *DM;
typedef struct _p_TS          *TS;
typedef struct _p_PetscViewer *PetscViewer;
typedef struct _p_PetscObject *PetscObject;
MPI_Comm PetscObjectComm(PetscObject o);
PetscErrorCode PetscObjectSetName(PetscObject o, const char *name);

typedef struct { PetscReal x, y; } DMDACoor2d;
typedef enum { DM_BOUNDARY_NONE, DM_BOUNDARY_GHOSTED, DM_BOUNDARY_MIRROR, DM_BOUNDARY_PERIODIC, DM_BOUNDARY_TWIST } DMBoundaryType;
typedef enum { DMDA_STENCIL_STAR, DMDA_STENCIL_BOX } DMDAStencilType;
typedef enum { NOT_SET_VALUES, INSERT_VALUES, ADD_VALUES } InsertMode;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_FROBENIUS = 2, NORM_INFINITY = 3 } NormType;
typedef enum { FILE_MODE_READ, FILE_MODE_WRITE, FILE_MODE_APPEND } PetscFileMode;

/* ---- Vec ----------------------------------------------------------------- */
PetscErrorCode VecDuplicate(Vec v, Vec *out);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecSet(Vec x, PetscScalar a);
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecAXPBY(Vec y, PetscScalar a, PetscScalar b, Vec x);
PetscErrorCode VecAXPBYPCZ(Vec z, PetscScalar a, PetscScalar b, PetscScalar c, Vec x, Vec y);
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal *out);
PetscErrorCode VecView(Vec x, PetscViewer v);
PetscErrorCode VecLoad(Vec x, PetscViewer v);
PetscErrorCode VecGetArray(Vec x, PetscScalar **a);
PetscErrorCode VecRestoreArray(Vec x, PetscScalar **a);
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar **a);
PetscErrorCode VecRestoreArrayRead(Vec x, const PetscScalar **a);
PetscErrorCode VecGetLocalSize(Vec x, PetscInt *n);

/* ---- DMDA ---------------------------------------------------------------- */
PetscErrorCode DMDACreate2d(MPI_Comm c, DMBoundaryType bx, DMBoundaryType by, DMDAStencilType st,
                            PetscInt M, PetscInt N, PetscInt m, PetscInt n, PetscInt dof, PetscInt s,
                            const PetscInt lx[], const PetscInt ly[], DM *da);
PetscErrorCode DMSetUp(DM da);
PetscErrorCode DMDestroy(DM *da);
PetscErrorCode DMView(DM da, PetscViewer v);
PetscErrorCode DMCreateGlobalVector(DM da, Vec *v);
PetscErrorCode DMCreateLocalVector(DM da, Vec *v);
PetscErrorCode DMGlobalToLocalBegin(DM da, Vec g, InsertMode m, Vec l);
PetscErrorCode DMGlobalToLocalEnd(DM da, Vec g, InsertMode m, Vec l);
PetscErrorCode DMDAGetCorners(DM da, PetscInt *xs, PetscInt *ys, PetscInt *zs, PetscInt *xm, PetscInt *ym, PetscInt *zm);
PetscErrorCode DMDAGetGhostCorners(DM da, PetscInt *xs, PetscInt *ys, PetscInt *zs, PetscInt *xm, PetscInt *ym, PetscInt *zm);
PetscErrorCode DMDAVecGetArray(DM da, Vec v, void *array);
PetscErrorCode DMDAVecRestoreArray(DM da, Vec v, void *array);
PetscErrorCode DMDAVecGetArrayRead(DM da, Vec v, void *array);
PetscErrorCode DMDAVecRestoreArrayRead(DM da, Vec v, void *array);
PetscErrorCode DMDASetUniformCoordinates(DM da, PetscReal xmin, PetscReal xmax, PetscReal ymin, PetscReal ymax, PetscReal zmin, PetscReal zmax);
PetscErrorCode DMGetCoordinateDM(DM da, DM *cda);
PetscErrorCode DMGetCoordinates(DM da, Vec *c);
PetscErrorCode DMDASetFieldName(DM da, PetscInt nf, const char *name);

/* ---- TS ------------------------------------------------------------------ */
typedef const char *TSType;
typedef const char *TSSSPType;
#define TSEULER    "euler"
#define TSSSP      "ssp"
#define TSSSPRKS2  "rks2"
#define TSSSPRKS3  "rks3"
#define TSSSPRK104 "rk104"
typedef enum { TS_LINEAR, TS_NONLINEAR } TSProblemType;
typedef enum { TS_EXACTFINALTIME_UNSPECIFIED, TS_EXACTFINALTIME_STEPOVER, TS_EXACTFINALTIME_INTERPOLATE, TS_EXACTFINALTIME_MATCHSTEP } TSExactFinalTimeOption;
typedef PetscErrorCode (*TSRHSFunctionFn)(TS, PetscReal, Vec, Vec, void *);
typedef PetscErrorCode (*TSMonitorFn)(TS, PetscInt, PetscReal, Vec, void *);

PetscErrorCode TSCreate(MPI_Comm c, TS *ts);
PetscErrorCode TSDestroy(TS *ts);
PetscErrorCode TSSetProblemType(TS ts, TSProblemType t);
PetscErrorCode TSSetDM(TS ts, DM da);
PetscErrorCode TSGetDM(TS ts, DM *da);
PetscErrorCode TSSetRHSFunction(TS ts, Vec r, TSRHSFunctionFn f, void *ctx);
PetscErrorCode TSSetStepNumber(TS ts, PetscInt n);
PetscErrorCode TSSetTime(TS ts, PetscReal t);
PetscErrorCode TSSetTimeStep(TS ts, PetscReal dt);
PetscErrorCode TSGetTimeStep(TS ts, PetscReal *dt);
PetscErrorCode TSMonitorSet(TS ts, TSMonitorFn f, void *ctx, void *destroy);
PetscErrorCode TSSetMaxTime(TS ts, PetscReal t);
PetscErrorCode TSSetMaxSteps(TS ts, PetscInt n);
PetscErrorCode TSSetExactFinalTime(TS ts, TSExactFinalTimeOption o);
PetscErrorCode TSSetFromOptions(TS ts);
PetscErrorCode TSSetType(TS ts, TSType t);
PetscErrorCode TSSSPSetType(TS ts, TSSSPType t);
PetscErrorCode TSSSPSetNumStages(TS ts, PetscInt n);
PetscErrorCode TSSolve(TS ts, Vec u);
PetscErrorCode TSGetStepNumber(TS ts, PetscInt *n);
PetscErrorCode TSGetTime(TS ts, PetscReal *t);

/* ---- misc ---------------------------------------------------------------- */
PetscErrorCode PetscPrintf(MPI_Comm c, const char *fmt, ...);
PetscErrorCode PetscTime(PetscLogDouble *t);
PetscErrorCode PetscViewerVTKOpen(MPI_Comm c, const char *name, PetscFileMode m, PetscViewer *v);
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm c, const char *name, PetscFileMode m, PetscViewer *v);
PetscErrorCode PetscViewerDestroy(PetscViewer *v);
#define PetscMalloc1(n, p) ((*(p) = calloc((size_t)(n) ? (size_t)(n) : 1, sizeof(**(p)))) == NULL)
#define PetscFree(p) (free(p), (p) = NULL, 0)

/* ---- stand-in control (not PETSc API) ------------------------------------ */
#include <setjmp.h>
void petsc_mini_set_abort_target(jmp_buf *env);   /* NULL: MPI_Abort exits the process */
int  petsc_mini_abort_count(void);
void petsc_mini_set_quiet(int quiet);

#ifdef __cplusplus
}
#endif
#endif
