/*
 * petsc_mini.c -- single-rank implementation of the PETSc subset declared in
 * petsc_mini.h.  TEST INFRASTRUCTURE ONLY (see the header for what it restates
 * and why parity at this boundary is unpinned).
 */
#include "petsc_mini.h"
#include <stdarg.h>
#include <time.h>
#include <stddef.h>
#include <stdatomic.h>
#include <sched.h>

/* ------------------------------------------------------------------------- */
/* MPI on one rank                                                            */
/* ------------------------------------------------------------------------- */

static jmp_buf *g_abort_env = NULL;
static int g_abort_count = 0;
static int g_quiet = 1;

void petsc_mini_set_abort_target(jmp_buf *env) { g_abort_env = env; }
int  petsc_mini_abort_count(void) { return g_abort_count; }
void petsc_mini_set_quiet(int quiet) { g_quiet = quiet; }

/* Emulation of one rank of a DMDA split over ranks in y (tests of code written for
 * several ranks, in one process): DMDAs created while it is on own rows ys..ys+ym-1,
 * their global vectors hold those rows only, and DMGlobalToLocal takes the other
 * ranks' rows from `full` (the whole grid's global array).  MPI reports the
 * emulated rank and size; MPI_Allreduce still returns this rank's own values. */
static int g_emu_size = 1, g_emu_rank = 0;
static PetscInt g_emu_ys = 0, g_emu_ym = -1;
static const PetscScalar *g_emu_full = NULL;
void petsc_mini_emulate_rank(int rank, int size, PetscInt ys, PetscInt ym, const PetscScalar *full)
{
    g_emu_rank = rank; g_emu_size = size; g_emu_ys = ys; g_emu_ym = ym; g_emu_full = full;
    if (size <= 1) { g_emu_rank = 0; g_emu_size = 1; g_emu_ys = 0; g_emu_ym = -1; g_emu_full = NULL; }
}

/* ------------------------------------------------------------------------- */
/* Live ranks: `size` processes that share one memory segment (what mpiexec   */
/* and MPI give the reference).  The segment holds a barrier, an abort flag,  */
/* one reduction slot per rank and an exchange copy of the grid through which */
/* DMGlobalToLocal passes each rank's edge strips to its neighbours.          */
/* ------------------------------------------------------------------------- */
#define LIVE_MAX_RANKS 1024
#define LIVE_RED_SLOTS 8
typedef struct {
    _Atomic int arrived;
    _Atomic int sense;
    _Atomic int aborted;
    int pad_;
    long long pad2_;
    double red[LIVE_MAX_RANKS][LIVE_RED_SLOTS];       /* MPI_Allreduce contributions */
} live_hdr;
static live_hdr *g_live = NULL;
static double *g_live_exch = NULL;
static int g_live_rank = 0, g_live_size = 1, g_live_px = 0, g_live_py = 0, g_live_sense = 0;
static long long g_live_exch_doubles = 0;   /* capacity of the exchange copy */
static double g_live_wait_s = 600.0;

static size_t live_hdr_bytes(void) { return (sizeof(live_hdr) + 255) & ~(size_t)255; }
size_t petsc_mini_live_bytes(long long grid_doubles) { return live_hdr_bytes() + (size_t)grid_doubles * sizeof(double); }

int petsc_mini_live_join(int rank, int size, int px, int py, void *shm, long long grid_doubles)
{
    if (size <= 1 || !shm) { g_live = NULL; g_live_exch = NULL; g_live_rank = 0; g_live_size = 1; return 0; }
    if (size > LIVE_MAX_RANKS || rank < 0 || rank >= size) return 1;
    if ((px > 0 || py > 0) && px * py != size) return 1;
    g_live = (live_hdr *)shm;
    g_live_exch = (double *)((char *)shm + live_hdr_bytes());
    g_live_rank = rank; g_live_size = size; g_live_px = px; g_live_py = py;
    g_live_sense = 0;
    g_live_exch_doubles = grid_doubles;
    return 0;
}
void petsc_mini_live_set_wait(double seconds) { g_live_wait_s = seconds; }

static double live_now(void)
{
    struct timespec t; clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* Sense-reversing barrier over the live ranks.  A rank that aborted (MPI_Abort)
 * raises the shared flag; the others leave the barrier through MPI_Abort too, as
 * mpiexec ends every rank of a job one of whose ranks called MPI_Abort.  A wait
 * longer than g_live_wait_s (a rank that died) counts as an abort as well. */
static void live_barrier(void)
{
    const int my = g_live_sense = !g_live_sense;
    if (atomic_fetch_add(&g_live->arrived, 1) == g_live_size - 1) {
        atomic_store(&g_live->arrived, 0);
        atomic_store(&g_live->sense, my);
        return;
    }
    const double t0 = live_now();
    for (long spin = 0;; ++spin) {
        if (atomic_load(&g_live->sense) == my) return;
        if (atomic_load(&g_live->aborted)) MPI_Abort(PETSC_COMM_WORLD, 1);
        if ((spin & 1023) == 1023) {
            sched_yield();
            if (live_now() - t0 > g_live_wait_s) { atomic_store(&g_live->aborted, 1); MPI_Abort(PETSC_COMM_WORLD, 1); }
        }
    }
}

int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)t; (void)c;
    if (!g_live) { memmove(r, s, (size_t)count * sizeof(double)); return 0; }
    if (count > LIVE_RED_SLOTS) { fprintf(stderr, "petsc_mini: MPI_Allreduce of %d values\n", count); MPI_Abort(c, 1); }
    const double *sv = (const double *)s;
    for (int k = 0; k < count; ++k) g_live->red[g_live_rank][k] = sv[k];
    live_barrier();
    double out[LIVE_RED_SLOTS];
    for (int k = 0; k < count; ++k) {
        double v = g_live->red[0][k];
        for (int q = 1; q < g_live_size; ++q) {
            const double x = g_live->red[q][k];
            if (op == MPIU_MIN) v = (x < v) ? x : v;
            else if (op == MPIU_MAX) v = (x > v) ? x : v;
            else v = v + x;
        }
        out[k] = v;
    }
    live_barrier();   /* every rank has read the slots before they are written again */
    memcpy(r, out, (size_t)count * sizeof(double));
    return 0;
}
int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = g_live ? g_live_size : g_emu_size; return 0; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = g_live ? g_live_rank : g_emu_rank; return 0; }
int MPI_Abort(MPI_Comm c, int code)
{
    (void)c;
    g_abort_count++;
    if (g_live) atomic_store(&g_live->aborted, 1);   /* ends the other ranks' collective calls */
    if (g_abort_env) longjmp(*g_abort_env, code ? code : 1);
    fprintf(stderr, "petsc_mini: MPI_Abort(%d)\n", code);
    exit(code ? code : 1);
}

struct _p_PetscObject { int dummy; };
MPI_Comm PetscObjectComm(PetscObject o) { (void)o; return PETSC_COMM_WORLD; }
PetscErrorCode PetscObjectSetName(PetscObject o, const char *name) { (void)o; (void)name; return 0; }

/* ------------------------------------------------------------------------- */
/* Vec                                                                        */
/* ------------------------------------------------------------------------- */

struct _p_Vec {
    PetscInt n;
    PetscScalar *a;
    DM dm;          /* owning DM (global or local layout) */
    int local;      /* 1: ghosted local layout */
};

static Vec vec_new(PetscInt n, DM dm, int local)
{
    Vec v = (Vec)calloc(1, sizeof(*v));
    v->n = n;
    v->a = (PetscScalar *)calloc((size_t)(n > 0 ? n : 1), sizeof(PetscScalar));
    v->dm = dm;
    v->local = local;
    return v;
}

PetscErrorCode VecDuplicate(Vec v, Vec *out) { *out = vec_new(v->n, v->dm, v->local); return 0; }
PetscErrorCode VecDestroy(Vec *v)
{
    if (v && *v) { free((*v)->a); free(*v); *v = NULL; }
    return 0;
}
PetscErrorCode VecCopy(Vec x, Vec y) { memcpy(y->a, x->a, (size_t)x->n * sizeof(PetscScalar)); return 0; }
PetscErrorCode VecSet(Vec x, PetscScalar a) { for (PetscInt i = 0; i < x->n; ++i) x->a[i] = a; return 0; }

/* y <- y + a x   (one rounding per product and per sum; no contraction) */
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x)
{
    for (PetscInt i = 0; i < y->n; ++i) { PetscScalar t = a * x->a[i]; y->a[i] = y->a[i] + t; }
    return 0;
}
/* y <- a x + b y */
PetscErrorCode VecAXPBY(Vec y, PetscScalar a, PetscScalar b, Vec x)
{
    for (PetscInt i = 0; i < y->n; ++i) { PetscScalar t0 = a * x->a[i]; PetscScalar t1 = b * y->a[i]; y->a[i] = t0 + t1; }
    return 0;
}
/* z <- a x + b y + c z ; the c == 0 form drops the third term as PETSc does */
PetscErrorCode VecAXPBYPCZ(Vec z, PetscScalar a, PetscScalar b, PetscScalar c, Vec x, Vec y)
{
    if (c == 0.0) {
        for (PetscInt i = 0; i < z->n; ++i) { PetscScalar t0 = a * x->a[i]; PetscScalar t1 = b * y->a[i]; z->a[i] = t0 + t1; }
    } else {
        for (PetscInt i = 0; i < z->n; ++i) {
            PetscScalar t0 = a * x->a[i]; PetscScalar t1 = b * y->a[i]; PetscScalar t2 = c * z->a[i];
            PetscScalar s = t0 + t1;
            z->a[i] = s + t2;
        }
    }
    return 0;
}
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal *out)
{
    PetscReal r = 0.0;
    if (t == NORM_INFINITY) { for (PetscInt i = 0; i < x->n; ++i) { PetscReal v = fabs(x->a[i]); if (v > r) r = v; } }
    else if (t == NORM_1) { for (PetscInt i = 0; i < x->n; ++i) r += fabs(x->a[i]); }
    else { for (PetscInt i = 0; i < x->n; ++i) r += x->a[i] * x->a[i]; r = sqrt(r); }
    *out = r;
    return 0;
}
PetscErrorCode VecView(Vec x, PetscViewer v);   /* binary viewers: below, with the viewers */
PetscErrorCode VecGetArray(Vec x, PetscScalar **a) { *a = x->a; return 0; }
PetscErrorCode VecRestoreArray(Vec x, PetscScalar **a) { (void)x; *a = NULL; return 0; }
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar **a) { *a = x->a; return 0; }
PetscErrorCode VecRestoreArrayRead(Vec x, const PetscScalar **a) { (void)x; *a = NULL; return 0; }
PetscErrorCode VecGetLocalSize(Vec x, PetscInt *n) { *n = x->n; return 0; }

/* ------------------------------------------------------------------------- */
/* DMDA                                                                       */
/* ------------------------------------------------------------------------- */

struct _p_DM {
    PetscInt M, N, dof, s;
    DMBoundaryType bx, by;
    PetscInt xs_g, ys_g, xm_g, ym_g;   /* ghost corners */
    PetscInt xs, xm, ys, ym;            /* owned block (the whole grid on one rank) */
    DM cda;                             /* coordinate DM (dof 2) */
    Vec coords;
};

/* Ownership ranges of a DMDA over an m x n process grid, as PETSc's DMSetUp_DA_2D
 * (src/dm/impls/da/da2.c) sets them up with PETSC_DECIDE: m = the integer nearest
 * sqrt(M size / N), lowered until it divides size, n = size / m, the two swapped
 * when M > N and m < n; then M / m points per rank along x, the first M % m ranks
 * one more (the same along y), ranks numbered x fastest. */
static void live_grid(PetscInt M, PetscInt N, int size, int *m_out, int *n_out)
{
    int m = g_live_px, n = g_live_py;
    if (m <= 0 || n <= 0) {
        m = (int)(0.5 + sqrt(((PetscReal)M) * ((PetscReal)size) / ((PetscReal)N)));
        if (!m) m = 1;
        while (m > 0) {
            n = size / m;
            if (m * n == size) break;
            m--;
        }
        if (M > N && m < n) { int t = m; m = n; n = t; }
    }
    *m_out = m; *n_out = n;
}
static void own_range(PetscInt M, int m, int r, PetscInt *start, PetscInt *len)
{
    PetscInt st = 0;
    for (int q = 0; q < r; ++q) st += M / m + ((M % m) > q);
    *start = st; *len = M / m + ((M % m) > r);
}

PetscErrorCode DMDACreate2d(MPI_Comm c, DMBoundaryType bx, DMBoundaryType by, DMDAStencilType st,
                            PetscInt M, PetscInt N, PetscInt m, PetscInt n, PetscInt dof, PetscInt s,
                            const PetscInt lx[], const PetscInt ly[], DM *da)
{
    (void)c; (void)st; (void)m; (void)n; (void)lx; (void)ly;
    DM d = (DM)calloc(1, sizeof(*d));
    d->M = M; d->N = N; d->dof = dof; d->s = s; d->bx = bx; d->by = by;
    /* GHOSTED and PERIODIC both carry s ghost layers on every side of a rank's block */
    int gx = (bx == DM_BOUNDARY_NONE) ? 0 : s;
    int gy = (by == DM_BOUNDARY_NONE) ? 0 : s;
    d->xs = 0; d->xm = M;
    d->ys = 0; d->ym = N;
    if (g_live) {
        int pm, pn;
        live_grid(M, N, g_live_size, &pm, &pn);
        own_range(M, pm, g_live_rank % pm, &d->xs, &d->xm);
        own_range(N, pn, g_live_rank / pm, &d->ys, &d->ym);
        if ((long long)M * N * dof > g_live_exch_doubles) {
            fprintf(stderr, "petsc_mini: live exchange copy too small for a %dx%dx%d DMDA\n", M, N, dof);
            MPI_Abort(c, 1);
        }
    } else if (g_emu_ym >= 0) {
        d->ys = g_emu_ys; d->ym = g_emu_ym;
    }
    d->xs_g = d->xs - gx; d->xm_g = d->xm + 2 * gx;
    d->ys_g = d->ys - gy; d->ym_g = d->ym + 2 * gy;
    *da = d;
    return 0;
}
PetscErrorCode DMSetUp(DM da) { (void)da; return 0; }
PetscErrorCode DMDestroy(DM *da)
{
    if (da && *da) {
        if ((*da)->coords) VecDestroy(&(*da)->coords);
        if ((*da)->cda) free((*da)->cda);
        free(*da); *da = NULL;
    }
    return 0;
}
PetscErrorCode DMView(DM da, PetscViewer v) { (void)da; (void)v; return 0; }
PetscErrorCode DMCreateGlobalVector(DM da, Vec *v) { *v = vec_new(da->xm * da->ym * da->dof, da, 0); return 0; }
PetscErrorCode DMCreateLocalVector(DM da, Vec *v) { *v = vec_new(da->xm_g * da->ym_g * da->dof, da, 1); return 0; }

static inline PetscInt wrap(PetscInt i, PetscInt n) { PetscInt r = i % n; return r < 0 ? r + n : r; }

PetscErrorCode DMGlobalToLocalBegin(DM da, Vec g, InsertMode m, Vec l)
{
    (void)m;
    const PetscInt dof = da->dof;
    if (g_live) {
        /* each rank publishes the strips of width s along its block's edges into the
         * exchange copy (what its neighbours read), then reads its ghosts from there */
        const PetscInt s = da->s;
        for (PetscInt j = da->ys; j < da->ys + da->ym; ++j) {
            PetscScalar *dst = g_live_exch + ((size_t)j * da->M + da->xs) * dof;
            const PetscScalar *src = g->a + (size_t)(j - da->ys) * da->xm * dof;
            if (j < da->ys + s || j >= da->ys + da->ym - s || da->xm <= 2 * s) {
                memcpy(dst, src, (size_t)da->xm * dof * sizeof(PetscScalar));
            } else {
                memcpy(dst, src, (size_t)s * dof * sizeof(PetscScalar));
                memcpy(dst + (size_t)(da->xm - s) * dof, src + (size_t)(da->xm - s) * dof, (size_t)s * dof * sizeof(PetscScalar));
            }
        }
        live_barrier();
    }
    for (PetscInt j = da->ys_g; j < da->ys_g + da->ym_g; ++j) {
        int jin = (j >= 0 && j < da->N);
        if (!jin && da->by != DM_BOUNDARY_PERIODIC) continue;       /* no source: keep */
        PetscInt js = jin ? j : wrap(j, da->N);
        for (PetscInt i = da->xs_g; i < da->xs_g + da->xm_g; ++i) {
            int iin = (i >= 0 && i < da->M);
            if (!iin && da->bx != DM_BOUNDARY_PERIODIC) continue;   /* no source: keep */
            PetscInt is = iin ? i : wrap(i, da->M);
            /* this rank's block from its global vector, the other ranks' points from the
             * live exchange copy or the emulation's array */
            const int own = js >= da->ys && js < da->ys + da->ym && is >= da->xs && is < da->xs + da->xm;
            const PetscScalar *other = g_live ? g_live_exch : g_emu_full;
            if (!own && !other) continue;
            const PetscScalar *src = own ? g->a + ((size_t)(js - da->ys) * da->xm + (is - da->xs)) * dof
                                         : other + ((size_t)js * da->M + is) * dof;
            PetscScalar *dst = l->a + ((size_t)(j - da->ys_g) * da->xm_g + (i - da->xs_g)) * dof;
            memcpy(dst, src, (size_t)dof * sizeof(PetscScalar));
        }
    }
    if (g_live) live_barrier();   /* every rank has read the copy before it is written again */
    return 0;
}
PetscErrorCode DMGlobalToLocalEnd(DM da, Vec g, InsertMode m, Vec l) { (void)da; (void)g; (void)m; (void)l; return 0; }

PetscErrorCode DMDAGetCorners(DM da, PetscInt *xs, PetscInt *ys, PetscInt *zs, PetscInt *xm, PetscInt *ym, PetscInt *zm)
{
    if (xs) *xs = da->xs;
    if (ys) *ys = da->ys;
    if (zs) *zs = 0;
    if (xm) *xm = da->xm;
    if (ym) *ym = da->ym;
    if (zm) *zm = 1;
    return 0;
}
PetscErrorCode DMDAGetGhostCorners(DM da, PetscInt *xs, PetscInt *ys, PetscInt *zs, PetscInt *xm, PetscInt *ym, PetscInt *zm)
{
    if (xs) *xs = da->xs_g;
    if (ys) *ys = da->ys_g;
    if (zs) *zs = 0;
    if (xm) *xm = da->xm_g;
    if (ym) *ym = da->ym_g;
    if (zm) *zm = 1;
    return 0;
}

/* Row-pointer table a[j] such that a[j][i] (record of dof reals) is valid over
 * the vector's corner range, as PETSc's DMDAVecGetArray returns it. */
PetscErrorCode DMDAVecGetArray(DM da, Vec v, void *array)
{
    PetscInt xs, ys, xm, ym;
    if (v->local) { xs = da->xs_g; ys = da->ys_g; xm = da->xm_g; ym = da->ym_g; }
    else { xs = v->dm->xs; ys = v->dm->ys; xm = v->dm->xm; ym = v->dm->ym; }
    const PetscInt dof = v->dm->dof;
    char **rows = (char **)malloc((size_t)ym * sizeof(char *));
    for (PetscInt r = 0; r < ym; ++r)
        rows[r] = (char *)(v->a + ((size_t)r * xm) * dof) - (ptrdiff_t)xs * dof * (ptrdiff_t)sizeof(PetscScalar);
    *(char ***)array = rows - ys;
    return 0;
}
PetscErrorCode DMDAVecRestoreArray(DM da, Vec v, void *array)
{
    PetscInt ys = v->local ? da->ys_g : v->dm->ys;
    char **rows = *(char ***)array;
    if (rows) free(rows + ys);
    *(char ***)array = NULL;
    return 0;
}
PetscErrorCode DMDAVecGetArrayRead(DM da, Vec v, void *array) { return DMDAVecGetArray(da, v, array); }
PetscErrorCode DMDAVecRestoreArrayRead(DM da, Vec v, void *array) { return DMDAVecRestoreArray(da, v, array); }

PetscErrorCode DMDASetUniformCoordinates(DM da, PetscReal xmin, PetscReal xmax, PetscReal ymin, PetscReal ymax, PetscReal zmin, PetscReal zmax)
{
    (void)zmin; (void)zmax;
    if (!da->cda) {
        da->cda = (DM)calloc(1, sizeof(*da->cda));
        *da->cda = *da;
        da->cda->dof = 2; da->cda->cda = NULL; da->cda->coords = NULL;
    }
    if (da->coords) VecDestroy(&da->coords);
    da->coords = vec_new(da->M * da->N * 2, da->cda, 0);
    /* PETSc: spacing (max-min)/M when periodic, (max-min)/(M-1) otherwise */
    PetscReal hx = (da->bx == DM_BOUNDARY_PERIODIC) ? (xmax - xmin) / da->M : (da->M > 1 ? (xmax - xmin) / (da->M - 1) : 0.0);
    PetscReal hy = (da->by == DM_BOUNDARY_PERIODIC) ? (ymax - ymin) / da->N : (da->N > 1 ? (ymax - ymin) / (da->N - 1) : 0.0);
    for (PetscInt j = 0; j < da->N; ++j)
        for (PetscInt i = 0; i < da->M; ++i) {
            da->coords->a[((size_t)j * da->M + i) * 2 + 0] = xmin + hx * i;
            da->coords->a[((size_t)j * da->M + i) * 2 + 1] = ymin + hy * j;
        }
    return 0;
}
PetscErrorCode DMGetCoordinateDM(DM da, DM *cda) { *cda = da->cda; return 0; }
PetscErrorCode DMGetCoordinates(DM da, Vec *c) { *c = da->coords; return 0; }
PetscErrorCode DMDASetFieldName(DM da, PetscInt nf, const char *name) { (void)da; (void)nf; (void)name; return 0; }

/* ------------------------------------------------------------------------- */
/* TS: SSP Runge-Kutta and forward Euler, MATCHSTEP, monitor                 */
/* ------------------------------------------------------------------------- */

struct _p_TS {
    DM dm;
    TSRHSFunctionFn rhs; void *rhs_ctx;
    TSMonitorFn mon; void *mon_ctx;
    PetscInt steps, max_steps;
    PetscReal ptime, time_step, max_time;
    TSExactFinalTimeOption efto;
    int type;            /* 0 euler, 1 ssp */
    int ssp;             /* 2 rks2, 3 rks3, 104 rk104 */
    PetscInt nstages;
    Vec work[3];
};

PetscErrorCode TSCreate(MPI_Comm c, TS *ts)
{
    (void)c;
    TS t = (TS)calloc(1, sizeof(*t));
    t->max_steps = 0x7fffffff; t->max_time = 5.0; t->time_step = 0.1;
    t->type = 1; t->ssp = 2; t->nstages = 5;
    *ts = t;
    return 0;
}
PetscErrorCode TSDestroy(TS *ts)
{
    if (ts && *ts) { for (int k = 0; k < 3; ++k) if ((*ts)->work[k]) VecDestroy(&(*ts)->work[k]); free(*ts); *ts = NULL; }
    return 0;
}
PetscErrorCode TSSetProblemType(TS ts, TSProblemType t) { (void)ts; (void)t; return 0; }
PetscErrorCode TSSetDM(TS ts, DM da) { ts->dm = da; return 0; }
PetscErrorCode TSGetDM(TS ts, DM *da) { *da = ts->dm; return 0; }
PetscErrorCode TSSetRHSFunction(TS ts, Vec r, TSRHSFunctionFn f, void *ctx) { (void)r; ts->rhs = f; ts->rhs_ctx = ctx; return 0; }
PetscErrorCode TSSetStepNumber(TS ts, PetscInt n) { ts->steps = n; return 0; }
PetscErrorCode TSSetTime(TS ts, PetscReal t) { ts->ptime = t; return 0; }
PetscErrorCode TSSetTimeStep(TS ts, PetscReal dt) { ts->time_step = dt; return 0; }
PetscErrorCode TSGetTimeStep(TS ts, PetscReal *dt) { *dt = ts->time_step; return 0; }
PetscErrorCode TSMonitorSet(TS ts, TSMonitorFn f, void *ctx, void *destroy) { (void)destroy; ts->mon = f; ts->mon_ctx = ctx; return 0; }
PetscErrorCode TSSetMaxTime(TS ts, PetscReal t) { ts->max_time = t; return 0; }
PetscErrorCode TSSetMaxSteps(TS ts, PetscInt n) { ts->max_steps = n; return 0; }
PetscErrorCode TSSetExactFinalTime(TS ts, TSExactFinalTimeOption o) { ts->efto = o; return 0; }
PetscErrorCode TSSetFromOptions(TS ts) { (void)ts; return 0; }
PetscErrorCode TSSetType(TS ts, TSType t) { ts->type = (strcmp(t, TSEULER) == 0) ? 0 : 1; return 0; }
PetscErrorCode TSSSPSetType(TS ts, TSSSPType t)
{
    if (strcmp(t, TSSSPRKS2) == 0) ts->ssp = 2;
    else if (strcmp(t, TSSSPRKS3) == 0) ts->ssp = 3;
    else ts->ssp = 104;
    return 0;
}
PetscErrorCode TSSSPSetNumStages(TS ts, PetscInt n) { ts->nstages = n; return 0; }
PetscErrorCode TSGetStepNumber(TS ts, PetscInt *n) { *n = ts->steps; return 0; }
PetscErrorCode TSGetTime(TS ts, PetscReal *t) { *t = ts->ptime; return 0; }

static PetscErrorCode ts_work(TS ts, Vec like)
{
    for (int k = 0; k < 3; ++k) if (!ts->work[k]) VecDuplicate(like, &ts->work[k]);
    return 0;
}

/* SSPRKS2 with s stages (s-1 forward-Euler substeps of dt/(s-1), then an average) */
static PetscErrorCode step_rks2(TS ts, PetscReal t0, PetscReal dt, Vec sol)
{
    PetscErrorCode ierr;
    Vec w = ts->work[0], F = ts->work[1];
    PetscInt s = ts->nstages;
    VecCopy(sol, w);
    for (PetscInt i = 0; i < s - 1; ++i) {
        PetscReal st = t0 + dt * (i / (s - 1.));
        ierr = ts->rhs(ts, st, w, F, ts->rhs_ctx); CHKERRQ(ierr);
        VecAXPY(w, dt / (s - 1.), F);
    }
    ierr = ts->rhs(ts, t0 + dt, w, F, ts->rhs_ctx); CHKERRQ(ierr);
    VecAXPBYPCZ(sol, (s - 1.) / s, dt / s, 1. / s, w, F);
    return 0;
}

/* SSPRKS3 with s = n^2 stages (Ketcheson's low-storage third-order family) */
static PetscErrorCode step_rks3(TS ts, PetscReal t0, PetscReal dt, Vec sol)
{
    PetscErrorCode ierr;
    Vec w0 = ts->work[0], w1 = ts->work[1], F = ts->work[2];
    PetscInt s = ts->nstages;
    PetscInt n = (PetscInt)(sqrt((PetscReal)s) + 0.001);
    PetscInt r = s - n, i;
    PetscReal c, st;
    VecCopy(sol, w0);
    for (i = 0; i < (n - 1) * (n - 2) / 2; ++i) {
        c = (i < n * (n + 1) / 2) ? 1. * i / (s - n) : (1. * i - n) / (s - n);
        st = t0 + c * dt;
        ierr = ts->rhs(ts, st, w0, F, ts->rhs_ctx); CHKERRQ(ierr);
        VecAXPY(w0, dt / r, F);
    }
    VecCopy(w0, w1);
    for (; i < n * (n + 1) / 2 - 1; ++i) {
        c = (i < n * (n + 1) / 2) ? 1. * i / (s - n) : (1. * i - n) / (s - n);
        st = t0 + c * dt;
        ierr = ts->rhs(ts, st, w0, F, ts->rhs_ctx); CHKERRQ(ierr);
        VecAXPY(w0, dt / r, F);
    }
    {
        c = (i < n * (n + 1) / 2) ? 1. * i / (s - n) : (1. * i - n) / (s - n);
        st = t0 + c * dt;
        ierr = ts->rhs(ts, st, w0, F, ts->rhs_ctx); CHKERRQ(ierr);
        VecAXPBYPCZ(w0, 1. * n / (2 * n - 1.), (n - 1.) * dt / (r * (2 * n - 1)), (n - 1.) / (2 * n - 1.), w1, F);
        ++i;
    }
    for (; i < s; ++i) {
        c = (i < n * (n + 1) / 2) ? 1. * i / (s - n) : (1. * i - n) / (s - n);
        st = t0 + c * dt;
        ierr = ts->rhs(ts, st, w0, F, ts->rhs_ctx); CHKERRQ(ierr);
        VecAXPY(w0, dt / r, F);
    }
    VecCopy(w0, sol);
    return 0;
}

/* Ten-stage fourth-order SSPRK(10,4) */
static PetscErrorCode step_rk104(TS ts, PetscReal t0, PetscReal dt, Vec sol)
{
    PetscErrorCode ierr;
    static const PetscReal c[10] = {0, 1. / 6, 2. / 6, 3. / 6, 4. / 6, 2. / 6, 3. / 6, 4. / 6, 5. / 6, 1};
    Vec w0 = ts->work[0], w1 = ts->work[1], F = ts->work[2];
    PetscInt i;
    VecCopy(sol, w0);
    for (i = 0; i < 5; ++i) {
        ierr = ts->rhs(ts, t0 + c[i] * dt, w0, F, ts->rhs_ctx); CHKERRQ(ierr);
        VecAXPY(w0, dt / 6, F);
    }
    VecAXPBYPCZ(w1, 1. / 25, 9. / 25, 0, sol, w0);
    VecAXPBY(w0, 15, -5, w1);
    for (; i < 9; ++i) {
        ierr = ts->rhs(ts, t0 + c[i] * dt, w0, F, ts->rhs_ctx); CHKERRQ(ierr);
        VecAXPY(w0, dt / 6, F);
    }
    ierr = ts->rhs(ts, t0 + dt, w0, F, ts->rhs_ctx); CHKERRQ(ierr);
    VecAXPBYPCZ(w1, 3. / 5, dt / 10, 1, w0, F);
    VecCopy(w1, sol);
    return 0;
}

static PetscErrorCode step_euler(TS ts, PetscReal t0, PetscReal dt, Vec sol)
{
    PetscErrorCode ierr;
    Vec F = ts->work[0];
    ierr = ts->rhs(ts, t0, sol, F, ts->rhs_ctx); CHKERRQ(ierr);
    VecAXPY(sol, dt, F);
    return 0;
}

PetscErrorCode TSSolve(TS ts, Vec u)
{
    PetscErrorCode ierr;
    ts_work(ts, u);
    if (ts->mon) { ierr = ts->mon(ts, ts->steps, ts->ptime, u, ts->mon_ctx); CHKERRQ(ierr); }
    for (;;) {
        if (ts->steps >= ts->max_steps) break;
        if (ts->ptime >= ts->max_time) break;
        PetscReal dt = ts->time_step;
        if (ts->efto == TS_EXACTFINALTIME_MATCHSTEP && ts->ptime + dt > ts->max_time) dt = ts->max_time - ts->ptime;
        PetscReal t0 = ts->ptime;
        if (ts->type == 0) ierr = step_euler(ts, t0, dt, u);
        else if (ts->ssp == 2) ierr = step_rks2(ts, t0, dt, u);
        else if (ts->ssp == 3) ierr = step_rks3(ts, t0, dt, u);
        else ierr = step_rk104(ts, t0, dt, u);
        CHKERRQ(ierr);
        ts->ptime = t0 + dt;
        ts->steps++;
        if (ts->mon) { ierr = ts->mon(ts, ts->steps, ts->ptime, u, ts->mon_ctx); CHKERRQ(ierr); }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* misc                                                                       */
/* ------------------------------------------------------------------------- */

PetscErrorCode PetscPrintf(MPI_Comm c, const char *fmt, ...)
{
    (void)c;
    if (g_quiet) return 0;
    va_list ap; va_start(ap, fmt); vprintf(fmt, ap); va_end(ap);
    return 0;
}
PetscErrorCode PetscTime(PetscLogDouble *t)
{
    struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
    *t = (PetscLogDouble)ts.tv_sec + 1e-9 * (PetscLogDouble)ts.tv_nsec;
    return 0;
}
/* Viewers.  A binary viewer follows PETSc's published binary format: VecView
 * writes the Vec class id 1211214 and the global length as big-endian 32-bit
 * integers, then the values as big-endian IEEE doubles in the DMDA's natural
 * (row-major, component-interleaved) order, and records "-vecload_block_size
 * <dof>" in the companion file <name>.info for a block size above 1; VecLoad
 * reads that layout back.  With live ranks every rank passes its block through
 * the exchange copy and rank 0 writes the file; on load every rank reads its own
 * block.
 * A VTK viewer does not restate PETSc's XML framing: VecView on it writes the
 * viewed Vec's values as raw little-endian doubles in natural order to the
 * viewer's file name, which is what a test compares with the data arrays of a
 * .vts file (DMView on it is a no-op). */
enum { VIEWER_NULL = 0, VIEWER_BINARY = 1, VIEWER_VTK = 2 };
struct _p_PetscViewer { int kind; FILE *f; FILE *info; int writing; char name[4096]; };
#define VEC_FILE_CLASSID 1211214

PetscErrorCode PetscViewerVTKOpen(MPI_Comm c, const char *name, PetscFileMode m, PetscViewer *v)
{
    (void)c; (void)m;
    PetscViewer b = (PetscViewer)calloc(1, sizeof(*b));
    b->kind = VIEWER_VTK;
    b->writing = 1;
    snprintf(b->name, sizeof(b->name), "%s", name);
    *v = b;
    return 0;
}
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm c, const char *name, PetscFileMode m, PetscViewer *v)
{
    (void)c;
    PetscViewer b = (PetscViewer)calloc(1, sizeof(*b));
    b->kind = VIEWER_BINARY;
    b->writing = (m != FILE_MODE_READ);
    if (!g_live || g_live_rank == 0 || !b->writing) {
        b->f = fopen(name, b->writing ? "wb" : "rb");
        if (!b->f) { free(b); *v = NULL; return 1; }
        if (b->writing) {
            char info[4096];
            snprintf(info, sizeof(info), "%s.info", name);
            b->info = fopen(info, "w");
        }
    }
    *v = b;
    return 0;
}
PetscErrorCode PetscViewerDestroy(PetscViewer *v)
{
    if (v && *v && (*v)->kind != VIEWER_NULL) {
        if ((*v)->f) fclose((*v)->f);
        if ((*v)->info) fclose((*v)->info);
        free(*v);
    }
    if (v) *v = NULL;
    return 0;
}

static void be32_put(unsigned char *p, unsigned u) { p[0] = u >> 24; p[1] = u >> 16; p[2] = u >> 8; p[3] = u; }
static unsigned be32_get(const unsigned char *p) { return ((unsigned)p[0] << 24) | ((unsigned)p[1] << 16) | ((unsigned)p[2] << 8) | p[3]; }
static void be64_put(unsigned char *p, double d)
{
    unsigned long long u; memcpy(&u, &d, 8);
    for (int k = 0; k < 8; ++k) p[k] = (unsigned char)(u >> (56 - 8 * k));
}
static double be64_get(const unsigned char *p)
{
    unsigned long long u = 0;
    for (int k = 0; k < 8; ++k) u = (u << 8) | p[k];
    double d; memcpy(&d, &u, 8);
    return d;
}

PetscErrorCode VecView(Vec x, PetscViewer v)
{
    if (!v || v->kind == VIEWER_NULL || !v->writing) return 0;
    DM da = x->dm;
    const PetscInt dof = da->dof;
    const size_t n = (size_t)da->M * da->N * dof;
    const PetscScalar *full = x->a;
    if (g_live) {   /* gather the blocks in natural order through the exchange copy */
        for (PetscInt j = da->ys; j < da->ys + da->ym; ++j)
            memcpy(g_live_exch + ((size_t)j * da->M + da->xs) * dof, x->a + (size_t)(j - da->ys) * da->xm * dof,
                   (size_t)da->xm * dof * sizeof(PetscScalar));
        live_barrier();
        full = g_live_exch;
    }
    int rc = 0;
    if (v->kind == VIEWER_VTK) {
        if (!g_live || g_live_rank == 0) {
            FILE *f = fopen(v->name, "wb");
            if (!f || fwrite(full, sizeof(PetscScalar), n, f) != n) rc = 1;
            if (f) fclose(f);
        }
    } else if (v->f) {
        unsigned char head[8];
        be32_put(head, VEC_FILE_CLASSID);
        be32_put(head + 4, (unsigned)n);
        unsigned char *body = (unsigned char *)malloc(n * 8);
        for (size_t k = 0; k < n; ++k) be64_put(body + 8 * k, full[k]);
        if (fwrite(head, 1, 8, v->f) != 8 || fwrite(body, 1, n * 8, v->f) != n * 8) rc = 1;
        free(body);
        if (v->info && dof > 1) fprintf(v->info, "-vecload_block_size %d\n", dof);
    }
    if (g_live) live_barrier();   /* rank 0 has written before the copy is reused */
    return rc;
}

PetscErrorCode VecLoad(Vec x, PetscViewer v)
{
    if (!v || v->kind != VIEWER_BINARY || v->writing || !v->f) return 1;
    DM da = x->dm;
    const PetscInt dof = da->dof;
    const size_t n = (size_t)da->M * da->N * dof;
    unsigned char head[8];
    if (fread(head, 1, 8, v->f) != 8 || be32_get(head) != VEC_FILE_CLASSID || be32_get(head + 4) != (unsigned)n) return 1;
    unsigned char *body = (unsigned char *)malloc(n * 8);
    const int ok = fread(body, 1, n * 8, v->f) == n * 8;
    if (ok)
        for (PetscInt j = da->ys; j < da->ys + da->ym; ++j)
            for (PetscInt i = da->xs; i < da->xs + da->xm; ++i)
                for (PetscInt c = 0; c < dof; ++c)
                    x->a[((size_t)(j - da->ys) * da->xm + (i - da->xs)) * dof + c] = be64_get(body + 8 * (((size_t)j * da->M + i) * dof + c));
    free(body);
    return ok ? 0 : 1;
}
