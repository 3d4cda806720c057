/*
 * hype_ic.c -- seeded initial data for the benchmark workloads (host code).
 *
 * The reference samples its test cases with 5x5 Gauss cell averages
 * (initialize_solution.c:21-81); the generators here either sample at cell
 * centres (the seeded shock-bubble / disc / quadrant workloads, which have no
 * reference counterpart) or use the same 5x5 Gauss average (SmoothVortex,
 * kapila_5eqn.c:527-562, the case behind the reference's convergence table).
 * Deterministic for a given seed on every platform: splitmix64 + integer-exact
 * conversions, libm only for sqrt/tanh/sin/cos/erfc.  The random parameters are
 * drawn first; the cells are then filled row band by row band on up to 16 host
 * threads (a cell's value does not depend on which thread computes it).
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include "../../include/hype_gpu.h"
#include "../../include/hype_ic.h"

typedef struct { uint64_t s; } rng_t;
static uint64_t next_u64(rng_t *r)
{
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double unif(rng_t *r, double a, double b) { return a + (b - a) * ((double)(next_u64(r) >> 11) * (1.0 / 9007199254740992.0)); }

/* fill(ctx, j0, j1) over rows 0..ny-1 in bands on host threads: one thread below
 * 65536 cells, else up to min(16, online cores) */
typedef void (*rows_fn)(const void *ctx, int j0, int j1);
typedef struct { rows_fn fn; const void *ctx; int j0, j1; } band_t;
static void *band_main(void *a)
{
    const band_t *b = (const band_t *)a;
    b->fn(b->ctx, b->j0, b->j1);
    return NULL;
}
static void par_rows(int nx, int ny, rows_fn fn, const void *ctx)
{
    long nproc = sysconf(_SC_NPROCESSORS_ONLN);
    int T = (long long)nx * ny < 65536 ? 1 : (int)(nproc < 1 ? 1 : nproc > 16 ? 16 : nproc);
    if (T > ny) T = ny;
    pthread_t th[16];
    band_t bands[16];
    int started = 0;
    for (int t = 1; t < T; ++t) {
        bands[t] = (band_t){fn, ctx, (int)((long long)ny * t / T), (int)((long long)ny * (t + 1) / T)};
        if (pthread_create(&th[t], NULL, band_main, &bands[t]) != 0) break;
        started = t;
    }
    /* this thread takes band 0 and every band a thread could not be started for */
    fn(ctx, 0, (int)((long long)ny / T));
    if (started + 1 < T) fn(ctx, (int)((long long)ny * (started + 1) / T), ny);
    for (int t = 1; t <= started; ++t) pthread_join(th[t], NULL);
}

/* Kapila primitive -> conserved (kapila_5eqn.c:41-61) */
static void kap_p2c(const hype_config *c, const double *V, double *Q)
{
    double a1 = V[5], a2 = 1.0 - a1;
    double rho = a1 * V[0] + a2 * V[1];
    double G1m1 = c->gamma1 - 1.0, G2m1 = c->gamma2 - 1.0;
    double e = (V[4] * (a1 * G2m1 + a2 * G1m1) + a1 * c->gamma1 * c->pi1 * G2m1 + a2 * c->gamma2 * c->pi2 * G1m1) / (G1m1 * G2m1);
    Q[0] = a1 * V[0]; Q[1] = a2 * V[1]; Q[2] = rho * V[2]; Q[3] = rho * V[3];
    Q[4] = e + 0.5 * rho * (V[2] * V[2] + V[3] * V[3]); Q[5] = a1;
}
/* Baer-Nunziato primitive -> conserved (baer_nunziato.c:47-60) */
static void bn_p2c(const hype_config *c, const double *V, double *Q)
{
    Q[0] = V[8] * V[0]; Q[1] = Q[0] * V[1]; Q[2] = Q[0] * V[2];
    Q[3] = Q[0] * (0.5 * (V[1] * V[1] + V[2] * V[2]) + (V[3] + c->gamma1 * c->pi1) / (V[0] * (c->gamma1 - 1.0)));
    Q[4] = (1.0 - V[8]) * V[4]; Q[5] = Q[4] * V[5]; Q[6] = Q[4] * V[6];
    Q[7] = Q[4] * (0.5 * (V[5] * V[5] + V[6] * V[6]) + (V[7] + c->gamma2 * c->pi2) / (V[4] * (c->gamma2 - 1.0)));
    Q[8] = V[8];
}
/* Euler primitive -> conserved (euler.c:29-38) */
static void eul_p2c(const hype_config *c, const double *V, double *Q)
{
    Q[0] = V[0]; Q[1] = V[0] * V[1]; Q[2] = V[0] * V[2];
    Q[3] = 0.5 * V[0] * (V[1] * V[1] + V[2] * V[2]) + V[3] / (c->gamma1 - 1.0);
}

/* Stiffened-gas Rankine-Hugoniot state behind a shock moving in +x into fluid
 * at rest (p0, rho0): pbar = p + pi; density ratio
 * ((g+1) pbar1 + (g-1) pbar0) / ((g-1) pbar1 + (g+1) pbar0); velocity behind
 * u1 = sqrt((p1 - p0)(1/rho0 - 1/rho1)). */
static void rh_state(double g, double pi, double p0, double rho0, double p1, double *rho1, double *u1)
{
    double pb0 = p0 + pi, pb1 = p1 + pi;
    double r = ((g + 1.0) * pb1 + (g - 1.0) * pb0) / ((g - 1.0) * pb1 + (g + 1.0) * pb0);
    *rho1 = rho0 * r;
    *u1 = sqrt((p1 - p0) * (1.0 / rho0 - 1.0 / *rho1));
}

typedef struct {
    const hype_config *c;
    double *U;
    double h, Lx, Ly, eps, p0, rho1, rho2, p1, r1s, u1s, r2s;
    int nbubbles;
    double bx[64], by[64], br[64];
} sb_ctx;
static void sb_rows(const void *ctx, int j0, int j1)
{
    const sb_ctx *k = (const sb_ctx *)ctx;
    const hype_config *c = k->c;
    const double h = k->h, Lx = k->Lx, Ly = k->Ly, eps = k->eps;
    for (int j = j0; j < j1; ++j)
        for (int i = 0; i < c->nx; ++i) {
            const double x = c->x_min + (i + 0.5) * h, y = c->y_min + (j + 0.5) * h;
            const double xn = (x - c->x_min) / Lx, yn = (y - c->y_min) / Ly;   /* unit-square coordinates */
            double a1 = 1.0 - eps;
            for (int b = 0; b < k->nbubbles; ++b) {
                const double d = sqrt((xn - k->bx[b]) * (xn - k->bx[b]) + (yn - k->by[b]) * (yn - k->by[b]));
                /* alpha_1 (phase 1 = liquid) drops to eps inside the bubble, tanh edge of width 2 cells */
                const double ab = eps + (1.0 - 2.0 * eps) * 0.5 * (1.0 + tanh((d - k->br[b]) * Lx / (2.0 * h)));
                if (ab < a1) a1 = ab;
            }
            double V[6];
            if (xn < 0.1) { V[0] = k->r1s; V[1] = k->r2s; V[2] = k->u1s; V[3] = 0.0; V[4] = k->p1; V[5] = 1.0 - eps; }
            else { V[0] = k->rho1; V[1] = k->rho2; V[2] = 0.0; V[3] = 0.0; V[4] = k->p0; V[5] = a1; }
            kap_p2c(c, V, k->U + ((size_t)j * c->nx + i) * 6);
        }
}

int hype_ic_shock_bubble(const hype_config *c, uint64_t seed, int nbubbles, double *U)
{
    if (!c || !U || c->system != HYPE_KAPILA_5EQN || nbubbles < 0 || nbubbles > 64) return HYPE_ERR_INVALID;
    rng_t r = {seed * 0x2545F4914F6CDD1Dull + 17};
    const double eps = 1e-6, p0 = 1e5, rho1 = 1000.0, rho2 = 1.0;
    const double h = (c->x_max - c->x_min) / c->nx;
    double bx[64], by[64], br[64];
    for (int b = 0; b < nbubbles; ++b) { br[b] = unif(&r, 0.1, 0.2); bx[b] = unif(&r, 0.4, 0.6); by[b] = unif(&r, 0.4, 0.6); }
    const double ratio = unif(&r, 10.0, 1000.0);
    const double p1 = ratio * p0;
    double r1s, u1s, r2s, u2s;
    rh_state(c->gamma1, c->pi1, p0, rho1, p1, &r1s, &u1s);   /* phase 1 carries the shock */
    rh_state(c->gamma2, c->pi2, p0, rho2, p1, &r2s, &u2s);   /* trace phase 2 compressed by the same jump */
    (void)u2s;
    sb_ctx k = {c, U, h, c->x_max - c->x_min, c->y_max - c->y_min, eps, p0, rho1, rho2, p1, r1s, u1s, r2s, nbubbles,
                {0}, {0}, {0}};
    memcpy(k.bx, bx, sizeof(double) * nbubbles);
    memcpy(k.by, by, sizeof(double) * nbubbles);
    memcpy(k.br, br, sizeof(double) * nbubbles);
    par_rows(c->nx, c->ny, sb_rows, &k);
    return HYPE_OK;
}

/* a smooth random field on the unit square: sum of 4 low Fourier modes, scaled to [lo, hi] */
typedef struct { double kx[4], ky[4], ph[4], amp[4]; } field_t;
static void field_init(field_t *f, rng_t *r)
{
    for (int m = 0; m < 4; ++m) {
        f->kx[m] = (double)(1 + (next_u64(r) % 3)); f->ky[m] = (double)(1 + (next_u64(r) % 3));
        f->ph[m] = unif(r, 0.0, 6.283185307179586); f->amp[m] = unif(r, 0.5, 1.0);
    }
}
static double field_at(const field_t *f, double x, double y, double lo, double hi)
{
    double s = 0.0, norm = 0.0;
    for (int m = 0; m < 4; ++m) {
        s += f->amp[m] * sin(6.283185307179586 * (f->kx[m] * x + f->ky[m] * y) + f->ph[m]);
        norm += f->amp[m];
    }
    return lo + (hi - lo) * 0.5 * (1.0 + s / norm);
}

typedef struct {
    const hype_config *c;
    double *U;
    double h, Lx, Ly, umax;
    double dx[8], dy[8], dr[8];
    field_t fr1, fr2, fu1, fv1, fu2, fv2, fp1, fp2;
} bn_ctx;
static void bn_rows(const void *ctx, int j0, int j1)
{
    const bn_ctx *K = (const bn_ctx *)ctx;
    const hype_config *c = K->c;
    const double h = K->h, Lx = K->Lx, Ly = K->Ly, umax = K->umax;
    for (int j = j0; j < j1; ++j)
        for (int i = 0; i < c->nx; ++i) {
            const double xn = ((i + 0.5) * h) / Lx, yn = ((j + 0.5) * h) / Ly;
            double a = 0.01;
            for (int k = 0; k < 8; ++k) {
                const double d = sqrt((xn - K->dx[k]) * (xn - K->dx[k]) + (yn - K->dy[k]) * (yn - K->dy[k]));
                a += 0.98 * 0.5 * (1.0 - tanh((d - K->dr[k]) * Lx / (2.0 * h)));
            }
            if (a > 0.99) a = 0.99;
            double V[9];
            V[0] = 1000.0 * field_at(&K->fr1, xn, yn, 0.5, 2.0);
            V[1] = field_at(&K->fu1, xn, yn, -umax, umax);
            V[2] = field_at(&K->fv1, xn, yn, -umax, umax);
            V[3] = field_at(&K->fp1, xn, yn, 1e5, 1e7);
            V[4] = 1.0 * field_at(&K->fr2, xn, yn, 0.5, 2.0);
            V[5] = field_at(&K->fu2, xn, yn, -umax, umax);
            V[6] = field_at(&K->fv2, xn, yn, -umax, umax);
            V[7] = field_at(&K->fp2, xn, yn, 1e5, 1e7);
            V[8] = a;
            bn_p2c(c, V, K->U + ((size_t)j * c->nx + i) * 9);
        }
}

int hype_ic_bn_discs(const hype_config *c, uint64_t seed, double *U)
{
    if (!c || !U || c->system != HYPE_BAER_NUNZIATO) return HYPE_ERR_INVALID;
    rng_t r = {seed * 0x9E3779B97F4A7C15ull + 3};
    const double h = (c->x_max - c->x_min) / c->nx;
    const double Lx = c->x_max - c->x_min, Ly = c->y_max - c->y_min;
    double dx[8], dy[8], dr[8];
    for (int k = 0; k < 8; ++k) { dx[k] = unif(&r, 0.1, 0.9); dy[k] = unif(&r, 0.1, 0.9); dr[k] = unif(&r, 0.04, 0.15); }
    field_t fr1, fr2, fu1, fv1, fu2, fv2, fp1, fp2;
    field_init(&fr1, &r); field_init(&fr2, &r); field_init(&fu1, &r); field_init(&fv1, &r);
    field_init(&fu2, &r); field_init(&fv2, &r); field_init(&fp1, &r); field_init(&fp2, &r);
    bn_ctx k = {c, U, h, Lx, Ly, 50.0 / sqrt(2.0) /* |u| <= 50 */, {0}, {0}, {0},
                fr1, fr2, fu1, fv1, fu2, fv2, fp1, fp2};
    memcpy(k.dx, dx, sizeof(dx));
    memcpy(k.dy, dy, sizeof(dy));
    memcpy(k.dr, dr, sizeof(dr));
    par_rows(c->nx, c->ny, bn_rows, &k);
    return HYPE_OK;
}

int hype_ic_euler_quadrants(const hype_config *c, uint64_t seed, double *U)
{
    if (!c || !U || c->system != HYPE_EULER) return HYPE_ERR_INVALID;
    rng_t r = {seed * 0xD1B54A32D192ED03ull + 5};
    double rho[4], p[4], u[4], v[4];
    for (int q = 0; q < 4; ++q) { rho[q] = unif(&r, 0.1, 1.5); p[q] = unif(&r, 0.03, 1.5); u[q] = unif(&r, -1.0, 1.0); v[q] = unif(&r, -1.0, 1.0); }
    const double h = (c->x_max - c->x_min) / c->nx;
    const double xm = 0.5 * (c->x_min + c->x_max), ym = 0.5 * (c->y_min + c->y_max);
    for (int j = 0; j < c->ny; ++j)
        for (int i = 0; i < c->nx; ++i) {
            const double x = c->x_min + (i + 0.5) * h, y = c->y_min + (j + 0.5) * h;
            const int q = (x >= xm ? 1 : 0) + (y >= ym ? 2 : 0);
            double V[4] = {rho[q], u[q], v[q], p[q]};
            eul_p2c(c, V, U + ((size_t)j * c->nx + i) * 4);
        }
    return HYPE_OK;
}

/* kapila_5eqn.c:527-562 with the 5x5 Gauss cell average of initialize_solution.c:41-72 */
int hype_ic_smooth_vortex(const hype_config *c, double *U)
{
    if (!c || !U || c->system != HYPE_KAPILA_5EQN) return HYPE_ERR_INVALID;
    static const double xg[5] = {0.0000000000000000, -0.2692346550528416, 0.2692346550528416, -0.4530899229693320, 0.4530899229693320};
    static const double wg[5] = {0.28444444444444444, 0.23931433524968326, 0.23931433524968326, 0.11846344252809456, 0.11846344252809456};
    const double h = (c->x_max - c->x_min) / c->nx;
    for (int j = 0; j < c->ny; ++j)
        for (int i = 0; i < c->nx; ++i) {
            const double xc = c->x_min + (i + 0.5) * h, yc = c->y_min + (j + 0.5) * h;
            double acc[6] = {0, 0, 0, 0, 0, 0};
            for (int l = 0; l < 5; ++l)
                for (int m = 0; m < 5; ++m) {
                    const double x = xc + h * xg[l], y = yc + h * xg[m];
                    const double omega = 3.14159265358979323846 / 3.0, r = sqrt(x * x + y * y);
                    double V[6], Q[6];
                    V[0] = 1000.0 + 0.1 * 1000.0 * sin(omega * (2.0 * x + y)) * cos(omega * (x - 2.0 * y));
                    V[1] = 1.0 + 0.1 * 1.0 * sin(omega * (x - 2.0 * y)) * cos(omega * (2.0 * x + y));
                    V[2] = 1.0; V[3] = 1.0; V[4] = 1.0;
                    V[5] = 0.25 + 0.5 * (0.75 - 0.25) * erfc((r / 1.0 - 1.0) / 0.3);
                    kap_p2c(c, V, Q);
                    for (int k = 0; k < 6; ++k) acc[k] += wg[l] * wg[m] * Q[k];
                }
            memcpy(U + ((size_t)j * c->nx + i) * 6, acc, sizeof(acc));
        }
    return HYPE_OK;
}
