/*
 * hype_oracle_ic.c -- the seeded initial states of the benchmark workloads, for
 * the CPU side of the checks.  TEST INFRASTRUCTURE ONLY.
 *
 * The product builds these states in its own library (include/hype_ic.h); the
 * CPU baseline and the reference arm of bench.py must not load that library,
 * so the oracle carries its own statement of the same generators, and
 * tests/test_oracle_ic.py holds the two to the same bits.  What is generated:
 *   shock_bubble  Kapila: liquid at rest (p 1e5, rho 1000 / 1) with gas discs
 *                 (alpha_1 down to 1e-6, tanh edge two cells wide) and a planar
 *                 stiffened-gas Rankine-Hugoniot shock in x < 0.1;
 *   bn_discs      Baer-Nunziato: alpha_1 from 8 tanh discs in [0.01, 0.99],
 *                 smooth random densities, velocities (|u| <= 50) and pressures;
 *   euler_quadrants  four constant quadrants.
 * The random stream is splitmix64; conversions are exact, and libm supplies
 * sqrt, tanh and sin, so the bits do not depend on the platform's compiler as
 * long as it keeps every operation separately rounded (-ffp-contract=off).
 * The primitive-to-conserved maps are the reference's PDEPrim2Cons
 * (kapila_5eqn.c:41-61, baer_nunziato.c:47-60, euler.c:29-38).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include "hype_oracle.h"

typedef struct { uint64_t state; } splitmix;

static uint64_t sm_next(splitmix *g)
{
    uint64_t z = (g->state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
/* uniform on [lo, hi): the top 53 bits as a fraction of 2^53 */
static double sm_uniform(splitmix *g, double lo, double hi)
{
    const double f = (double)(sm_next(g) >> 11) * (1.0 / 9007199254740992.0);
    return lo + (hi - lo) * f;
}

static void kapila_cons(const hyo_config *c, const double *V, double *Q)
{
    const double a1 = V[5], a2 = 1.0 - a1;
    const double rho = a1 * V[0] + a2 * V[1];
    const double G1m1 = c->gamma1 - 1.0, G2m1 = c->gamma2 - 1.0;
    const double e = (V[4] * (a1 * G2m1 + a2 * G1m1) + a1 * c->gamma1 * c->pi1 * G2m1 + a2 * c->gamma2 * c->pi2 * G1m1) /
                     (G1m1 * G2m1);
    Q[0] = a1 * V[0];
    Q[1] = a2 * V[1];
    Q[2] = rho * V[2];
    Q[3] = rho * V[3];
    Q[4] = e + 0.5 * rho * (V[2] * V[2] + V[3] * V[3]);
    Q[5] = a1;
}

static void bn_cons(const hyo_config *c, const double *V, double *Q)
{
    Q[0] = V[8] * V[0];
    Q[1] = Q[0] * V[1];
    Q[2] = Q[0] * V[2];
    Q[3] = Q[0] * (0.5 * (V[1] * V[1] + V[2] * V[2]) + (V[3] + c->gamma1 * c->pi1) / (V[0] * (c->gamma1 - 1.0)));
    Q[4] = (1.0 - V[8]) * V[4];
    Q[5] = Q[4] * V[5];
    Q[6] = Q[4] * V[6];
    Q[7] = Q[4] * (0.5 * (V[5] * V[5] + V[6] * V[6]) + (V[7] + c->gamma2 * c->pi2) / (V[4] * (c->gamma2 - 1.0)));
    Q[8] = V[8];
}

static void euler_cons(const hyo_config *c, const double *V, double *Q)
{
    Q[0] = V[0];
    Q[1] = V[0] * V[1];
    Q[2] = V[0] * V[2];
    Q[3] = 0.5 * V[0] * (V[1] * V[1] + V[2] * V[2]) + V[3] / (c->gamma1 - 1.0);
}

/* density and velocity behind a shock of pressure p1 running into a stiffened gas
 * (gamma g, P_inf pi) at rest at (p0, rho0): Rankine-Hugoniot with pbar = p + pi */
static void shocked(double g, double pi, double p0, double rho0, double p1, double *rho1, double *u1)
{
    const double q0 = p0 + pi, q1 = p1 + pi;
    const double ratio = ((g + 1.0) * q1 + (g - 1.0) * q0) / ((g - 1.0) * q1 + (g + 1.0) * q0);
    *rho1 = rho0 * ratio;
    *u1 = sqrt((p1 - p0) * (1.0 / rho0 - 1.0 / *rho1));
}

int hyo_ic_shock_bubble(const hyo_config *c, uint64_t seed, int nbubbles, double *U)
{
    if (!c || !U || c->system != HYO_KAPILA || nbubbles < 0 || nbubbles > 64) return HYO_ERR_CONFIG;
    splitmix g = {seed * 0x2545F4914F6CDD1Dull + 17};
    const double eps = 1e-6, p0 = 1e5, rho_l = 1000.0, rho_g = 1.0;
    const double h = (c->x_max - c->x_min) / c->nx;
    const double Lx = c->x_max - c->x_min, Ly = c->y_max - c->y_min;
    double cx[64], cy[64], rad[64];
    for (int b = 0; b < nbubbles; ++b) {
        rad[b] = sm_uniform(&g, 0.1, 0.2);
        cx[b] = sm_uniform(&g, 0.4, 0.6);
        cy[b] = sm_uniform(&g, 0.4, 0.6);
    }
    const double p1 = sm_uniform(&g, 10.0, 1000.0) * p0;
    double rl1, ul1, rg1, ug1;
    shocked(c->gamma1, c->pi1, p0, rho_l, p1, &rl1, &ul1);
    shocked(c->gamma2, c->pi2, p0, rho_g, p1, &rg1, &ug1);
    (void)ug1;
    for (int j = 0; j < c->ny; ++j) {
        for (int i = 0; i < c->nx; ++i) {
            const double x = c->x_min + (i + 0.5) * h, y = c->y_min + (j + 0.5) * h;
            const double xu = (x - c->x_min) / Lx, yu = (y - c->y_min) / Ly;
            double alpha = 1.0 - eps;
            for (int b = 0; b < nbubbles; ++b) {
                const double r = sqrt((xu - cx[b]) * (xu - cx[b]) + (yu - cy[b]) * (yu - cy[b]));
                const double edge = eps + (1.0 - 2.0 * eps) * 0.5 * (1.0 + tanh((r - rad[b]) * Lx / (2.0 * h)));
                if (edge < alpha) alpha = edge;
            }
            double V[6];
            if (xu < 0.1) {
                V[0] = rl1; V[1] = rg1; V[2] = ul1; V[3] = 0.0; V[4] = p1; V[5] = 1.0 - eps;
            } else {
                V[0] = rho_l; V[1] = rho_g; V[2] = 0.0; V[3] = 0.0; V[4] = p0; V[5] = alpha;
            }
            kapila_cons(c, V, U + ((size_t)j * c->nx + i) * 6);
        }
    }
    return HYO_OK;
}

/* smooth random field: four low Fourier modes mapped onto [lo, hi] */
typedef struct { double kx[4], ky[4], phase[4], amp[4]; } modes;

static void modes_draw(modes *f, splitmix *g)
{
    for (int q = 0; q < 4; ++q) {
        f->kx[q] = (double)(1 + (sm_next(g) % 3));
        f->ky[q] = (double)(1 + (sm_next(g) % 3));
        f->phase[q] = sm_uniform(g, 0.0, 6.283185307179586);
        f->amp[q] = sm_uniform(g, 0.5, 1.0);
    }
}
static double modes_at(const modes *f, double x, double y, double lo, double hi)
{
    double acc = 0.0, wsum = 0.0;
    for (int q = 0; q < 4; ++q) {
        acc += f->amp[q] * sin(6.283185307179586 * (f->kx[q] * x + f->ky[q] * y) + f->phase[q]);
        wsum += f->amp[q];
    }
    return lo + (hi - lo) * 0.5 * (1.0 + acc / wsum);
}

int hyo_ic_bn_discs(const hyo_config *c, uint64_t seed, double *U)
{
    if (!c || !U || c->system != HYO_BN) return HYO_ERR_CONFIG;
    splitmix g = {seed * 0x9E3779B97F4A7C15ull + 3};
    const double h = (c->x_max - c->x_min) / c->nx;
    const double Lx = c->x_max - c->x_min, Ly = c->y_max - c->y_min;
    double cx[8], cy[8], rad[8];
    for (int k = 0; k < 8; ++k) {
        cx[k] = sm_uniform(&g, 0.1, 0.9);
        cy[k] = sm_uniform(&g, 0.1, 0.9);
        rad[k] = sm_uniform(&g, 0.04, 0.15);
    }
    /* drawn in this order: rho1, rho2, u1, v1, u2, v2, p1, p2 */
    modes f_r1, f_r2, f_u1, f_v1, f_u2, f_v2, f_p1, f_p2;
    modes_draw(&f_r1, &g); modes_draw(&f_r2, &g); modes_draw(&f_u1, &g); modes_draw(&f_v1, &g);
    modes_draw(&f_u2, &g); modes_draw(&f_v2, &g); modes_draw(&f_p1, &g); modes_draw(&f_p2, &g);
    const double umax = 50.0 / sqrt(2.0);
    for (int j = 0; j < c->ny; ++j) {
        for (int i = 0; i < c->nx; ++i) {
            const double xu = ((i + 0.5) * h) / Lx, yu = ((j + 0.5) * h) / Ly;
            double alpha = 0.01;
            for (int k = 0; k < 8; ++k) {
                const double r = sqrt((xu - cx[k]) * (xu - cx[k]) + (yu - cy[k]) * (yu - cy[k]));
                alpha += 0.98 * 0.5 * (1.0 - tanh((r - rad[k]) * Lx / (2.0 * h)));
            }
            if (alpha > 0.99) alpha = 0.99;
            double V[9];
            V[0] = 1000.0 * modes_at(&f_r1, xu, yu, 0.5, 2.0);
            V[1] = modes_at(&f_u1, xu, yu, -umax, umax);
            V[2] = modes_at(&f_v1, xu, yu, -umax, umax);
            V[3] = modes_at(&f_p1, xu, yu, 1e5, 1e7);
            V[4] = 1.0 * modes_at(&f_r2, xu, yu, 0.5, 2.0);
            V[5] = modes_at(&f_u2, xu, yu, -umax, umax);
            V[6] = modes_at(&f_v2, xu, yu, -umax, umax);
            V[7] = modes_at(&f_p2, xu, yu, 1e5, 1e7);
            V[8] = alpha;
            bn_cons(c, V, U + ((size_t)j * c->nx + i) * 9);
        }
    }
    return HYO_OK;
}

int hyo_ic_euler_quadrants(const hyo_config *c, uint64_t seed, double *U)
{
    if (!c || !U || c->system != HYO_EULER) return HYO_ERR_CONFIG;
    splitmix g = {seed * 0xD1B54A32D192ED03ull + 5};
    double rho[4], p[4], u[4], v[4];
    for (int q = 0; q < 4; ++q) {
        rho[q] = sm_uniform(&g, 0.1, 1.5);
        p[q] = sm_uniform(&g, 0.03, 1.5);
        u[q] = sm_uniform(&g, -1.0, 1.0);
        v[q] = sm_uniform(&g, -1.0, 1.0);
    }
    const double h = (c->x_max - c->x_min) / c->nx;
    const double xm = 0.5 * (c->x_min + c->x_max), ym = 0.5 * (c->y_min + c->y_max);
    for (int j = 0; j < c->ny; ++j) {
        for (int i = 0; i < c->nx; ++i) {
            const double x = c->x_min + (i + 0.5) * h, y = c->y_min + (j + 0.5) * h;
            const int q = (x >= xm ? 1 : 0) + (y >= ym ? 2 : 0);
            const double V[4] = {rho[q], u[q], v[q], p[q]};
            euler_cons(c, V, U + ((size_t)j * c->nx + i) * 4);
        }
    }
    return HYO_OK;
}
