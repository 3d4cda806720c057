/*
 * hype_oracle.c -- CPU restatement of HyPE-2D's RHSFunctionPrim / RHSFunction
 * and its SSP-RK time loop.  TEST INFRASTRUCTURE ONLY (see hype_oracle.h).
 *
 * Every floating-point expression keeps the operand order of the reference C
 * it restates (file:line cited at each function), and the file is compiled
 * with -ffp-contract=off, so results are bit-identical to the reference's own
 * code.  The surrounding structure is this project's: one pass converts and
 * ghost-fills a padded array, one pass reconstructs every cell of the 1-cell
 * ring into a coefficient array, faces are evaluated from the coefficients on
 * demand, and the divergence is assembled per cell.
 */
#include "hype_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXV 9       /* largest nVar (Baer-Nunziato) */
#define MAXDOF 10    /* nDOF for N = 3 */
#define GH 3         /* ghost width of the DMDA (hype.c:117) */

/* hype.h:50-62 */
static const double PRS_FLOOR = 1.0e-12;
static const double RHO_FLOOR = 1.0e-14;
static const double SMALL_NUM = 1.0e-12;
static const double R1_6 = 1. / 6.;
static const double R13_3 = 13. / 3.;
static const double R7_6 = 7. / 6.;
static const double R11_120 = 11. / 120.;
static const double R1_12 = 1. / 12.;
static const double R41_60 = 41. / 60.;

typedef struct { double g1, g2, pi1, pi2; int fix_p2; } eos_t;

static _Thread_local long tl_pad_fallbacks = 0;
long hyo_last_pad_fallbacks(void) { return tl_pad_fallbacks; }

int hyo_nvar(int system)
{
    switch (system) { case HYO_EULER: return 4; case HYO_KAPILA: return 6; case HYO_BN: return 9; default: return 0; }
}

/* ===================================================================== */
/* Kapila five-equation model, kapila_5eqn.c                              */
/* ===================================================================== */

/* kapila_5eqn.c:14-35 */
static void kap_cons2prim(const eos_t *e, const double *Q, double *V)
{
    double alpha_1 = Q[5];
    double alpha_2 = 1.0 - alpha_1;
    double rho = Q[0] + Q[1];
    double u = Q[2] / rho;
    double v = Q[3] / rho;
    double E = Q[4];
    double ei = E - 0.5 * rho * (u * u + v * v);
    double G1m1 = e->g1 - 1.0;
    double G2m1 = e->g2 - 1.0;
    double p = (ei * G1m1 * G2m1 - alpha_1 * e->g1 * e->pi1 * G2m1 - alpha_2 * e->g2 * e->pi2 * G1m1) / (alpha_1 * G2m1 + alpha_2 * G1m1);
    V[0] = Q[0] / alpha_1;
    V[1] = Q[1] / alpha_2;
    V[2] = u;
    V[3] = v;
    V[4] = p;
    V[5] = alpha_1;
}

/* kapila_5eqn.c:41-61 */
static void kap_prim2cons(const eos_t *e, const double *V, double *Q)
{
    double alpha_1 = V[5];
    double alpha_2 = 1.0 - alpha_1;
    double rho = alpha_1 * V[0] + alpha_2 * V[1];
    double u = V[2], v = V[3], p = V[4];
    double G1m1 = e->g1 - 1.0;
    double G2m1 = e->g2 - 1.0;
    double ei = (p * (alpha_1 * G2m1 + alpha_2 * G1m1) + alpha_1 * e->g1 * e->pi1 * G2m1 + alpha_2 * e->g2 * e->pi2 * G1m1) / (G1m1 * G2m1);
    double E = ei + 0.5 * rho * (u * u + v * v);
    Q[0] = alpha_1 * V[0];
    Q[1] = alpha_2 * V[1];
    Q[2] = rho * V[2];
    Q[3] = rho * V[3];
    Q[4] = E;
    Q[5] = alpha_1;
}

/* kapila_5eqn.c:326-371; *bad set where the reference aborts (353-357) */
static double kap_flux_prim(const eos_t *e, const double *V, double nx, double ny, double *F, int *bad)
{
    double alpha_1 = V[5];
    double alpha_2 = 1.0 - alpha_1;
    double rho_1 = V[0], rho_2 = V[1];
    double rho = alpha_1 * rho_1 + alpha_2 * rho_2;
    double u = V[2], v = V[3], p = V[4];
    double G1m1 = e->g1 - 1.0;
    double G2m1 = e->g2 - 1.0;
    double ei = (p * (alpha_1 * G2m1 + alpha_2 * G1m1) + alpha_1 * e->g1 * e->pi1 * G2m1 + alpha_2 * e->g2 * e->pi2 * G1m1) / (G1m1 * G2m1);
    double E = ei + 0.5 * rho * (u * u + v * v);
    double un = u * nx + v * ny;
    double a1_sq = e->g1 * (p + e->pi1) / rho_1;
    double a2_sq = e->g2 * (p + e->pi2) / rho_2;
    double a_sq = (rho_1 * a1_sq * rho_2 * a2_sq) / (rho * (alpha_2 * rho_1 * a1_sq + alpha_1 * rho_2 * a2_sq));
    if (a_sq < PRS_FLOOR) *bad = 1;
    F[0] = alpha_1 * rho_1 * un;
    F[1] = alpha_2 * rho_2 * un;
    F[2] = rho * u * un + p * nx;
    F[3] = rho * v * un + p * ny;
    F[4] = (E + p) * un;
    F[5] = 0.0;
    return fabs(un) + sqrt(a_sq);
}

/* kapila_5eqn.c:417-444 */
static void kap_ncp_prim(const eos_t *e, const double *V, const double *gx, const double *gy, double *B)
{
    double alpha_1 = V[5];
    double alpha_2 = 1.0 - alpha_1;
    double rho_1 = V[0], rho_2 = V[1], u = V[2], v = V[3], p = V[4];
    double phi_x = gx[5], phi_y = gy[5];
    double u_x = gx[2], v_y = gy[3];
    double a_1_sq = e->g1 * (p + e->pi1) / rho_1;
    double a_2_sq = e->g2 * (p + e->pi2) / rho_2;
    double K = (alpha_1 * alpha_2 * (rho_2 * a_2_sq - rho_1 * a_1_sq)) / (alpha_1 * rho_2 * a_2_sq + alpha_2 * rho_1 * a_1_sq);
    B[0] = 0.0; B[1] = 0.0; B[2] = 0.0; B[3] = 0.0; B[4] = 0.0;
    B[5] = u * phi_x + v * phi_y - K * (u_x + v_y);
}

/* kapila_5eqn.c:450-479 */
static int kap_pad_prim(const eos_t *e, const double *V)
{
    double alpha_1 = V[5];
    double alpha_2 = 1.0 - alpha_1;
    double rho_1 = V[0], rho_2 = V[1];
    double rho = alpha_1 * rho_1 + alpha_2 * rho_2;
    double p = V[4];
    double a1_sq = e->g1 * (p + e->pi1) / rho_1;
    double a2_sq = e->g2 * (p + e->pi2) / rho_2;
    double a_sq = (rho_1 * a1_sq * rho_2 * a2_sq) / (rho * (alpha_2 * rho_1 * a1_sq + alpha_1 * rho_2 * a2_sq));
    if (rho < RHO_FLOOR) return 0;
    if (a_sq < PRS_FLOOR) return 0;
    if (alpha_1 < 0.0 || alpha_1 > 1.0) return 0;
    return 1;
}

/* kapila_5eqn.c:485-513 (time-independent jet profile) */
static void kap_inlet_prim(const eos_t *e, double x, double y, double *V)
{
    (void)x;
    const double M = 2.0, rho_air = 1.0, rho_water = 1000.0, P = 1.013;
    const double U_avg = M * sqrt(e->g2 * P / rho_air);
    const double phi_R = 1.0 - 1.0e-6, phi_L = 1.0e-6;
    const double PHI = 0.5 * (phi_R + phi_L);
    const double dif_phi = (phi_L - phi_R) / 2.0;
    const double h = 30.0 / 500.0;
    const double epsilon = 3.0 * h;
    const double r_0 = 1.0;
    double r = fabs(y);
    V[0] = rho_water;
    V[1] = rho_air;
    V[2] = (r < 1.0) ? 2.0 * U_avg * (1.0 - y * y) : 0.0;
    V[3] = 0.0;
    V[4] = P;
    V[5] = PHI + dif_phi * tanh(-(r - r_0) / epsilon);
}

/* kapila_5eqn.c:67-113 (conservative input) */
static double kap_flux_cons(const eos_t *e, const double *Q, double nx, double ny, double *F, int *bad)
{
    double alpha_1 = Q[5];
    double alpha_2 = 1.0 - alpha_1;
    double rho_1 = Q[0] / alpha_1;
    double rho_2 = Q[1] / alpha_2;
    double rho = Q[0] + Q[1];
    double u = Q[2] / rho, v = Q[3] / rho, E = Q[4];
    double ei = E - 0.5 * rho * (u * u + v * v);
    double G1m1 = e->g1 - 1.0, G2m1 = e->g2 - 1.0;
    double p = (ei * G1m1 * G2m1 - alpha_1 * e->g1 * e->pi1 * G2m1 - alpha_2 * e->g2 * e->pi2 * G1m1) / (alpha_1 * G2m1 + alpha_2 * G1m1);
    double un = u * nx + v * ny;
    double a1_sq = e->g1 * (p + e->pi1) / rho_1;
    double a2_sq = e->g2 * (p + e->pi2) / rho_2;
    double a_sq = (rho_1 * a1_sq * rho_2 * a2_sq) / (rho * (alpha_2 * rho_1 * a1_sq + alpha_1 * rho_2 * a2_sq));
    if (a_sq < PRS_FLOOR) *bad = 1;
    F[0] = alpha_1 * rho_1 * un;
    F[1] = alpha_2 * rho_2 * un;
    F[2] = rho * u * un + p * nx;
    F[3] = rho * v * un + p * ny;
    F[4] = (E + p) * un;
    F[5] = 0.0;
    return fabs(un) + sqrt(a_sq);
}

/* kapila_5eqn.c:164-198 */
static void kap_ncp_cons(const eos_t *e, const double *Q, const double *gx, const double *gy, double *B)
{
    double alpha_1 = Q[5];
    double alpha_2 = 1.0 - alpha_1;
    double rho_1 = Q[0] / alpha_1;
    double rho_2 = Q[1] / alpha_2;
    double rho = Q[0] + Q[1];
    double irho = 1.0 / rho;
    double u = Q[2] / rho, v = Q[3] / rho, E = Q[4];
    double ei = E - 0.5 * rho * (u * u + v * v);
    double G1m1 = e->g1 - 1.0, G2m1 = e->g2 - 1.0;
    double p = (ei * G1m1 * G2m1 - alpha_1 * e->g1 * e->pi1 * G2m1 - alpha_2 * e->g2 * e->pi2 * G1m1) / (alpha_1 * G2m1 + alpha_2 * G1m1);
    double a1_sq = e->g1 * (p + e->pi1) / rho_1;
    double a2_sq = e->g2 * (p + e->pi2) / rho_2;
    double K = alpha_1 * alpha_2 * (rho_2 * a2_sq - rho_1 * a1_sq) / (alpha_1 * rho_2 * a2_sq + alpha_2 * rho_1 * a1_sq);
    double alpha1_x = gx[5], alpha1_y = gy[5];
    double u_x = irho * irho * (gx[2] * rho - Q[2] * (gx[0] + gx[1]));
    double v_y = irho * irho * (gy[3] * rho - Q[3] * (gy[0] + gy[1]));
    B[0] = 0.0; B[1] = 0.0; B[2] = 0.0; B[3] = 0.0; B[4] = 0.0;
    B[5] = u * alpha1_x + v * alpha1_y - K * (u_x + v_y);
}

/* kapila_5eqn.c:247-283 -- the alpha test rejects every alpha_1 != 1 (line 278) */
static int kap_pad_cons(const eos_t *e, const double *Q)
{
    double alpha_1 = Q[5];
    double alpha_2 = 1.0 - alpha_1;
    double rho_1 = Q[0] / alpha_1;
    double rho_2 = Q[1] / alpha_2;
    double rho = Q[0] + Q[1];
    double u = Q[2] / rho, v = Q[3] / rho, E = Q[4];
    double ei = E - 0.5 * rho * (u * u + v * v);
    double G1m1 = e->g1 - 1.0, G2m1 = e->g2 - 1.0;
    double p = (ei * G1m1 * G2m1 - alpha_1 * e->g1 * e->pi1 * G2m1 - alpha_2 * e->g2 * e->pi2 * G1m1) / (alpha_1 * G2m1 + alpha_2 * G1m1);
    double a1_sq = e->g1 * (p + e->pi1) / rho_1;
    double a2_sq = e->g2 * (p + e->pi2) / rho_2;
    double a_sq = (rho_1 * a1_sq * rho_2 * a2_sq) / (rho * (alpha_2 * rho_1 * a1_sq + alpha_1 * rho_2 * a2_sq));
    if (rho < RHO_FLOOR) return 0;
    if (a_sq < PRS_FLOOR) return 0;
    if (alpha_1 < 1.0 || alpha_1 > 1.0) return 0;
    return 1;
}

/* kapila_5eqn.c:377-411: viscous flux in the normal direction from primitive
 * values V and gradients g[c][dim]; returns the viscous eigenvalue */
static double kap_visc_prim(const double *V, const double g[][2], double nx, double ny, double mu1, double mu2, double *F)
{
    double r2_3 = 2. / 3., r4_3 = 4. / 3.;
    double phi = V[5];
    double mu = phi * mu1 + (1.0 - phi) * mu2;
    double u = V[2], v = V[3];
    double u_x = g[2][0], u_y = g[2][1], v_x = g[3][0], v_y = g[3][1];
    double div_v = u_x + v_y;
    double tau_xx = mu * (2.0 * u_x - r2_3 * div_v);
    double tau_xy = mu * (u_y + v_x);
    double tau_yy = mu * (2.0 * v_y - r2_3 * div_v);
    F[0] = 0.0;
    F[1] = 0.0;
    F[2] = -nx * tau_xx - ny * tau_xy;
    F[3] = -nx * tau_xy - ny * tau_yy;
    F[4] = -nx * (u * tau_xx + v * tau_xy) - ny * (u * tau_xy + v * tau_yy);
    F[5] = 0.0;
    return r4_3 * mu / V[0];
}

/* kapila_5eqn.c:119-158: the same from conserved values Q and their gradients */
static double kap_visc_cons(const double *Q, const double g[][2], double nx, double ny, double mu1, double mu2, double *F)
{
    double r2_3 = 2. / 3., r4_3 = 4. / 3.;
    double phi = Q[5];
    double mu = phi * mu1 + (1.0 - phi) * mu2;
    double irho = 1.0 / (Q[0] + Q[1]);
    double u = irho * Q[2];
    double v = irho * Q[3];
    double rho_x = g[0][0] + g[1][0];
    double rho_y = g[0][1] + g[1][1];
    double u_x = irho * (g[2][0] - u * rho_x);
    double u_y = irho * (g[2][1] - u * rho_y);
    double v_x = irho * (g[3][0] - v * rho_x);
    double v_y = irho * (g[3][1] - v * rho_y);
    double div_v = u_x + v_y;
    double tau_xx = mu * (2.0 * u_x - r2_3 * div_v);
    double tau_xy = mu * (u_y + v_x);
    double tau_yy = mu * (2.0 * v_y - r2_3 * div_v);
    F[0] = 0.0;
    F[1] = 0.0;
    F[2] = -nx * tau_xx - ny * tau_xy;
    F[3] = -nx * tau_xy - ny * tau_yy;
    F[4] = -nx * (u * tau_xx + v * tau_xy) - ny * (u * tau_xy + v * tau_yy);
    F[5] = 0.0;
    return r4_3 * mu * irho;
}

/* ===================================================================== */
/* Baer-Nunziato, baer_nunziato.c                                         */
/* ===================================================================== */

/* baer_nunziato.c:14-41 */
static void bn_cons2prim(const eos_t *e, const double *Q, double *V)
{
    double phi_1 = Q[8];
    double phi_2 = 1.0 - Q[8];
    double rho_1 = Q[0] / phi_1;
    double rho_2 = Q[4] / phi_2;
    double u_1 = Q[1] / Q[0], v_1 = Q[2] / Q[0];
    double u_2 = Q[5] / Q[4], v_2 = Q[6] / Q[4];
    double E_1 = Q[3] / phi_1;
    double E_2 = Q[7] / phi_2;
    double p_1 = (e->g1 - 1.0) * (E_1 - 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1)) - e->g1 * e->pi1;
    double p_2 = (e->g2 - 1.0) * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e->g2 * e->pi2;
    V[0] = rho_1; V[1] = u_1; V[2] = v_1; V[3] = p_1;
    V[4] = rho_2; V[5] = u_2; V[6] = v_2; V[7] = p_2;
    V[8] = phi_1;
}

/* baer_nunziato.c:47-60 */
static void bn_prim2cons(const eos_t *e, const double *V, double *Q)
{
    Q[0] = V[8] * V[0];
    Q[1] = Q[0] * V[1];
    Q[2] = Q[0] * V[2];
    Q[3] = Q[0] * (0.5 * (V[1] * V[1] + V[2] * V[2]) + (V[3] + e->g1 * e->pi1) / (V[0] * (e->g1 - 1.0)));
    Q[4] = (1.0 - V[8]) * V[4];
    Q[5] = Q[4] * V[5];
    Q[6] = Q[4] * V[6];
    Q[7] = Q[4] * (0.5 * (V[5] * V[5] + V[6] * V[6]) + (V[7] + e->g2 * e->pi2) / (V[4] * (e->g2 - 1.0)));
    Q[8] = V[8];
}

/* baer_nunziato.c:256-321.  The reference takes the phase-2 pressure from
 * V[8] (alpha_1, line 271); fix_p2 selects V[7] instead. */
static double bn_flux_prim(const eos_t *e, const double *V, double nx, double ny, double *F, int *bad)
{
    double phi_1 = V[8];
    double phi_2 = 1.0 - V[8];
    double rho_1 = V[0], rho_2 = V[4];
    double u_1 = V[1], v_1 = V[2];
    double u_2 = V[5], v_2 = V[6];
    double p_1 = V[3];
    double p_2 = e->fix_p2 ? V[7] : V[8];
    double E_1 = (p_1 + e->g1 * e->pi1) / (e->g1 - 1.0) + 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1);
    double E_2 = (p_2 + e->g2 * e->pi2) / (e->g2 - 1.0) + 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2);
    double un_1 = nx * u_1 + ny * v_1;
    double un_2 = nx * u_2 + ny * v_2;
    if (rho_1 < RHO_FLOOR) *bad = 1;
    if (rho_2 < RHO_FLOOR) *bad = 1;
    if ((p_1 + e->pi1) < PRS_FLOOR) *bad = 1;
    if ((p_2 + e->pi2) < PRS_FLOOR) *bad = 1;
    F[0] = phi_1 * rho_1 * un_1;
    F[1] = phi_1 * (rho_1 * u_1 * un_1 + nx * p_1);
    F[2] = phi_1 * (rho_1 * v_1 * un_1 + ny * p_1);
    F[3] = phi_1 * un_1 * (E_1 + p_1);
    F[4] = phi_2 * rho_2 * un_2;
    F[5] = phi_2 * (rho_2 * u_2 * un_2 + nx * p_2);
    F[6] = phi_2 * (rho_2 * v_2 * un_2 + ny * p_2);
    F[7] = phi_2 * un_2 * (E_2 + p_2);
    F[8] = 0.0;
    double s_1 = fabs(un_1) + sqrt(e->g1 * (p_1 + e->pi1) / rho_1);
    double s_2 = fabs(un_2) + sqrt(e->g2 * (p_2 + e->pi2) / rho_2);
    return (s_1 < s_2) ? s_2 : s_1;
}

/* baer_nunziato.c:327-344 (u_I = u_1, p_I = p_2) */
static void bn_ncp_prim(const eos_t *e, const double *V, const double *gx, const double *gy, double *B)
{
    (void)e;
    double u_I = V[1], v_I = V[2];
    double p_I = V[7];
    double phi_x = gx[8], phi_y = gy[8];
    B[0] = 0.0;
    B[1] = -p_I * phi_x;
    B[2] = -p_I * phi_y;
    B[3] = -p_I * (u_I * phi_x + v_I * phi_y);
    B[4] = 0.0;
    B[5] = p_I * phi_x;
    B[6] = p_I * phi_y;
    B[7] = p_I * (u_I * phi_x + v_I * phi_y);
    B[8] = u_I * phi_x + v_I * phi_y;
}

/* baer_nunziato.c:350-385 */
static int bn_pad_prim(const eos_t *e, const double *V)
{
    int pad = 1;
    double phi_1 = V[8];
    double rho_1 = V[0], rho_2 = V[4];
    double p_1 = V[3], p_2 = V[7];
    if (rho_1 < RHO_FLOOR) pad = 0;
    if (rho_2 < RHO_FLOOR) pad = 0;
    if ((p_1 + e->pi1) < PRS_FLOOR) pad = 0;
    if ((p_2 + e->pi2) < PRS_FLOOR) pad = 0;
    if (phi_1 < 0.0 || phi_1 > 1.0) pad = 0;
    return pad;
}

/* baer_nunziato.c:66-131 */
static double bn_flux_cons(const eos_t *e, const double *Q, double nx, double ny, double *F, int *bad)
{
    double phi_1 = Q[8];
    double phi_2 = 1.0 - Q[8];
    double rho_1 = Q[0] / phi_1;
    double rho_2 = Q[4] / phi_2;
    double u_1 = Q[1] / Q[0], v_1 = Q[2] / Q[0];
    double u_2 = Q[5] / Q[4], v_2 = Q[6] / Q[4];
    double E_1 = Q[3] / phi_1;
    double E_2 = Q[7] / phi_2;
    double p_1 = (e->g1 - 1.0) * (E_1 - 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1)) - e->g1 * e->pi1;
    double p_2 = (e->g2 - 1.0) * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e->g2 * e->pi2;
    double un_1 = nx * u_1 + ny * v_1;
    double un_2 = nx * u_2 + ny * v_2;
    if (rho_1 < RHO_FLOOR) *bad = 1;
    if (rho_2 < RHO_FLOOR) *bad = 1;
    if ((p_1 + e->pi1) < PRS_FLOOR) *bad = 1;
    if ((p_2 + e->pi2) < PRS_FLOOR) *bad = 1;
    F[0] = phi_1 * rho_1 * un_1;
    F[1] = phi_1 * (rho_1 * u_1 * un_1 + nx * p_1);
    F[2] = phi_1 * (rho_1 * v_1 * un_1 + ny * p_1);
    F[3] = phi_1 * un_1 * (E_1 + p_1);
    F[4] = phi_2 * rho_2 * un_2;
    F[5] = phi_2 * (rho_2 * u_2 * un_2 + nx * p_2);
    F[6] = phi_2 * (rho_2 * v_2 * un_2 + ny * p_2);
    F[7] = phi_2 * un_2 * (E_2 + p_2);
    F[8] = 0.0;
    double s_1 = fabs(un_1) + sqrt(e->g1 * (p_1 + e->pi1) / rho_1);
    double s_2 = fabs(un_2) + sqrt(e->g2 * (p_2 + e->pi2) / rho_2);
    return (s_1 < s_2) ? s_2 : s_1;
}

/* baer_nunziato.c:137-165 */
static void bn_ncp_cons(const eos_t *e, const double *Q, const double *gx, const double *gy, double *B)
{
    double phi_2 = 1.0 - Q[8];
    double rho_2 = Q[4] / phi_2;
    double u_1 = Q[1] / Q[0], v_1 = Q[2] / Q[0];
    double u_2 = Q[5] / Q[4], v_2 = Q[6] / Q[4];
    double E_2 = Q[7] / phi_2;
    double p_I = (e->g2 - 1.0) * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e->g2 * e->pi2;
    double phi_x = gx[8], phi_y = gy[8];
    B[0] = 0.0;
    B[1] = -p_I * phi_x;
    B[2] = -p_I * phi_y;
    B[3] = -p_I * (u_1 * phi_x + v_1 * phi_y);
    B[4] = 0.0;
    B[5] = p_I * phi_x;
    B[6] = p_I * phi_y;
    B[7] = p_I * (u_1 * phi_x + v_1 * phi_y);
    B[8] = u_1 * phi_x + v_1 * phi_y;
}

/* baer_nunziato.c:207-250 */
static int bn_pad_cons(const eos_t *e, const double *Q)
{
    int pad = 1;
    double phi_1 = Q[8];
    double phi_2 = 1.0 - Q[8];
    double rho_1 = Q[0] / phi_1;
    double rho_2 = Q[4] / phi_2;
    double u_1 = Q[1] / Q[0], v_1 = Q[2] / Q[0];
    double u_2 = Q[5] / Q[4], v_2 = Q[6] / Q[4];
    double E_1 = Q[3] / phi_1;
    double E_2 = Q[7] / phi_2;
    double p_1 = (e->g1 - 1.0) * (E_1 - 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1)) - e->g1 * e->pi1;
    double p_2 = (e->g2 - 1.0) * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e->g2 * e->pi2;
    if (rho_1 < RHO_FLOOR) pad = 0;
    if (rho_2 < RHO_FLOOR) pad = 0;
    if ((p_1 + e->pi1) < PRS_FLOOR) pad = 0;
    if ((p_2 + e->pi2) < PRS_FLOOR) pad = 0;
    if (phi_1 < 0.0 || phi_1 > 1.0) pad = 0;
    return pad;
}

/* ===================================================================== */
/* Euler (single phase, ideal gas GAMMA_1), euler.c                       */
/* ===================================================================== */

/* euler.c:14-23 */
static void eul_cons2prim(const eos_t *e, const double *Q, double *V)
{
    double irho = 1.0 / Q[0];
    V[0] = Q[0];
    V[1] = irho * Q[1];
    V[2] = irho * Q[2];
    V[3] = (e->g1 - 1.0) * (Q[3] - 0.5 * irho * (Q[1] * Q[1] + Q[2] * Q[2]));
}

/* euler.c:29-38 */
static void eul_prim2cons(const eos_t *e, const double *V, double *Q)
{
    double ei = (V[3]) / (e->g1 - 1.0);
    double k = 0.5 * V[0] * (V[1] * V[1] + V[2] * V[2]);
    Q[0] = V[0];
    Q[1] = V[0] * V[1];
    Q[2] = V[0] * V[2];
    Q[3] = k + ei;
}

/* euler.c:197-236 */
static double eul_flux_prim(const eos_t *e, const double *V, double nx, double ny, double *F, int *bad)
{
    double rho = V[0], u = V[1], v = V[2];
    double un = nx * u + ny * v;
    double rhoun = rho * un;
    double p = V[3];
    double E = p / (e->g1 - 1.0) + 0.5 * rho * (u * u + v * v);
    if (rho < RHO_FLOOR) *bad = 1;
    if (p < PRS_FLOOR) *bad = 1;
    F[0] = rhoun;
    F[1] = rhoun * u + nx * p;
    F[2] = rhoun * v + ny * p;
    F[3] = un * (E + p);
    return fabs(un) + sqrt(e->g1 * p / rho);
}

/* euler.c:292-310 */
static int eul_pad_prim(const eos_t *e, const double *V)
{
    (void)e;
    int pad = 1;
    if (V[0] < RHO_FLOOR) pad = 0;
    if (V[3] < PRS_FLOOR) pad = 0;
    return pad;
}

/* euler.c:44-84 */
static double eul_flux_cons(const eos_t *e, const double *Q, double nx, double ny, double *F, int *bad)
{
    double rho = Q[0];
    double irho = 1.0 / rho;
    double u = irho * Q[1], v = irho * Q[2];
    double un = nx * u + ny * v;
    double rhoun = rho * un;
    double E = Q[3];
    double p = (e->g1 - 1.0) * (E - 0.5 * rho * (u * u + v * v));
    if (rho < RHO_FLOOR) *bad = 1;
    if (p < PRS_FLOOR) *bad = 1;
    F[0] = rhoun;
    F[1] = rhoun * u + nx * p;
    F[2] = rhoun * v + ny * p;
    F[3] = un * (E + p);
    return fabs(un) + sqrt(e->g1 * p * irho);
}

/* euler.c:169-191 */
static int eul_pad_cons(const eos_t *e, const double *Q)
{
    int pad = 1;
    double rho = Q[0];
    double irho = 1.0 / rho;
    double u = irho * Q[1], v = irho * Q[2];
    double E = Q[3];
    double p = (e->g1 - 1.0) * (E - 0.5 * rho * (u * u + v * v));
    if (rho < RHO_FLOOR) pad = 0;
    if (p < PRS_FLOOR) pad = 0;
    return pad;
}

static void zero_ncp(const eos_t *e, const double *V, const double *gx, const double *gy, double *B)
{
    (void)e; (void)V; (void)gx; (void)gy;
    B[0] = 0.0; B[1] = 0.0; B[2] = 0.0; B[3] = 0.0;   /* euler.c:142-148, 278-286 */
}

/* ===================================================================== */
/* system table                                                           */
/* ===================================================================== */

typedef struct {
    int nv;
    void (*c2p)(const eos_t *, const double *, double *);
    void (*p2c)(const eos_t *, const double *, double *);
    double (*flux)(const eos_t *, const double *, double, double, double *, int *);
    void (*ncp)(const eos_t *, const double *, const double *, const double *, double *);
    int (*pad)(const eos_t *, const double *);
    int refl_x[2], refl_y[2];  /* velocity/momentum components negated by a reflective wall (-1: none) */
    int refl_xv, refl_yv;      /* and the tangential ones the VISCOUS build negates too (-1: none) */
    double (*visc)(const double *, const double g[][2], double, double, double, double, double *);
} sys_t;

static int get_sys(const hyo_config *c, sys_t *s)
{
    int cons = c->conservative;
    memset(s, 0, sizeof(*s));
    switch (c->system) {
    case HYO_EULER:
        s->nv = 4; s->c2p = eul_cons2prim; s->p2c = eul_prim2cons;
        s->flux = cons ? eul_flux_cons : eul_flux_prim; s->ncp = zero_ncp; s->pad = cons ? eul_pad_cons : eul_pad_prim;
        s->refl_x[0] = 1; s->refl_x[1] = -1; s->refl_y[0] = 2; s->refl_y[1] = -1;   /* rhs_function_prim.c:101-102,230-231 */
        s->refl_xv = -1; s->refl_yv = -1;   /* no viscous restatement: euler.c:269 writes past nVar */
        return 0;
    case HYO_KAPILA:
        s->nv = 6; s->c2p = kap_cons2prim; s->p2c = kap_prim2cons;
        s->flux = cons ? kap_flux_cons : kap_flux_prim; s->ncp = cons ? kap_ncp_cons : kap_ncp_prim;
        s->pad = cons ? kap_pad_cons : kap_pad_prim;
        s->refl_x[0] = 2; s->refl_x[1] = -1; s->refl_y[0] = 3; s->refl_y[1] = -1;   /* :124-125, :253-254 */
        s->refl_xv = 3; s->refl_yv = 2;                                             /* :126-127, :255-256 (VISCOUS) */
        s->visc = cons ? kap_visc_cons : kap_visc_prim;
        return 0;
    case HYO_BN:
        s->nv = 9; s->c2p = bn_cons2prim; s->p2c = bn_prim2cons;
        s->flux = cons ? bn_flux_cons : bn_flux_prim; s->ncp = cons ? bn_ncp_cons : bn_ncp_prim;
        s->pad = cons ? bn_pad_cons : bn_pad_prim;
        s->refl_x[0] = 1; s->refl_x[1] = 5; s->refl_y[0] = 2; s->refl_y[1] = 6;    /* :115-117, :244-246 */
        s->refl_xv = -1; s->refl_yv = -1;   /* baer_nunziato.c has no viscous flux */
        return 0;
    default:
        return -1;
    }
}

/* ===================================================================== */
/* reconstruction, reconstruction.c                                       */
/* ===================================================================== */

/* reconstruction.c:11-47 */
static double basis_val(double x, double y, int n)
{
    switch (n) {
    case 0: return 1.0;
    case 1: return x;
    case 2: return y;
    case 3: return x * x - 1. / 12.;
    case 4: return y * y - 1. / 12.;
    case 5: return x * y;
    case 6: return x * (x * x - 3. / 20.);
    case 7: return y * (y * y - 3. / 20.);
    case 8: return y * (x * x - 1. / 12.);
    case 9: return x * (y * y - 1. / 12.);
    default: return 0.0;
    }
}

/* reconstruction.c:53-100 */
static void basis_grad_val(double x, double y, int n, double *gx, double *gy)
{
    switch (n) {
    case 0: *gx = 0.0; *gy = 0.0; break;
    case 1: *gx = 1.0; *gy = 0.0; break;
    case 2: *gx = 0.0; *gy = 1.0; break;
    case 3: *gx = 2.0 * x; *gy = 0.0; break;
    case 4: *gx = 0.0; *gy = 2.0 * y; break;
    case 5: *gx = y; *gy = x; break;
    case 6: *gx = 3.0 * x * x - 3. / 20.; *gy = 0.0; break;
    case 7: *gx = 0.0; *gy = 3.0 * y * y - 3. / 20.; break;
    case 8: *gx = 2.0 * x * y; *gy = (x * x - 1. / 12.); break;
    case 9: *gx = (y * y - 1. / 12.); *gy = 2.0 * x * y; break;
    default: *gx = 0.0; *gy = 0.0;
    }
}

/* reconstruction.c:106-117 */
static double minmod(double a, double b)
{
    if (a * b < 0.0) return 0.0;
    return (fabs(a) < fabs(b)) ? a : b;
}

/* reconstruction.c:123-127 */
static double pow4(double a) { double a2 = a * a; return a2 * a2; }

/* Stencil of one variable around a cell: the 5-point cross and 4 diagonals
 * (rhs_function_prim.c:332-348). */
typedef struct {
    double c;                        /* u_0        */
    double xm2, xm1, xp1, xp2;       /* u_{i-2..i+2} */
    double ym2, ym1, yp1, yp2;       /* u_{j-2..j+2} */
    double pp, pm, mp, mm;           /* u_{i+1,j+1}, u_{i+1,j-1}, u_{i-1,j+1}, u_{i-1,j-1} */
} stencil_t;

/* reconstruction.c:129-142 (N = 1: minmod slopes) */
static void rec_deg1(const stencil_t *s, double *c)
{
    c[0] = s->c;
    c[1] = minmod(s->xp1 - s->c, s->c - s->xm1);
    c[2] = minmod(s->yp1 - s->c, s->c - s->ym1);
}

/* one direction of reconstruction.c:157-178 (x) / 182-199 (y): returns slope and curvature */
static void weno3_1d(double u_m2, double u_m1, double u_0, double u_p1, double u_p2, double *slope, double *curv)
{
    const double central_cell_wt = 100.0;
    double u_x[3], u_xx[3], wt[3], IS[3], total;
    u_x[0] = -2.0 * u_m1 + 0.5 * u_m2 + 1.5 * u_0; u_xx[0] = 0.5 * (u_m2 - 2.0 * u_m1 + u_0);
    u_x[1] = 0.5 * (u_p1 - u_m1);                  u_xx[1] = 0.5 * (u_m1 - 2.0 * u_0 + u_p1);
    u_x[2] = -1.5 * u_0 + 2.0 * u_p1 - 0.5 * u_p2; u_xx[2] = 0.5 * (u_0 - 2.0 * u_p1 + u_p2);
    IS[0] = u_x[0] * u_x[0] + R13_3 * u_xx[0] * u_xx[0]; wt[0] = 1.0 / (pow4(IS[0] + SMALL_NUM));
    IS[1] = u_x[1] * u_x[1] + R13_3 * u_xx[1] * u_xx[1]; wt[1] = central_cell_wt / (pow4(IS[1] + SMALL_NUM));
    IS[2] = u_x[2] * u_x[2] + R13_3 * u_xx[2] * u_xx[2]; wt[2] = 1.0 / (pow4(IS[2] + SMALL_NUM));
    total = wt[0] + wt[1] + wt[2];
    wt[0] = wt[0] / total;
    wt[1] = wt[1] / total;
    wt[2] = wt[2] / total;
    *slope = wt[0] * u_x[0] + wt[1] * u_x[1] + wt[2] * u_x[2];
    *curv = wt[0] * u_xx[0] + wt[1] * u_xx[1] + wt[2] * u_xx[2];
}

/* reconstruction.c:144-221 (N = 2) */
static void rec_deg2(const stencil_t *s, double *c)
{
    double u_0 = s->c, u_xy[4], wt[4], IS[4], total, temp;
    c[0] = u_0;
    weno3_1d(s->xm2, s->xm1, u_0, s->xp1, s->xp2, &c[1], &c[3]);
    weno3_1d(s->ym2, s->ym1, u_0, s->yp1, s->yp2, &c[2], &c[4]);
    u_xy[0] =  s->pp - u_0 - c[1] - c[2] - c[3] - c[4];
    u_xy[1] = -s->pm + u_0 + c[1] - c[2] + c[3] + c[4];
    u_xy[2] = -s->mp + u_0 - c[1] + c[2] + c[3] + c[4];
    u_xy[3] =  s->mm - u_0 + c[1] + c[2] - c[3] - c[4];
    temp = 4.0 * (c[3] * c[3] + c[4] * c[4]);
    IS[0] = temp + u_xy[0] * u_xy[0]; wt[0] = 1.0 / (pow4(IS[0] + SMALL_NUM));
    IS[1] = temp + u_xy[1] * u_xy[1]; wt[1] = 1.0 / (pow4(IS[1] + SMALL_NUM));
    IS[2] = temp + u_xy[2] * u_xy[2]; wt[2] = 1.0 / (pow4(IS[2] + SMALL_NUM));
    IS[3] = temp + u_xy[3] * u_xy[3]; wt[3] = 1.0 / (pow4(IS[3] + SMALL_NUM));
    total = wt[0] + wt[1] + wt[2] + wt[3];
    wt[0] = wt[0] / total; wt[1] = wt[1] / total; wt[2] = wt[2] / total; wt[3] = wt[3] / total;
    c[5] = wt[0] * u_xy[0] + wt[1] * u_xy[1] + wt[2] * u_xy[2] + wt[3] * u_xy[3];
}

/* reconstruction.c:223-357 (N = 3) */
static void rec_deg3(const stencil_t *s, double *coeffs)
{
    double gammaHi = 0.85, gammaLo = 0.85;
    double u_0 = s->c;
    double u_ip1 = s->xp1, u_jp1 = s->yp1, u_ip1jp1 = s->pp;
    double u_im1 = s->xm1, u_jm1 = s->ym1, u_ip1jm1 = s->pm;
    double u_ip2 = s->xp2, u_jp2 = s->yp2, u_im1jp1 = s->mp;
    double u_im2 = s->xm2, u_jm2 = s->ym2, u_im1jm1 = s->mm;
    double u_xR4, u_yR4, u_xxR4, u_yyR4, u_xyR4, u_xxxR4, u_yyyR4, u_xxyR4, u_xyyR4;
    double u_xR3[5], u_yR3[5], u_xxR3[5], u_yyR3[5], u_xyR3[5];
    double IS_R4, gamma_R4, w_R4, IS_R3[5], gamma_R3[5], w_R3[5], sum = 0.0, wt_ratio;
    int i;

    gamma_R4 = gammaHi;
    gamma_R3[0] = (1.0 - gammaHi) * gammaLo;
    for (i = 1; i < 5; ++i) gamma_R3[i] = 0.25 * (1 - gammaHi) * (1 - gammaLo);

    u_xR4   = R41_60 * (-u_im1 + u_ip1) + R11_120 * (u_im2 - u_ip2);
    u_yR4   = R41_60 * (-u_jm1 + u_jp1) + R11_120 * (u_jm2 - u_jp2);
    u_xxR4  = -u_0 + 0.5 * (u_im1 + u_ip1);
    u_yyR4  = -u_0 + 0.5 * (u_jm1 + u_jp1);
    u_xyR4  = 0.25 * (u_im1jm1 - u_im1jp1 - u_ip1jm1 + u_ip1jp1);
    u_xxxR4 = R1_6 * (u_im1 - u_ip1) + R1_12 * (u_ip2 - u_im2);
    u_yyyR4 = R1_6 * (u_jm1 - u_jp1) + R1_12 * (u_jp2 - u_jm2);
    u_xxyR4 = 0.25 * (-u_im1jm1 + u_im1jp1 - u_ip1jm1 + u_ip1jp1) + 0.5 * (u_jm1 - u_jp1);
    u_xyyR4 = 0.5 * (u_im1 - u_ip1) + 0.25 * (u_ip1jp1 - u_im1jm1 - u_im1jp1 + u_ip1jm1);

    IS_R4 = (u_xR4 + 0.1 * u_xxxR4) * (u_xR4 + 0.1 * u_xxxR4) + R13_3 * (u_xxR4 * u_xxR4 + u_yyR4 * u_yyR4) +
            (u_yR4 + 0.1 * u_yyyR4) * (u_yR4 + 0.1 * u_yyyR4) + 39.05 * (u_xxxR4 * u_xxxR4 + u_yyyR4 * u_yyyR4) +
            R7_6 * u_xyR4 * u_xyR4 + 4.7 * (u_xxyR4 * u_xxyR4 + u_xyyR4 * u_xyyR4);
    w_R4 = gamma_R4 / (pow4(IS_R4 + SMALL_NUM));
    sum = w_R4;

    u_xR3[0] = 0.5 * (-u_im1 + u_ip1);
    u_yR3[0] = 0.5 * (-u_jm1 + u_jp1);
    u_xxR3[0] = -u_0 + 0.5 * (u_im1 + u_ip1);
    u_yyR3[0] = -u_0 + 0.5 * (u_jm1 + u_jp1);
    u_xyR3[0] = 0.25 * (u_im1jm1 - u_im1jp1 - u_ip1jm1 + u_ip1jp1);

    u_xR3[1] = 1.5 * u_0 - 2.0 * u_im1 + 0.5 * u_im2;
    u_yR3[1] = 0.5 * (-u_jm1 + u_jp1);
    u_xxR3[1] = 0.5 * u_0 - u_im1 + 0.5 * u_im2;
    u_yyR3[1] = -u_0 + 0.5 * u_jm1 + 0.5 * u_jp1;
    u_xyR3[1] = 0.5 * (u_im1jm1 - u_im1jp1 - u_jm1 + u_jp1);

    u_xR3[2] = -1.5 * u_0 + 2.0 * u_ip1 - 0.5 * u_ip2;
    u_yR3[2] = 0.5 * (-u_jm1 + u_jp1);
    u_xxR3[2] = 0.5 * u_0 - u_ip1 + 0.5 * u_ip2;
    u_yyR3[2] = -u_0 + 0.5 * u_jm1 + 0.5 * u_jp1;
    u_xyR3[2] = 0.5 * (-u_ip1jm1 + u_ip1jp1 + u_jm1 - u_jp1);

    u_xR3[3] = 0.5 * (-u_im1 + u_ip1);
    u_yR3[3] = 1.5 * u_0 - 2.0 * u_jm1 + 0.5 * u_jm2;
    u_xxR3[3] = -u_0 + 0.5 * u_im1 + 0.5 * u_ip1;
    u_yyR3[3] = 0.5 * u_0 - u_jm1 + 0.5 * u_jm2;
    u_xyR3[3] = 0.5 * (-u_im1 + u_im1jm1 + u_ip1 - u_ip1jm1);

    u_xR3[4] = 0.5 * (-u_im1 + u_ip1);
    u_yR3[4] = -1.5 * u_0 + 2.0 * u_jp1 - 0.5 * u_jp2;
    u_xxR3[4] = -u_0 + 0.5 * u_im1 + 0.5 * u_ip1;
    u_yyR3[4] = 0.5 * u_0 - u_jp1 + 0.5 * u_jp2;
    u_xyR3[4] = 0.5 * (u_im1 - u_im1jp1 - u_ip1 + u_ip1jp1);

    for (i = 0; i < 5; ++i) {
        IS_R3[i] = u_xR3[i] * u_xR3[i] + u_yR3[i] * u_yR3[i] + R13_3 * (u_xxR3[i] * u_xxR3[i] + u_yyR3[i] * u_yyR3[i]) + R7_6 * u_xyR3[i] * u_xyR3[i];
        w_R3[i] = gamma_R3[i] / (pow4(IS_R3[i] + SMALL_NUM));
        sum += w_R3[i];
    }
    w_R4 = w_R4 / sum;
    for (i = 0; i < 5; ++i) w_R3[i] = w_R3[i] / sum;
    wt_ratio = w_R4 / gamma_R4;

    coeffs[0] = u_0;
    coeffs[1] = wt_ratio * (u_xR4 - gamma_R3[0] * u_xR3[0] - gamma_R3[1] * u_xR3[1] - gamma_R3[2] * u_xR3[2] - gamma_R3[3] * u_xR3[3] - gamma_R3[4] * u_xR3[4])
              + w_R3[0] * u_xR3[0] + w_R3[1] * u_xR3[1] + w_R3[2] * u_xR3[2] + w_R3[3] * u_xR3[3] + w_R3[4] * u_xR3[4];
    coeffs[2] = wt_ratio * (u_yR4 - gamma_R3[0] * u_yR3[0] - gamma_R3[1] * u_yR3[1] - gamma_R3[2] * u_yR3[2] - gamma_R3[3] * u_yR3[3] - gamma_R3[4] * u_yR3[4])
              + w_R3[0] * u_yR3[0] + w_R3[1] * u_yR3[1] + w_R3[2] * u_yR3[2] + w_R3[3] * u_yR3[3] + w_R3[4] * u_yR3[4];
    coeffs[3] = wt_ratio * (u_xxR4 - gamma_R3[0] * u_xxR3[0] - gamma_R3[1] * u_xxR3[1] - gamma_R3[2] * u_xxR3[2] - gamma_R3[3] * u_xxR3[3] - gamma_R3[4] * u_xxR3[4])
              + w_R3[0] * u_xxR3[0] + w_R3[1] * u_xxR3[1] + w_R3[2] * u_xxR3[2] + w_R3[3] * u_xxR3[3] + w_R3[4] * u_xxR3[4];
    coeffs[4] = wt_ratio * (u_yyR4 - gamma_R3[0] * u_yyR3[0] - gamma_R3[1] * u_yyR3[1] - gamma_R3[2] * u_yyR3[2] - gamma_R3[3] * u_yyR3[3] - gamma_R3[4] * u_yyR3[4])
              + w_R3[0] * u_yyR3[0] + w_R3[1] * u_yyR3[1] + w_R3[2] * u_yyR3[2] + w_R3[3] * u_yyR3[3] + w_R3[4] * u_yyR3[4];
    coeffs[5] = wt_ratio * (u_xyR4 - gamma_R3[0] * u_xyR3[0] - gamma_R3[1] * u_xyR3[1] - gamma_R3[2] * u_xyR3[2] - gamma_R3[3] * u_xyR3[3] - gamma_R3[4] * u_xyR3[4])
              + w_R3[0] * u_xyR3[0] + w_R3[1] * u_xyR3[1] + w_R3[2] * u_xyR3[2] + w_R3[3] * u_xyR3[3] + w_R3[4] * u_xyR3[4];
    coeffs[6] = wt_ratio * u_xxxR4;
    coeffs[7] = wt_ratio * u_yyyR4;
    coeffs[8] = wt_ratio * u_xxyR4;
    coeffs[9] = wt_ratio * u_xyyR4;
}

/* The unlimited central coefficients u_coeffs that Reconstruct also returns
 * (reconstruction.c:139-141, 172-174, 195-196, 217, 258-267); the VISCOUS
 * build takes the face gradients from them.  N = 0 leaves them unset in the
 * reference, so the viscous path starts at N = 1. */
static void ucoef(int N, const stencil_t *s, double *uc)
{
    const double u_0 = s->c;
    uc[0] = u_0;
    if (N == 1) {
        uc[1] = 0.5 * (s->xp1 - s->xm1);
        uc[2] = 0.5 * (s->yp1 - s->ym1);
    } else if (N == 2) {
        uc[1] = 0.5 * (s->xp1 - s->xm1);
        uc[3] = 0.5 * (s->xm1 - 2.0 * u_0 + s->xp1);
        uc[2] = 0.5 * (s->yp1 - s->ym1);
        uc[4] = 0.5 * (s->ym1 - 2.0 * u_0 + s->yp1);
        uc[5] = 0.25 * (s->pp - s->pm - s->mp + s->mm);
    } else if (N == 3) {
        const double u_ip1 = s->xp1, u_jp1 = s->yp1, u_ip1jp1 = s->pp, u_im1 = s->xm1, u_jm1 = s->ym1, u_ip1jm1 = s->pm;
        const double u_ip2 = s->xp2, u_jp2 = s->yp2, u_im1jp1 = s->mp, u_im2 = s->xm2, u_jm2 = s->ym2, u_im1jm1 = s->mm;
        uc[1] = R41_60 * (-u_im1 + u_ip1) + R11_120 * (u_im2 - u_ip2);
        uc[2] = R41_60 * (-u_jm1 + u_jp1) + R11_120 * (u_jm2 - u_jp2);
        uc[3] = -u_0 + 0.5 * (u_im1 + u_ip1);
        uc[4] = -u_0 + 0.5 * (u_jm1 + u_jp1);
        uc[5] = 0.25 * (u_im1jm1 - u_im1jp1 - u_ip1jm1 + u_ip1jp1);
        uc[6] = R1_6 * (u_im1 - u_ip1) + R1_12 * (u_ip2 - u_im2);
        uc[7] = R1_6 * (u_jm1 - u_jp1) + R1_12 * (u_jp2 - u_jm2);
        uc[8] = 0.25 * (-u_im1jm1 + u_im1jp1 - u_ip1jm1 + u_ip1jp1) + 0.5 * (u_jm1 - u_jp1);
        uc[9] = 0.5 * (u_im1 - u_ip1) + 0.25 * (u_ip1jp1 - u_im1jm1 - u_im1jp1 + u_ip1jm1);
    }
}

/* ===================================================================== */
/* quadrature tables (hype.c:194-305)                                      */
/* ===================================================================== */

typedef struct {
    int ndof, nfgp, nvgp, nnode;
    double wf[2], wv[4];
    double phi_face[4][2][MAXDOF];          /* [face L,R,B,T][gp][k] */
    double phi_node[8][MAXDOF];
    double phi_vol[4][MAXDOF], dphi_vol_x[4][MAXDOF], dphi_vol_y[4][MAXDOF];
    double dphi_face[4][2][2][MAXDOF];      /* [face][gp][dim][k]: gradphiFace_x / _y (hype.c:255-285) */
} tables_t;

static void make_tables(int N, tables_t *T)
{
    const double g = 0.28867513459481287;
    double xf[2], xv[4], yv[4], xn[8], yn[8];
    memset(T, 0, sizeof(*T));
    T->ndof = (N + 1) * (N + 2) / 2;
    if (N < 2) {
        T->nfgp = 1; T->nvgp = 1;
        xf[0] = 0.0; T->wf[0] = 1.0;
        xv[0] = 0.0; yv[0] = 0.0; T->wv[0] = 1.0;
        xn[0] = 0.5; yn[0] = 0.0; xn[1] = -0.5; yn[1] = 0.0; xn[2] = 0.0; yn[2] = 0.5; xn[3] = 0.0; yn[3] = -0.5;
    } else {
        T->nfgp = 2; T->nvgp = 4;
        xf[0] = -g; xf[1] = g; T->wf[0] = 0.5; T->wf[1] = 0.5;
        xv[0] = -g; yv[0] = -g; xv[1] = -g; yv[1] = g; xv[2] = g; yv[2] = -g; xv[3] = g; yv[3] = g;
        for (int q = 0; q < 4; ++q) T->wv[q] = 0.25;
        xn[0] = 0.5; yn[0] = -g; xn[1] = 0.5; yn[1] = g; xn[2] = -0.5; yn[2] = -g; xn[3] = -0.5; yn[3] = g;
        xn[4] = -g; yn[4] = 0.5; xn[5] = g; yn[5] = 0.5; xn[6] = -g; yn[6] = -0.5; xn[7] = g; yn[7] = -0.5;
    }
    T->nnode = 4 * T->nfgp;
    for (int q = 0; q < T->nfgp; ++q)
        for (int k = 0; k < T->ndof; ++k) {
            T->phi_face[0][q][k] = basis_val(-0.5, xf[q], k);
            T->phi_face[1][q][k] = basis_val(0.5, xf[q], k);
            T->phi_face[2][q][k] = basis_val(xf[q], -0.5, k);
            T->phi_face[3][q][k] = basis_val(xf[q], 0.5, k);
            basis_grad_val(-0.5, xf[q], k, &T->dphi_face[0][q][0][k], &T->dphi_face[0][q][1][k]);
            basis_grad_val(0.5, xf[q], k, &T->dphi_face[1][q][0][k], &T->dphi_face[1][q][1][k]);
            basis_grad_val(xf[q], -0.5, k, &T->dphi_face[2][q][0][k], &T->dphi_face[2][q][1][k]);
            basis_grad_val(xf[q], 0.5, k, &T->dphi_face[3][q][0][k], &T->dphi_face[3][q][1][k]);
        }
    for (int q = 0; q < T->nnode; ++q)
        for (int k = 0; k < T->ndof; ++k) T->phi_node[q][k] = basis_val(xn[q], yn[q], k);
    for (int q = 0; q < T->nvgp; ++q)
        for (int k = 0; k < T->ndof; ++k) {
            T->phi_vol[q][k] = basis_val(xv[q], yv[q], k);
            basis_grad_val(xv[q], yv[q], k, &T->dphi_vol_x[q][k], &T->dphi_vol_y[q][k]);
        }
}

/* ===================================================================== */
/* the right-hand side                                                    */
/* ===================================================================== */

/* value of a cell's polynomial (coefficients cf[k*nv+c]) at a face quadrature
 * point, accumulated as u_bnd is in rhs_function_prim.c:429-440 */
static void face_value(const tables_t *T, const double *cf, int f, int q, int nv, double *out)
{
    for (int c = 0; c < nv; ++c) {
        double v = 0.0;
        for (int k = 0; k < T->ndof; ++k) v += cf[k * nv + c] * T->phi_face[f][q][k];
        out[c] = v;
    }
}

static inline int wrapi(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }

int hyo_rhs(const hyo_config *cfg, double t, const double *U, double *RHS, double *dt_out)
{
    sys_t S;
    (void)t;
    if (get_sys(cfg, &S)) return HYO_ERR_CONFIG;
    if (cfg->order < 0 || cfg->order > 3 || cfg->nx < 1 || cfg->ny < 1) return HYO_ERR_CONFIG;
    const int visc = cfg->viscous != 0;
    if (visc && (!S.visc || cfg->order < 1)) return HYO_ERR_CONFIG;
    int bcs[4] = {cfg->bc_left, cfg->bc_right, cfg->bc_bottom, cfg->bc_top};
    for (int k = 0; k < 4; ++k) {
        if (bcs[k] == HYO_BC_WALL || bcs[k] < 0 || bcs[k] > 4) return HYO_ERR_CONFIG;   /* wall: ghosts never set by the reference */
        if (bcs[k] == HYO_BC_INLET && (k != 0 || cfg->system != HYO_KAPILA)) return HYO_ERR_CONFIG;
    }
    const eos_t eos = {cfg->gamma1, cfg->gamma2, cfg->pi1, cfg->pi2, cfg->bn_fixed_p2};
    const int nv = S.nv, nx = cfg->nx, ny = cfg->ny, N = cfg->order;
    const int px = (cfg->bc_left == HYO_BC_PERIODIC || cfg->bc_right == HYO_BC_PERIODIC);
    const int py = (cfg->bc_bottom == HYO_BC_PERIODIC || cfg->bc_top == HYO_BC_PERIODIC);
    const double h = (cfg->x_max - cfg->x_min) / (double)nx;   /* hype.c:57 */
    const double r1_h = 1. / h;
    tables_t T;
    make_tables(N, &T);
    const int ndof = T.ndof;
    tl_pad_fallbacks = 0;

    /* ---- padded state W[(j+GH)*(nx+2GH) + (i+GH)][c]: primitive (prim path)
     *      or conserved (conservative path) variables, ghosts filled ---- */
    const int gw = nx + 2 * GH, gh = ny + 2 * GH;
    double *W = (double *)calloc((size_t)gw * gh * nv, sizeof(double));
#define WAT(j, i) (W + ((size_t)((j) + GH) * gw + (size_t)((i) + GH)) * nv)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double *Q = U + ((size_t)j * nx + i) * nv;
            if (cfg->conservative) memcpy(WAT(j, i), Q, sizeof(double) * nv);
            else S.c2p(&eos, Q, WAT(j, i));          /* post_process.c:165-200 */
        }
    /* periodic wrap of the halo (DMGlobalToLocal on a periodic DMDA) */
    for (int j = -GH; j < ny + GH; ++j) {
        int jin = (j >= 0 && j < ny);
        if (!jin && !py) continue;
        for (int i = -GH; i < nx + GH; ++i) {
            int iin = (i >= 0 && i < nx);
            if (jin && iin) continue;
            if (!iin && !px) continue;
            memcpy(WAT(j, i), WAT(jin ? j : wrapi(j, ny), iin ? i : wrapi(i, nx)), sizeof(double) * nv);
        }
    }
    /* x pass then y pass, as rhs_function_prim.c:75-202 and 204-315 */
    for (int j = -GH; j < ny + GH; ++j)
        for (int i = -GH; i < nx + GH; ++i) {
            if (i >= 0 && i < nx) continue;
            int left = (i < 0), bc = left ? cfg->bc_left : cfg->bc_right;
            double *dst = WAT(j, i);
            if (bc == HYO_BC_TRANSMISSIVE) {
                memcpy(dst, WAT(j, left ? 0 : nx - 1), sizeof(double) * nv);
            } else if (bc == HYO_BC_REFLECTIVE) {
                memcpy(dst, WAT(j, left ? -1 - i : 2 * (nx - 1) - i + 1), sizeof(double) * nv);
                for (int r = 0; r < 2; ++r) if (S.refl_x[r] >= 0) dst[S.refl_x[r]] = -dst[S.refl_x[r]];
                if (visc) dst[S.refl_xv] = -dst[S.refl_xv];
            } else if (bc == HYO_BC_INLET) {
                double x_loc = cfg->x_min + ((double)i + 0.5) * h;
                double y_loc = cfg->y_min + ((double)j + 0.5) * h;
                double V[MAXV];
                kap_inlet_prim(&eos, x_loc, y_loc, V);
                if (cfg->conservative) kap_prim2cons(&eos, V, dst); else memcpy(dst, V, sizeof(double) * nv);
            }
        }
    for (int j = -GH; j < ny + GH; ++j) {
        if (j >= 0 && j < ny) continue;
        int bot = (j < 0), bc = bot ? cfg->bc_bottom : cfg->bc_top;
        for (int i = -GH; i < nx + GH; ++i) {
            double *dst = WAT(j, i);
            if (bc == HYO_BC_TRANSMISSIVE) {
                memcpy(dst, WAT(bot ? 0 : ny - 1, i), sizeof(double) * nv);
            } else if (bc == HYO_BC_REFLECTIVE) {
                memcpy(dst, WAT(bot ? -1 - j : 2 * (ny - 1) - j + 1, i), sizeof(double) * nv);
                for (int r = 0; r < 2; ++r) if (S.refl_y[r] >= 0) dst[S.refl_y[r]] = -dst[S.refl_y[r]];
                if (visc) dst[S.refl_yv] = -dst[S.refl_yv];
            }
        }
    }

    /* ---- reconstruction over the owned cells and the 1-cell ring
     *      (rhs_function_prim.c:321-456); corner cells of the ring feed no face ---- */
    const int cw = nx + 2, ch = ny + 2;
    double *C = (double *)calloc((size_t)cw * ch * ndof * nv, sizeof(double));
#define CAT(j, i) (C + ((size_t)((j) + 1) * cw + (size_t)((i) + 1)) * (size_t)ndof * nv)   /* [k][c] */
    /* VISCOUS: the unlimited coefficients of every reconstructed cell, [k][c] */
    double *UC = visc ? (double *)calloc((size_t)cw * ch * ndof * nv, sizeof(double)) : NULL;
#define UCAT(j, i) (UC + ((size_t)((j) + 1) * cw + (size_t)((i) + 1)) * (size_t)ndof * nv)
    for (int j = -1; j <= ny; ++j)
        for (int i = -1; i <= nx; ++i) {
            if ((j < 0 || j >= ny) && (i < 0 || i >= nx)) continue;
            double *cf = CAT(j, i);
            double coef[MAXDOF];
            for (int c = 0; c < nv; ++c) {
                stencil_t s;
                s.c = WAT(j, i)[c];
                s.xm2 = WAT(j, i - 2)[c]; s.xm1 = WAT(j, i - 1)[c]; s.xp1 = WAT(j, i + 1)[c]; s.xp2 = WAT(j, i + 2)[c];
                s.ym2 = WAT(j - 2, i)[c]; s.ym1 = WAT(j - 1, i)[c]; s.yp1 = WAT(j + 1, i)[c]; s.yp2 = WAT(j + 2, i)[c];
                s.pp = WAT(j + 1, i + 1)[c]; s.pm = WAT(j - 1, i + 1)[c]; s.mp = WAT(j + 1, i - 1)[c]; s.mm = WAT(j - 1, i - 1)[c];
                memset(coef, 0, sizeof(coef));
                if (N == 0) coef[0] = s.c;
                else if (N == 1) rec_deg1(&s, coef);
                else if (N == 2) rec_deg2(&s, coef);
                else rec_deg3(&s, coef);
                for (int k = 0; k < ndof; ++k) cf[k * nv + c] = coef[k];
                if (visc) {
                    double uc[MAXDOF];
                    ucoef(N, &s, uc);
                    for (int k = 0; k < ndof; ++k) UCAT(j, i)[k * nv + c] = uc[k];
                }
            }
            /* admissibility at the nodes (rhs_function_prim.c:382-404) */
            int pad = 1;
            for (int q = 0; q < T.nnode && pad; ++q) {
                double V[MAXV];
                for (int c = 0; c < nv; ++c) {
                    double val = 0.0;
                    for (int k = 0; k < ndof; ++k) val += cf[k * nv + c] * T.phi_node[q][k];
                    V[c] = val;
                }
                pad = S.pad(&eos, V);
            }
            if (!pad) {
                /* rhs_function_prim.c:407-421 (prim: zero from k = 3);
                 * rhs_function.c:410-420 (conservative: zero from k = 1) */
                tl_pad_fallbacks++;
                for (int c = 0; c < nv; ++c) {
                    double w0 = WAT(j, i)[c];
                    cf[0 * nv + c] = w0;
                    if (ndof > 1) cf[1 * nv + c] = minmod(WAT(j, i + 1)[c] - w0, w0 - WAT(j, i - 1)[c]);
                    if (ndof > 2) cf[2 * nv + c] = minmod(WAT(j + 1, i)[c] - w0, w0 - WAT(j - 1, i)[c]);
                    for (int k = cfg->conservative ? 1 : 3; k < ndof; ++k) cf[k * nv + c] = 0.0;
                }
            }
        }

    /* ---- face fluxes: x faces (rhs_function_prim.c:485-533), y faces (537-585) ---- */
    double *Fx = (double *)malloc(sizeof(double) * (size_t)(nx + 1) * ny * nv);
    double *Dx = (double *)malloc(sizeof(double) * (size_t)(nx + 1) * ny * nv);
    double *Gy = (double *)malloc(sizeof(double) * (size_t)nx * (ny + 1) * nv);
    double *Ey = (double *)malloc(sizeof(double) * (size_t)nx * (ny + 1) * nv);
    double s_max_c = 0.0, s_max_v = 0.0;
    int bad = 0;
    for (int dir = 0; dir < 2; ++dir) {
        const double nxv = dir == 0 ? 1.0 : 0.0, nyv = dir == 0 ? 0.0 : 1.0;
        const int nj = dir == 0 ? ny : ny + 1, ni = dir == 0 ? nx + 1 : nx;
        for (int j = 0; j < nj; ++j)
            for (int i = 0; i < ni; ++i) {
                const double *cl = dir == 0 ? CAT(j, i - 1) : CAT(j - 1, i);
                const double *cr = CAT(j, i);
                double Flux[MAXV], NCP[MAXV];
                for (int c = 0; c < nv; ++c) { Flux[c] = 0.0; NCP[c] = 0.0; }
                for (int q = 0; q < T.nfgp; ++q) {
                    double VL[MAXV], VR[MAXV], QL[MAXV], QR[MAXV], FL[MAXV], FR[MAXV];
                    double Vav[MAXV], gxv[MAXV], gyv[MAXV], Fc[MAXV], Dc[MAXV];
                    face_value(&T, cl, dir == 0 ? 1 : 3, q, nv, VL);
                    face_value(&T, cr, dir == 0 ? 0 : 2, q, nv, VR);
                    double s;
                    if (!cfg->conservative) {
                        /* riemann.c:112-140 */
                        S.p2c(&eos, VL, QL); S.p2c(&eos, VR, QR);
                        double sl = S.flux(&eos, VL, nxv, nyv, FL, &bad);
                        double sr = S.flux(&eos, VR, nxv, nyv, FR, &bad);
                        s = (sl < sr) ? sr : sl;
                        for (int c = 0; c < nv; ++c) {
                            Vav[c] = 0.5 * (VR[c] + VL[c]);
                            gxv[c] = nxv * (VR[c] - VL[c]);
                            gyv[c] = nyv * (VR[c] - VL[c]);
                            Fc[c] = 0.5 * (FR[c] + FL[c] - s * (QR[c] - QL[c]));
                        }
                    } else {
                        /* riemann.c:52-105 */
                        double sl = S.flux(&eos, VL, nxv, nyv, FL, &bad);
                        double sr = S.flux(&eos, VR, nxv, nyv, FR, &bad);
                        s = (sl < sr) ? sr : sl;
                        for (int c = 0; c < nv; ++c) {
                            Vav[c] = 0.5 * (VR[c] + VL[c]);
                            gxv[c] = nxv * (VR[c] - VL[c]);
                            gyv[c] = nyv * (VR[c] - VL[c]);
                            Fc[c] = 0.5 * (FR[c] + FL[c] - s * (VR[c] - VL[c]));
                        }
                    }
                    S.ncp(&eos, Vav, gxv, gyv, Dc);
                    if (s > s_max_c) s_max_c = s;
                    double Fv[MAXV];
                    if (visc) {
                        /* rhs_function_prim.c:356-374 (face gradients from u_coeffs) and
                         * riemann.c:146-186 (ViscRiemannSolver[Prim]: the mean of both sides) */
                        const double *ul = dir == 0 ? UCAT(j, i - 1) : UCAT(j - 1, i), *ur = UCAT(j, i);
                        const int fl = dir == 0 ? 1 : 3, fr = dir == 0 ? 0 : 2;
                        double gL[MAXV][2], gR[MAXV][2], FvL[MAXV], FvR[MAXV];
                        for (int c = 0; c < nv; ++c)
                            for (int d = 0; d < 2; ++d) {
                                double al = 0.0, ar = 0.0;
                                for (int k = 0; k < ndof; ++k) {
                                    al += ul[k * nv + c] * T.dphi_face[fl][q][d][k];
                                    ar += ur[k * nv + c] * T.dphi_face[fr][q][d][k];
                                }
                                gL[c][d] = r1_h * al;
                                gR[c][d] = r1_h * ar;
                            }
                        double svl = S.visc(VL, (const double(*)[2])gL, nxv, nyv, cfg->mu1, cfg->mu2, FvL);
                        double svr = S.visc(VR, (const double(*)[2])gR, nxv, nyv, cfg->mu1, cfg->mu2, FvR);
                        double sv = (svl < svr) ? svr : svl;
                        for (int c = 0; c < nv; ++c) Fv[c] = 0.5 * (FvR[c] + FvL[c]);
                        if (sv > s_max_v) s_max_v = sv;
                    }
                    for (int c = 0; c < nv; ++c) {
                        Flux[c] += T.wf[q] * Fc[c];
                        NCP[c] += T.wf[q] * Dc[c];
                        if (visc) Flux[c] += T.wf[q] * Fv[c];
                    }
                }
                double *fo = (dir == 0 ? Fx + ((size_t)j * (nx + 1) + i) * nv : Gy + ((size_t)j * nx + i) * nv);
                double *d_o = (dir == 0 ? Dx + ((size_t)j * (nx + 1) + i) * nv : Ey + ((size_t)j * nx + i) * nv);
                memcpy(fo, Flux, sizeof(double) * nv);
                memcpy(d_o, NCP, sizeof(double) * nv);
            }
    }

    /* ---- volume NCP (rhs_function_prim.c:459-479) and divergence (589-602) ---- */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double *cf = CAT(j, i);
            double *rhs = RHS + ((size_t)j * nx + i) * nv;
            for (int c = 0; c < nv; ++c) rhs[c] = 0.0;
            for (int q = 0; q < T.nvgp; ++q) {
                double V[MAXV], gxv[MAXV], gyv[MAXV], B[MAXV];
                for (int c = 0; c < nv; ++c) {
                    double value = 0.0, grad_x = 0.0, grad_y = 0.0;
                    for (int k = 0; k < ndof; ++k) {
                        value += cf[k * nv + c] * T.phi_vol[q][k];
                        grad_x += cf[k * nv + c] * T.dphi_vol_x[q][k];
                        grad_y += cf[k * nv + c] * T.dphi_vol_y[q][k];
                    }
                    V[c] = value; gxv[c] = r1_h * grad_x; gyv[c] = r1_h * grad_y;
                }
                S.ncp(&eos, V, gxv, gyv, B);
                for (int c = 0; c < nv; ++c) rhs[c] += -T.wv[q] * B[c];
            }
            const double *F0 = Fx + ((size_t)j * (nx + 1) + i) * nv, *F1 = F0 + nv;
            const double *D0 = Dx + ((size_t)j * (nx + 1) + i) * nv, *D1 = D0 + nv;
            const double *G0 = Gy + ((size_t)j * nx + i) * nv, *G1 = Gy + ((size_t)(j + 1) * nx + i) * nv;
            const double *E0 = Ey + ((size_t)j * nx + i) * nv, *E1 = Ey + ((size_t)(j + 1) * nx + i) * nv;
            for (int c = 0; c < nv; ++c)
                rhs[c] += -r1_h * (F1[c] - F0[c] + 0.5 * (D1[c] + D0[c])) - r1_h * (G1[c] - G0[c] + 0.5 * (E1[c] + E0[c]));
        }
#undef CAT
#undef WAT
#undef UCAT
    free(W); free(C); free(UC); free(Fx); free(Dx); free(Gy); free(Ey);
    if (dt_out) {
        if (visc) *dt_out = (cfg->cfl * h) / (2.0 * (s_max_c + (r1_h * s_max_v) * 2.0));   /* rhs_function_prim.c:617 */
        else *dt_out = (cfg->cfl * h) / (2.0 * s_max_c);                                 /* rhs_function_prim.c:620 */
    }
    return bad ? HYO_ERR_INADMISSIBLE : HYO_OK;
}

/* ===================================================================== */
/* SSP-RK time loop (hype.c:337-384 on PETSc TSSSP; see petsc_mini.c)      */
/* ===================================================================== */

static void axpy(size_t n, double *y, double a, const double *x)
{ for (size_t i = 0; i < n; ++i) { double t = a * x[i]; y[i] = y[i] + t; } }
static void axpbypcz(size_t n, double *z, double a, double b, double c, const double *x, const double *y)
{
    if (c == 0.0) { for (size_t i = 0; i < n; ++i) { double t0 = a * x[i], t1 = b * y[i]; z[i] = t0 + t1; } }
    else for (size_t i = 0; i < n; ++i) { double t0 = a * x[i], t1 = b * y[i], t2 = c * z[i]; double s = t0 + t1; z[i] = s + t2; }
}
static void axpby(size_t n, double *y, double a, double b, const double *x)
{ for (size_t i = 0; i < n; ++i) { double t0 = a * x[i], t1 = b * y[i]; y[i] = t0 + t1; } }

int hyo_solve(const hyo_config *cfg, double *U, double t0, double t_final, int max_steps,
              int *steps_out, double *t_out, double *dt_out)
{
    const int nv = hyo_nvar(cfg->system);
    if (!nv) return HYO_ERR_CONFIG;
    const size_t n = (size_t)cfg->nx * cfg->ny * nv;
    double *w0 = (double *)malloc(n * sizeof(double)), *w1 = (double *)malloc(n * sizeof(double)), *F = (double *)malloc(n * sizeof(double));
    double dt_ctx, t = t0;
    int steps = 0, rc;
#define RHS_AT(st, in) do { rc = hyo_rhs(cfg, (st), (in), F, &dt_ctx); if (rc) goto done; } while (0)
    double time_step;                           /* declared before the first RHS_AT: valid C++ too */
    RHS_AT(t0, U);                              /* hype.c:343 seeds Ctx.dt */
    for (;;) {
        time_step = dt_ctx;                     /* MonitorFunction, post_process.c:19 */
        if (steps >= max_steps || t >= t_final) break;
        double dt = time_step;
        if (t + dt > t_final) dt = t_final - t; /* TS_EXACTFINALTIME_MATCHSTEP */
        if (cfg->order == 0) {
            RHS_AT(t, U); axpy(n, U, dt, F);
        } else if (cfg->order == 1) {           /* TSSSPRKS2, 2 stages */
            const int s = 2;
            memcpy(w0, U, n * sizeof(double));
            for (int i = 0; i < s - 1; ++i) { RHS_AT(t + dt * (i / (s - 1.)), w0); axpy(n, w0, dt / (s - 1.), F); }
            RHS_AT(t + dt, w0);
            axpbypcz(n, U, (s - 1.) / s, dt / s, 1. / s, w0, F);
        } else if (cfg->order == 2) {           /* TSSSPRKS3, 4 stages (n = 2, r = 2) */
            const int s = 4, nn = 2, r = s - nn;
            int i = 0;
            memcpy(w0, U, n * sizeof(double));
            memcpy(w1, w0, n * sizeof(double));
            for (; i < nn * (nn + 1) / 2 - 1; ++i) {
                double c = (i < nn * (nn + 1) / 2) ? 1. * i / (s - nn) : (1. * i - nn) / (s - nn);
                RHS_AT(t + c * dt, w0); axpy(n, w0, dt / r, F);
            }
            {
                double c = (i < nn * (nn + 1) / 2) ? 1. * i / (s - nn) : (1. * i - nn) / (s - nn);
                RHS_AT(t + c * dt, w0);
                axpbypcz(n, w0, 1. * nn / (2 * nn - 1.), (nn - 1.) * dt / (r * (2 * nn - 1)), (nn - 1.) / (2 * nn - 1.), w1, F);
                ++i;
            }
            for (; i < s; ++i) {
                double c = (i < nn * (nn + 1) / 2) ? 1. * i / (s - nn) : (1. * i - nn) / (s - nn);
                RHS_AT(t + c * dt, w0); axpy(n, w0, dt / r, F);
            }
            memcpy(U, w0, n * sizeof(double));
        } else {                                /* TSSSPRK104 */
            static const double c[10] = {0, 1. / 6, 2. / 6, 3. / 6, 4. / 6, 2. / 6, 3. / 6, 4. / 6, 5. / 6, 1};
            int i;
            memcpy(w0, U, n * sizeof(double));
            for (i = 0; i < 5; ++i) { RHS_AT(t + c[i] * dt, w0); axpy(n, w0, dt / 6, F); }
            axpbypcz(n, w1, 1. / 25, 9. / 25, 0, U, w0);
            axpby(n, w0, 15, -5, w1);
            for (; i < 9; ++i) { RHS_AT(t + c[i] * dt, w0); axpy(n, w0, dt / 6, F); }
            RHS_AT(t + dt, w0);
            axpbypcz(n, w1, 3. / 5, dt / 10, 1, w0, F);
            memcpy(U, w1, n * sizeof(double));
        }
        t = t + dt;
        ++steps;
    }
    rc = HYO_OK;
done:
#undef RHS_AT
    free(w0); free(w1); free(F);
    if (steps_out) *steps_out = steps;
    if (t_out) *t_out = t;
    if (dt_out) *dt_out = dt_ctx;
    return rc;
}
