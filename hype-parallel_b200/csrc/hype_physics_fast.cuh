// hype_physics_fast.cuh -- the FP64 performance form of the physics
// (HYPE_PREC_FP64_FAST): the same PDE systems, reconstruction and admissibility
// checks as hype_physics.cuh, with the divisions that dominate the FP64 pipe
// replaced by reciprocals shared between several quotients, and compiled with
// FMA contraction.  Not bit-compatible with the reference by design; held to a
// relative L-infinity difference (max |diff| / max |reference|, per field) of
// at most 1e-12 per RHS evaluation against the reference's arithmetic.
//
// The rewrites, each algebraically exact:
//  * stiffened-gas sound speeds enter the Wood mixture speed and the Kapila
//    K-term only through rho_k a_k^2 = gamma_k (p + pi_k) =: A_k, so
//    a^2 = A1 A2 / (rho (alpha_2 A1 + alpha_1 A2)) and
//    K = alpha_1 alpha_2 (A2 - A1) / (alpha_1 A2 + alpha_2 A1) each take one
//    reciprocal (kapila_5eqn.c:347-349, 431, 458-460 take three or four divisions);
//  * divisions by (gamma - 1) and (gamma_1 - 1)(gamma_2 - 1) become products with
//    their inverses (Eos::derive);
//  * WENO weights w_k = (g_k / P_k) / sum_j (g_j / P_j), P_k = (IS_k + eps)^4
//    (reconstruction.c:163-170, 186-193, 207-215), are formed from products of
//    the P_j with a single reciprocal of their sum; where those products would
//    overflow, the weights fall back to one reciprocal per P_k;
//  * several quotients by one denominator share its reciprocal.
#pragma once
#include "hype_physics.cuh"

namespace hype {

// 1/x: the GPU's approximate FP64 reciprocal (rcp.approx.ftz.f64) refined by two
// Newton-Raphson steps y <- y + y (1 - x y) in fused multiply-adds (the classical
// iteration for the reciprocal, each step roughly doubling the number of correct
// bits).  Normal, finite, nonzero x only: no special handling of 0, infinities,
// NaN or subnormals.  tests/test_gpu_fast.py holds it to within 1 ulp of IEEE
// division over normal arguments of every exponent used here.
__device__ __forceinline__ double fast_rcp(double x)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

template <int SYS> struct FastSystem;

// kapila_5eqn.c, cons [a1 r1, a2 r2, rho u, rho v, E, a1], prim [r1, r2, u, v, p, a1]
template <> struct FastSystem<SYS_KAPILA> : System<SYS_KAPILA> {
    // kapila_5eqn.c:14-35
    __device__ __forceinline__ static void cons2prim(const Eos &e, const double *Q, double *V)
    {
        const double a1 = Q[5], a2 = 1.0 - a1;
        const double rho = Q[0] + Q[1];
        const double ir = fast_rcp(rho);
        const double u = Q[2] * ir, v = Q[3] * ir;
        const double ei = Q[4] - 0.5 * rho * (u * u + v * v);
        const double p = (ei * (e.g1m1 * e.g2m1) - a1 * e.c1 - a2 * e.c2) * fast_rcp(a1 * e.g2m1 + a2 * e.g1m1);
        V[0] = Q[0] * fast_rcp(a1);
        V[1] = Q[1] * fast_rcp(a2);
        V[2] = u;
        V[3] = v;
        V[4] = p;
        V[5] = a1;
    }
    // kapila_5eqn.c:41-61
    __device__ __forceinline__ static void prim2cons(const Eos &e, const double *V, double *Q)
    {
        const double a1 = V[5], a2 = 1.0 - a1;
        const double rho = a1 * V[0] + a2 * V[1];
        const double u = V[2], v = V[3], p = V[4];
        const double ei = (p * (a1 * e.g2m1 + a2 * e.g1m1) + a1 * e.c1 + a2 * e.c2) * e.inv_g12;
        Q[0] = a1 * V[0];
        Q[1] = a2 * V[1];
        Q[2] = rho * u;
        Q[3] = rho * v;
        Q[4] = ei + 0.5 * rho * (u * u + v * v);
        Q[5] = a1;
    }
    // kapila_5eqn.c:326-371
    template <int DIR>
    __device__ __forceinline__ static double flux(const Eos &e, const double *V, double *F, bool &bad)
    {
        const double a1 = V[5], a2 = 1.0 - a1;
        const double r1 = V[0], r2 = V[1];
        const double rho = a1 * r1 + a2 * r2;
        const double u = V[2], v = V[3], p = V[4];
        const double ei = (p * (a1 * e.g2m1 + a2 * e.g1m1) + a1 * e.c1 + a2 * e.c2) * e.inv_g12;
        const double E = ei + 0.5 * rho * (u * u + v * v);
        const double un = DIR == 0 ? u : v;
        const double A1 = e.g1 * (p + e.pi1), A2 = e.g2 * (p + e.pi2);
        const double a_sq = (A1 * A2) * fast_rcp(rho * (a2 * A1 + a1 * A2));
        bad |= (a_sq < PRS_FLOOR);
        F[0] = a1 * r1 * un;
        F[1] = a2 * r2 * un;
        F[2] = rho * u * un + (DIR == 0 ? p : 0.0);
        F[3] = rho * v * un + (DIR == 0 ? 0.0 : p);
        F[4] = (E + p) * un;
        F[5] = 0.0;
        return fabs(un) + sqrt(a_sq);
    }
    // kapila_5eqn.c:417-444
    __device__ __forceinline__ static void ncp(const Eos &e, const double *V, const double *gx, const double *gy, double *B)
    {
        const double a1 = V[5], a2 = 1.0 - a1;
        const double p = V[4];
        const double A1 = e.g1 * (p + e.pi1), A2 = e.g2 * (p + e.pi2);
        const double K = (a1 * a2 * (A2 - A1)) * fast_rcp(a1 * A2 + a2 * A1);
        B[0] = 0.0; B[1] = 0.0; B[2] = 0.0; B[3] = 0.0; B[4] = 0.0;
        B[5] = V[2] * gx[5] + V[3] * gy[5] - K * (gx[2] + gy[3]);
    }
    // kapila_5eqn.c:450-479
    __device__ __forceinline__ static bool pad(const Eos &e, const double *V)
    {
        const double a1 = V[5], a2 = 1.0 - a1;
        const double rho = a1 * V[0] + a2 * V[1];
        const double p = V[4];
        const double A1 = e.g1 * (p + e.pi1), A2 = e.g2 * (p + e.pi2);
        const double a_sq = (A1 * A2) * fast_rcp(rho * (a2 * A1 + a1 * A2));
        if (rho < RHO_FLOOR) return false;
        if (a_sq < PRS_FLOOR) return false;
        if (a1 < 0.0 || a1 > 1.0) return false;
        return true;
    }
};

// baer_nunziato.c, cons [a1 r1, a1 r1 u1, a1 r1 v1, a1 E1, a2 r2, a2 r2 u2, a2 r2 v2, a2 E2, a1]
template <> struct FastSystem<SYS_BN> : System<SYS_BN> {
    // baer_nunziato.c:14-41
    __device__ __forceinline__ static void cons2prim(const Eos &e, const double *Q, double *V)
    {
        const double phi_1 = Q[8], phi_2 = 1.0 - Q[8];
        const double i1 = fast_rcp(phi_1), i2 = fast_rcp(phi_2);
        const double q0 = fast_rcp(Q[0]), q4 = fast_rcp(Q[4]);
        const double rho_1 = Q[0] * i1, rho_2 = Q[4] * i2;
        const double u_1 = Q[1] * q0, v_1 = Q[2] * q0;
        const double u_2 = Q[5] * q4, v_2 = Q[6] * q4;
        const double E_1 = Q[3] * i1, E_2 = Q[7] * i2;
        V[0] = rho_1; V[1] = u_1; V[2] = v_1;
        V[3] = e.g1m1 * (E_1 - 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1)) - e.g1pi1;
        V[4] = rho_2; V[5] = u_2; V[6] = v_2;
        V[7] = e.g2m1 * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e.g2pi2;
        V[8] = phi_1;
    }
    // baer_nunziato.c:47-60
    __device__ __forceinline__ static void prim2cons(const Eos &e, const double *V, double *Q)
    {
        Q[0] = V[8] * V[0];
        Q[1] = Q[0] * V[1];
        Q[2] = Q[0] * V[2];
        Q[3] = Q[0] * (0.5 * (V[1] * V[1] + V[2] * V[2]) + (V[3] + e.g1pi1) * e.inv_g1m1 * fast_rcp(V[0]));
        Q[4] = (1.0 - V[8]) * V[4];
        Q[5] = Q[4] * V[5];
        Q[6] = Q[4] * V[6];
        Q[7] = Q[4] * (0.5 * (V[5] * V[5] + V[6] * V[6]) + (V[7] + e.g2pi2) * e.inv_g2m1 * fast_rcp(V[4]));
        Q[8] = V[8];
    }
    // baer_nunziato.c:256-321 (phase-2 flux pressure from V[8] unless fix_p2)
    template <int DIR>
    __device__ __forceinline__ static double flux(const Eos &e, const double *V, double *F, bool &bad)
    {
        const double phi_1 = V[8], phi_2 = 1.0 - V[8];
        const double rho_1 = V[0], rho_2 = V[4];
        const double u_1 = V[1], v_1 = V[2], u_2 = V[5], v_2 = V[6];
        const double p_1 = V[3];
        const double p_2 = e.fix_p2 ? V[7] : V[8];
        const double E_1 = (p_1 + e.g1pi1) * e.inv_g1m1 + 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1);
        const double E_2 = (p_2 + e.g2pi2) * e.inv_g2m1 + 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2);
        const double un_1 = DIR == 0 ? u_1 : v_1;
        const double un_2 = DIR == 0 ? u_2 : v_2;
        bad |= (rho_1 < RHO_FLOOR) | (rho_2 < RHO_FLOOR) | ((p_1 + e.pi1) < PRS_FLOOR) | ((p_2 + e.pi2) < PRS_FLOOR);
        F[0] = phi_1 * rho_1 * un_1;
        F[1] = phi_1 * (rho_1 * u_1 * un_1 + (DIR == 0 ? p_1 : 0.0));
        F[2] = phi_1 * (rho_1 * v_1 * un_1 + (DIR == 0 ? 0.0 : p_1));
        F[3] = phi_1 * un_1 * (E_1 + p_1);
        F[4] = phi_2 * rho_2 * un_2;
        F[5] = phi_2 * (rho_2 * u_2 * un_2 + (DIR == 0 ? p_2 : 0.0));
        F[6] = phi_2 * (rho_2 * v_2 * un_2 + (DIR == 0 ? 0.0 : p_2));
        F[7] = phi_2 * un_2 * (E_2 + p_2);
        F[8] = 0.0;
        const double s_1 = fabs(un_1) + sqrt(e.g1 * (p_1 + e.pi1) * fast_rcp(rho_1));
        const double s_2 = fabs(un_2) + sqrt(e.g2 * (p_2 + e.pi2) * fast_rcp(rho_2));
        return (s_1 < s_2) ? s_2 : s_1;
    }
};

// euler.c, cons [rho, rho u, rho v, E], prim [rho, u, v, p]
template <> struct FastSystem<SYS_EULER> : System<SYS_EULER> {
    // euler.c:14-23
    __device__ __forceinline__ static void cons2prim(const Eos &e, const double *Q, double *V)
    {
        const double irho = fast_rcp(Q[0]);
        V[0] = Q[0];
        V[1] = irho * Q[1];
        V[2] = irho * Q[2];
        V[3] = e.g1m1 * (Q[3] - 0.5 * irho * (Q[1] * Q[1] + Q[2] * Q[2]));
    }
    // euler.c:29-38
    __device__ __forceinline__ static void prim2cons(const Eos &e, const double *V, double *Q)
    {
        Q[0] = V[0];
        Q[1] = V[0] * V[1];
        Q[2] = V[0] * V[2];
        Q[3] = 0.5 * V[0] * (V[1] * V[1] + V[2] * V[2]) + V[3] * e.inv_g1m1;
    }
    // euler.c:197-236
    template <int DIR>
    __device__ __forceinline__ static double flux(const Eos &e, const double *V, double *F, bool &bad)
    {
        const double rho = V[0], u = V[1], v = V[2], p = V[3];
        const double un = DIR == 0 ? u : v;
        const double rhoun = rho * un;
        const double E = p * e.inv_g1m1 + 0.5 * rho * (u * u + v * v);
        bad |= (rho < RHO_FLOOR) | (p < PRS_FLOOR);
        F[0] = rhoun;
        F[1] = rhoun * u + (DIR == 0 ? p : 0.0);
        F[2] = rhoun * v + (DIR == 0 ? 0.0 : p);
        F[3] = un * (E + p);
        return fabs(un) + sqrt(e.g1 * p * fast_rcp(rho));
    }
};

// ---------------------------------------------------------------------------
// reconstruction with shared reciprocals (reconstruction.c)
// ---------------------------------------------------------------------------
constexpr double DBL_MAX_FINITE = 1.7976931348623157e308;

// reconstruction.c:157-178 for one direction: weights (1, 100, 1) / P_k
__device__ __forceinline__ void weno3_1d_fast(double u_m2, double u_m1, double u_0, double u_p1, double u_p2, double &slope,
                                              double &curv)
{
    const double ux0 = -2.0 * u_m1 + 0.5 * u_m2 + 1.5 * u_0, uxx0 = 0.5 * (u_m2 - 2.0 * u_m1 + u_0);
    const double ux1 = 0.5 * (u_p1 - u_m1), uxx1 = 0.5 * (u_m1 - 2.0 * u_0 + u_p1);
    const double ux2 = -1.5 * u_0 + 2.0 * u_p1 - 0.5 * u_p2, uxx2 = 0.5 * (u_0 - 2.0 * u_p1 + u_p2);
    const double P0 = pow4(ux0 * ux0 + R13_3 * uxx0 * uxx0 + SMALL_NUM);
    const double P1 = pow4(ux1 * ux1 + R13_3 * uxx1 * uxx1 + SMALL_NUM);
    const double P2 = pow4(ux2 * ux2 + R13_3 * uxx2 * uxx2 + SMALL_NUM);
    // w_0 : w_1 : w_2 = P1 P2 : 100 P0 P2 : P0 P1
    double n0 = P1 * P2, n1 = 100.0 * (P0 * P2), n2 = P0 * P1;
    double D = n0 + n1 + n2;
    if (!(D <= DBL_MAX_FINITE)) {   // the products overflow: one reciprocal per weight
        n0 = fast_rcp(P0); n1 = 100.0 * fast_rcp(P1); n2 = fast_rcp(P2);
        D = n0 + n1 + n2;
    }
    const double r = fast_rcp(D);
    const double w0 = n0 * r, w1 = n1 * r, w2 = n2 * r;
    slope = w0 * ux0 + w1 * ux1 + w2 * ux2;
    curv = w0 * uxx0 + w1 * uxx1 + w2 * uxx2;
}

template <int N> struct ReconFast : Recon<N> {};   // N = 0, 1: no division
// reconstruction.c:144-221
template <> struct ReconFast<2> {
    __device__ __forceinline__ static void run(const Stencil &s, double *c)
    {
        const double u_0 = s.c;
        c[0] = u_0;
        weno3_1d_fast(s.xm2, s.xm1, u_0, s.xp1, s.xp2, c[1], c[3]);
        weno3_1d_fast(s.ym2, s.ym1, u_0, s.yp1, s.yp2, c[2], c[4]);
        const double uxy0 = s.pp - u_0 - c[1] - c[2] - c[3] - c[4];
        const double uxy1 = -s.pm + u_0 + c[1] - c[2] + c[3] + c[4];
        const double uxy2 = -s.mp + u_0 - c[1] + c[2] + c[3] + c[4];
        const double uxy3 = s.mm - u_0 + c[1] + c[2] - c[3] - c[4];
        const double temp = 4.0 * (c[3] * c[3] + c[4] * c[4]);
        const double P0 = pow4(temp + uxy0 * uxy0 + SMALL_NUM), P1 = pow4(temp + uxy1 * uxy1 + SMALL_NUM);
        const double P2 = pow4(temp + uxy2 * uxy2 + SMALL_NUM), P3 = pow4(temp + uxy3 * uxy3 + SMALL_NUM);
        // w_k proportional to the product of the other three P_j
        const double p01 = P0 * P1, p23 = P2 * P3;
        double n0 = P1 * p23, n1 = P0 * p23, n2 = p01 * P3, n3 = p01 * P2;
        double D = (n0 + n1) + (n2 + n3);
        if (!(D <= DBL_MAX_FINITE)) {
            n0 = fast_rcp(P0); n1 = fast_rcp(P1); n2 = fast_rcp(P2); n3 = fast_rcp(P3);
            D = (n0 + n1) + (n2 + n3);
        }
        const double r = fast_rcp(D);
        c[5] = (n0 * r) * uxy0 + (n1 * r) * uxy1 + (n2 * r) * uxy2 + (n3 * r) * uxy3;
    }
};
// reconstruction.c:223-357: the weights take one reciprocal each and one of their sum
template <> struct ReconFast<3> {
    __device__ __forceinline__ static void run(const Stencil &s, double *coeffs)
    {
        const double gammaHi = 0.85, gammaLo = 0.85;
        const double u_0 = s.c;
        const double u_ip1 = s.xp1, u_jp1 = s.yp1, u_ip1jp1 = s.pp;
        const double u_im1 = s.xm1, u_jm1 = s.ym1, u_ip1jm1 = s.pm;
        const double u_ip2 = s.xp2, u_jp2 = s.yp2, u_im1jp1 = s.mp;
        const double u_im2 = s.xm2, u_jm2 = s.ym2, u_im1jm1 = s.mm;
        const double gamma_R4 = gammaHi;
        double gamma_R3[5];
        gamma_R3[0] = (1.0 - gammaHi) * gammaLo;
        for (int i = 1; i < 5; ++i) gamma_R3[i] = 0.25 * (1 - gammaHi) * (1 - gammaLo);
        const double u_xR4 = R41_60 * (-u_im1 + u_ip1) + R11_120 * (u_im2 - u_ip2);
        const double u_yR4 = R41_60 * (-u_jm1 + u_jp1) + R11_120 * (u_jm2 - u_jp2);
        const double u_xxR4 = -u_0 + 0.5 * (u_im1 + u_ip1);
        const double u_yyR4 = -u_0 + 0.5 * (u_jm1 + u_jp1);
        const double u_xyR4 = 0.25 * (u_im1jm1 - u_im1jp1 - u_ip1jm1 + u_ip1jp1);
        const double u_xxxR4 = R1_6 * (u_im1 - u_ip1) + R1_12 * (u_ip2 - u_im2);
        const double u_yyyR4 = R1_6 * (u_jm1 - u_jp1) + R1_12 * (u_jp2 - u_jm2);
        const double u_xxyR4 = 0.25 * (-u_im1jm1 + u_im1jp1 - u_ip1jm1 + u_ip1jp1) + 0.5 * (u_jm1 - u_jp1);
        const double u_xyyR4 = 0.5 * (u_im1 - u_ip1) + 0.25 * (u_ip1jp1 - u_im1jm1 - u_im1jp1 + u_ip1jm1);
        const double IS_R4 = (u_xR4 + 0.1 * u_xxxR4) * (u_xR4 + 0.1 * u_xxxR4) + R13_3 * (u_xxR4 * u_xxR4 + u_yyR4 * u_yyR4) +
                             (u_yR4 + 0.1 * u_yyyR4) * (u_yR4 + 0.1 * u_yyyR4) + 39.05 * (u_xxxR4 * u_xxxR4 + u_yyyR4 * u_yyyR4) +
                             R7_6 * u_xyR4 * u_xyR4 + 4.7 * (u_xxyR4 * u_xxyR4 + u_xyyR4 * u_xyyR4);
        double w_R4 = gamma_R4 * fast_rcp(pow4(IS_R4 + SMALL_NUM));
        double sum = w_R4;
        double u_xR3[5], u_yR3[5], u_xxR3[5], u_yyR3[5], u_xyR3[5], w_R3[5];
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
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            const double IS = u_xR3[i] * u_xR3[i] + u_yR3[i] * u_yR3[i] + R13_3 * (u_xxR3[i] * u_xxR3[i] + u_yyR3[i] * u_yyR3[i]) +
                              R7_6 * u_xyR3[i] * u_xyR3[i];
            w_R3[i] = gamma_R3[i] * fast_rcp(pow4(IS + SMALL_NUM));
            sum += w_R3[i];
        }
        const double rs = fast_rcp(sum);
        w_R4 = w_R4 * rs;
#pragma unroll
        for (int i = 0; i < 5; ++i) w_R3[i] = w_R3[i] * rs;
        const double wt_ratio = w_R4 * (1.0 / gammaHi);
        coeffs[0] = u_0;
#define HYPE_W4F(R4, R3) (wt_ratio * (R4 - gamma_R3[0] * R3[0] - gamma_R3[1] * R3[1] - gamma_R3[2] * R3[2] - gamma_R3[3] * R3[3] - gamma_R3[4] * R3[4]) \
                          + w_R3[0] * R3[0] + w_R3[1] * R3[1] + w_R3[2] * R3[2] + w_R3[3] * R3[3] + w_R3[4] * R3[4])
        coeffs[1] = HYPE_W4F(u_xR4, u_xR3);
        coeffs[2] = HYPE_W4F(u_yR4, u_yR3);
        coeffs[3] = HYPE_W4F(u_xxR4, u_xxR3);
        coeffs[4] = HYPE_W4F(u_yyR4, u_yyR3);
        coeffs[5] = HYPE_W4F(u_xyR4, u_xyR3);
#undef HYPE_W4F
        coeffs[6] = wt_ratio * u_xxxR4;
        coeffs[7] = wt_ratio * u_yyyR4;
        coeffs[8] = wt_ratio * u_xxyR4;
        coeffs[9] = wt_ratio * u_xyyR4;
    }
};

}  // namespace hype
