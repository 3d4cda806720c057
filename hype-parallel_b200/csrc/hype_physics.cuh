// hype_physics.cuh -- device-side physics of HyPE-2D's primitive-variable right
// hand side: stiffened-gas systems (Kapila five-equation, Baer-Nunziato, Euler),
// WENO reconstruction, admissibility checks, Rusanov flux + fluctuation.
//
// Bit compatibility: every expression keeps the operand order of the reference
// C it restates (file:line at each function) and the translation units that
// include this header are compiled with --fmad=false, so each product and sum
// rounds on its own exactly as the reference's `gcc -O2` code does on x86-64.
// IEEE division and square root are correctly rounded on both sides.
#pragma once
#include "hype_div.cuh"
#include <cstdint>
#include <utility>
#include <type_traits>

namespace hype {

enum : int { SYS_EULER = 0, SYS_KAPILA = 1, SYS_BN = 2 };
// HyPE-2D/hype.h:76 enum bndry_type
enum : int { BC_WALL = 0, BC_INLET = 1, BC_PERIODIC = 2, BC_REFLECTIVE = 3, BC_TRANSMISSIVE = 4,
             // internal: a y-slab edge inside the grid; its ghost rows are the neighbouring
             // slab's rows, kept in the slab's own halo rows (rows -3..-1 or ny..ny+2)
             BC_HALO = 5 };

// error bits reported through the device error word
enum : unsigned { ERR_INADMISSIBLE_FACE = 1u, ERR_NONFINITE = 2u, ERR_TMA_TIMEOUT = 4u, ERR_BAD_LAUNCH = 8u };

struct Eos {
    double g1, g2, pi1, pi2;
    int fix_p2;   // Baer-Nunziato: 0 = flux pressure of phase 2 read from V[8] as baer_nunziato.c:271 does
    // constants the FP64 performance form (hype_physics_fast.cuh) reads instead of
    // dividing by them; filled by derive() at the start of each of its tiles
    double g1m1, g2m1, inv_g1m1, inv_g2m1, inv_g12, g1pi1, g2pi2, c1, c2;
    __host__ __device__ void derive()
    {
        g1m1 = g1 - 1.0;
        g2m1 = g2 - 1.0;
        inv_g1m1 = 1.0 / g1m1;
        inv_g2m1 = 1.0 / g2m1;
        inv_g12 = 1.0 / (g1m1 * g2m1);
        g1pi1 = g1 * pi1;
        g2pi2 = g2 * pi2;
        c1 = g1pi1 * g2m1;   // alpha_1 gamma_1 pi_1 (gamma_2 - 1) per unit alpha_1 (kapila_5eqn.c:27)
        c2 = g2pi2 * g1m1;
    }
};

// HyPE-2D/hype.h:50-62
constexpr double PRS_FLOOR = 1.0e-12;
constexpr double RHO_FLOOR = 1.0e-14;
constexpr double SMALL_NUM = 1.0e-12;
constexpr double R1_6 = 1. / 6.;
constexpr double R13_3 = 13. / 3.;
constexpr double R7_6 = 7. / 6.;
constexpr double R11_120 = 11. / 120.;
constexpr double R1_12 = 1. / 12.;
constexpr double R41_60 = 41. / 60.;

template <int V> using ic = std::integral_constant<int, V>;
template <class F, int... Is>
__host__ __device__ __forceinline__ void static_for_impl(F &&f, std::integer_sequence<int, Is...>) { (f(ic<Is>{}), ...); }
template <int N, class F>
__host__ __device__ __forceinline__ void static_for(F &&f) { static_for_impl(f, std::make_integer_sequence<int, N>{}); }

// ---------------------------------------------------------------------------
// modal basis (reconstruction.c:11-100) and quadrature tables (hype.c:194-305)
// ---------------------------------------------------------------------------
constexpr double GP = 0.28867513459481287;

constexpr double basis_c(double x, double y, int n)
{
    return n == 0 ? 1.0 : n == 1 ? x : n == 2 ? y : n == 3 ? x * x - 1. / 12. : n == 4 ? y * y - 1. / 12.
         : n == 5 ? x * y : n == 6 ? x * (x * x - 3. / 20.) : n == 7 ? y * (y * y - 3. / 20.)
         : n == 8 ? y * (x * x - 1. / 12.) : n == 9 ? x * (y * y - 1. / 12.) : 0.0;
}
constexpr double basis_gx_c(double x, double y, int n)
{
    return n == 1 ? 1.0 : n == 3 ? 2.0 * x : n == 5 ? y : n == 6 ? 3.0 * x * x - 3. / 20. : n == 8 ? 2.0 * x * y
         : n == 9 ? (y * y - 1. / 12.) : 0.0;
}
constexpr double basis_gy_c(double x, double y, int n)
{
    return n == 2 ? 1.0 : n == 4 ? 2.0 * y : n == 5 ? x : n == 7 ? 3.0 * y * y - 3. / 20. : n == 8 ? (x * x - 1. / 12.)
         : n == 9 ? 2.0 * x * y : 0.0;
}

template <int N>
struct Quad {
    static constexpr int NDOF = (N + 1) * (N + 2) / 2;
    static constexpr int NFGP = N < 2 ? 1 : 2;
    static constexpr int NVGP = N < 2 ? 1 : 4;
    static constexpr int NNODE = 4 * NFGP;
    static constexpr double xf(int q) { return N < 2 ? 0.0 : (q == 0 ? -GP : GP); }
    static constexpr double wf(int q) { return N < 2 ? 1.0 : 0.5; }
    static constexpr double xv(int q) { return N < 2 ? 0.0 : (q < 2 ? -GP : GP); }
    static constexpr double yv(int q) { return N < 2 ? 0.0 : ((q & 1) ? GP : -GP); }
    static constexpr double wv(int q) { return N < 2 ? 1.0 : 0.25; }
    static constexpr double xn(int q)
    {
        return N < 2 ? (q == 0 ? 0.5 : q == 1 ? -0.5 : 0.0)
                     : (q < 2 ? 0.5 : q < 4 ? -0.5 : ((q & 1) ? GP : -GP));
    }
    static constexpr double yn(int q)
    {
        return N < 2 ? (q == 2 ? 0.5 : q == 3 ? -0.5 : 0.0)
                     : (q < 4 ? ((q & 1) ? GP : -GP) : (q < 6 ? 0.5 : -0.5));
    }
    // face f: 0 left (x=-1/2), 1 right, 2 bottom (y=-1/2), 3 top
    static constexpr double face_x(int f, int q) { return f == 0 ? -0.5 : f == 1 ? 0.5 : xf(q); }
    static constexpr double face_y(int f, int q) { return f == 2 ? -0.5 : f == 3 ? 0.5 : xf(q); }
    static constexpr double phi_face(int f, int q, int k) { return basis_c(face_x(f, q), face_y(f, q), k); }
    static constexpr double phi_node(int q, int k) { return basis_c(xn(q), yn(q), k); }
    static constexpr double phi_vol(int q, int k) { return basis_c(xv(q), yv(q), k); }
    static constexpr double dphi_vol_x(int q, int k) { return basis_gx_c(xv(q), yv(q), k); }
    static constexpr double dphi_vol_y(int q, int k) { return basis_gy_c(xv(q), yv(q), k); }
    // gradphiFace_x / _y (hype.c:255-285), d = 0 (x) or 1 (y)
    static constexpr double dphi_face(int f, int q, int d, int k)
    {
        return d == 0 ? basis_gx_c(face_x(f, q), face_y(f, q), k) : basis_gy_c(face_x(f, q), face_y(f, q), k);
    }
};

// Accumulate sum_k c[k]*phi(k) from 0.0 in ascending k, as the reference's
// loops do.  A term with phi == 0 is dropped at compile time: the running sum
// starts at +0 and can never become -0, so adding (c*0) = +-0 never changes it
// for finite c.
template <int NDOF, class PHI>
__device__ __forceinline__ double poly_eval(const double *c, PHI phi)
{
    double v = 0.0;
    static_for<NDOF>([&](auto k) {
        constexpr double p = PHI::template at<decltype(k)::value>();
        if constexpr (p != 0.0) {
            if constexpr (p == 1.0) v = v + c[k];
            else v = v + c[k] * p;
        }
    });
    return v;
}
template <int N, int F, int Q> struct PhiFace { template <int K> static constexpr double at() { return Quad<N>::phi_face(F, Q, K); } };
template <int N, int Q> struct PhiNode { template <int K> static constexpr double at() { return Quad<N>::phi_node(Q, K); } };
template <int N, int Q> struct PhiVol { template <int K> static constexpr double at() { return Quad<N>::phi_vol(Q, K); } };
template <int N, int Q> struct DPhiVolX { template <int K> static constexpr double at() { return Quad<N>::dphi_vol_x(Q, K); } };
template <int N, int Q> struct DPhiVolY { template <int K> static constexpr double at() { return Quad<N>::dphi_vol_y(Q, K); } };

// ---------------------------------------------------------------------------
// PDE systems (primitive-variable path)
// ---------------------------------------------------------------------------
template <int SYS> struct System;

// kapila_5eqn.c: cons [a1 r1, a2 r2, rho u, rho v, E, a1], prim [r1, r2, u, v, p, a1]
template <> struct System<SYS_KAPILA> {
    static constexpr int NV = 6;
    static constexpr int RX0 = 2, RX1 = -1, RY0 = 3, RY1 = -1;   // rhs_function_prim.c:124-125, 253-254
    static constexpr int RXV = 3, RYV = 2;                         // tangential, VISCOUS only: :126-127, :255-256
    // kapila_5eqn.c:14-35; dv(a, b) = a / b (cons2prim_dv: the bit-exact tile's row staging
    // passes the branch-free correctly rounded division, so the independent divisions overlap)
    template <class Dv>
    __device__ __forceinline__ static void cons2prim_dv(const Eos &e, const double *Q, double *V, Dv dv)
    {
        double alpha_1 = Q[5];
        double alpha_2 = 1.0 - alpha_1;
        double rho = Q[0] + Q[1];
        double u = dv(Q[2], rho);
        double v = dv(Q[3], rho);
        double E = Q[4];
        double ei = E - 0.5 * rho * (u * u + v * v);
        double G1m1 = e.g1 - 1.0;
        double G2m1 = e.g2 - 1.0;
        double p = dv(ei * G1m1 * G2m1 - alpha_1 * e.g1 * e.pi1 * G2m1 - alpha_2 * e.g2 * e.pi2 * G1m1, alpha_1 * G2m1 + alpha_2 * G1m1);
        V[0] = dv(Q[0], alpha_1);
        V[1] = dv(Q[1], alpha_2);
        V[2] = u;
        V[3] = v;
        V[4] = p;
        V[5] = alpha_1;
    }
    __device__ __forceinline__ static void cons2prim(const Eos &e, const double *Q, double *V)
    {
        cons2prim_dv(e, Q, V, [](double a, double b) { return a / b; });
    }
    // kapila_5eqn.c:41-61
    __device__ __forceinline__ static void prim2cons(const Eos &e, const double *V, double *Q)
    {
        double alpha_1 = V[5];
        double alpha_2 = 1.0 - alpha_1;
        double rho = alpha_1 * V[0] + alpha_2 * V[1];
        double u = V[2], v = V[3], p = V[4];
        double G1m1 = e.g1 - 1.0;
        double G2m1 = e.g2 - 1.0;
        double ei = (p * (alpha_1 * G2m1 + alpha_2 * G1m1) + alpha_1 * e.g1 * e.pi1 * G2m1 + alpha_2 * e.g2 * e.pi2 * G1m1) / (G1m1 * G2m1);
        double E = ei + 0.5 * rho * (u * u + v * v);
        Q[0] = alpha_1 * V[0];
        Q[1] = alpha_2 * V[1];
        Q[2] = rho * V[2];
        Q[3] = rho * V[3];
        Q[4] = E;
        Q[5] = alpha_1;
    }
    // kapila_5eqn.c:326-371
    template <int DIR>
    __device__ __forceinline__ static double flux(const Eos &e, const double *V, double *F, bool &bad)
    {
        constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
        double alpha_1 = V[5];
        double alpha_2 = 1.0 - alpha_1;
        double rho_1 = V[0], rho_2 = V[1];
        double rho = alpha_1 * rho_1 + alpha_2 * rho_2;
        double u = V[2], v = V[3], p = V[4];
        double G1m1 = e.g1 - 1.0;
        double G2m1 = e.g2 - 1.0;
        double ei = (p * (alpha_1 * G2m1 + alpha_2 * G1m1) + alpha_1 * e.g1 * e.pi1 * G2m1 + alpha_2 * e.g2 * e.pi2 * G1m1) / (G1m1 * G2m1);
        double E = ei + 0.5 * rho * (u * u + v * v);
        double un = u * nx + v * ny;
        double a1_sq = e.g1 * (p + e.pi1) / rho_1;
        double a2_sq = e.g2 * (p + e.pi2) / rho_2;
        double a_sq = (rho_1 * a1_sq * rho_2 * a2_sq) / (rho * (alpha_2 * rho_1 * a1_sq + alpha_1 * rho_2 * a2_sq));
        bad |= (a_sq < PRS_FLOOR);
        F[0] = alpha_1 * rho_1 * un;
        F[1] = alpha_2 * rho_2 * un;
        F[2] = rho * u * un + p * nx;
        F[3] = rho * v * un + p * ny;
        F[4] = (E + p) * un;
        F[5] = 0.0;
        return fabs(un) + sqrt(a_sq);
    }
    // kapila_5eqn.c:417-444
    __device__ __forceinline__ static void ncp(const Eos &e, const double *V, const double *gx, const double *gy, double *B)
    {
        double alpha_1 = V[5];
        double alpha_2 = 1.0 - alpha_1;
        double rho_1 = V[0], rho_2 = V[1], u = V[2], v = V[3], p = V[4];
        double phi_x = gx[5], phi_y = gy[5];
        double u_x = gx[2], v_y = gy[3];
        double a_1_sq = e.g1 * (p + e.pi1) / rho_1;
        double a_2_sq = e.g2 * (p + e.pi2) / rho_2;
        double K = (alpha_1 * alpha_2 * (rho_2 * a_2_sq - rho_1 * a_1_sq)) / (alpha_1 * rho_2 * a_2_sq + alpha_2 * rho_1 * a_1_sq);
        B[0] = 0.0; B[1] = 0.0; B[2] = 0.0; B[3] = 0.0; B[4] = 0.0;
        B[5] = u * phi_x + v * phi_y - K * (u_x + v_y);
    }
    static constexpr bool ncp_nonzero(int c) { return c == 5; }
    // kapila_5eqn.c:450-479
    __device__ __forceinline__ static bool pad(const Eos &e, const double *V)
    {
        double alpha_1 = V[5];
        double alpha_2 = 1.0 - alpha_1;
        double rho_1 = V[0], rho_2 = V[1];
        double rho = alpha_1 * rho_1 + alpha_2 * rho_2;
        double p = V[4];
        double a1_sq = e.g1 * (p + e.pi1) / rho_1;
        double a2_sq = e.g2 * (p + e.pi2) / rho_2;
        double a_sq = (rho_1 * a1_sq * rho_2 * a2_sq) / (rho * (alpha_2 * rho_1 * a1_sq + alpha_1 * rho_2 * a2_sq));
        if (rho < RHO_FLOOR) return false;
        if (a_sq < PRS_FLOOR) return false;
        if (alpha_1 < 0.0 || alpha_1 > 1.0) return false;
        return true;
    }

    // ---- viscous fluxes (the VISCOUS build, hype.h:36) ----
    // kapila_5eqn.c:377-411: from primitive values V and gradients g[c][dim]
    // (only u, v: g[2], g[3] are read); returns the viscous eigenvalue
    template <int DIR>
    __device__ __forceinline__ static double visc_prim(const double *V, const double (*g)[2], double mu1, double mu2, double *F)
    {
        constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
        const double r2_3 = 2. / 3., r4_3 = 4. / 3.;
        double phi = V[5];
        double mu = phi * mu1 + (1.0 - phi) * mu2;
        double u = V[2];
        double v = V[3];
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
    // kapila_5eqn.c:119-158: from conserved values Q and their gradients (g[0..3] read)
    template <int DIR>
    __device__ __forceinline__ static double visc_cons(const double *Q, const double (*g)[2], double mu1, double mu2, double *F)
    {
        constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
        const double r2_3 = 2. / 3., r4_3 = 4. / 3.;
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

    // ---- conservative-variable path (RHSFunction, rhs_function.c) ----
    // kapila_5eqn.c:67-113
    template <int DIR>
    __device__ __forceinline__ static double flux_cons(const Eos &e, const double *Q, double *F, bool &bad)
    {
        constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
        double alpha_1 = Q[5];
        double alpha_2 = 1.0 - alpha_1;
        double rho_1 = Q[0] / alpha_1;
        double rho_2 = Q[1] / alpha_2;
        double rho = Q[0] + Q[1];
        double u = Q[2] / rho;
        double v = Q[3] / rho;
        double E = Q[4];
        double ei = E - 0.5 * rho * (u * u + v * v);
        double G1m1 = e.g1 - 1.0;
        double G2m1 = e.g2 - 1.0;
        double p = (ei * G1m1 * G2m1 - alpha_1 * e.g1 * e.pi1 * G2m1 - alpha_2 * e.g2 * e.pi2 * G1m1) / (alpha_1 * G2m1 + alpha_2 * G1m1);
        double un = u * nx + v * ny;
        double a1_sq = e.g1 * (p + e.pi1) / rho_1;
        double a2_sq = e.g2 * (p + e.pi2) / rho_2;
        double a_sq = (rho_1 * a1_sq * rho_2 * a2_sq) / (rho * (alpha_2 * rho_1 * a1_sq + alpha_1 * rho_2 * a2_sq));
        bad |= (a_sq < PRS_FLOOR);
        F[0] = alpha_1 * rho_1 * un;
        F[1] = alpha_2 * rho_2 * un;
        F[2] = rho * u * un + p * nx;
        F[3] = rho * v * un + p * ny;
        F[4] = (E + p) * un;
        F[5] = 0.0;
        return fabs(un) + sqrt(a_sq);
    }
    // kapila_5eqn.c:164-198
    __device__ __forceinline__ static void ncp_cons(const Eos &e, const double *Q, const double *gx, const double *gy, double *B)
    {
        double alpha_1 = Q[5];
        double alpha_2 = 1.0 - alpha_1;
        double rho_1 = Q[0] / alpha_1;
        double rho_2 = Q[1] / alpha_2;
        double rho = Q[0] + Q[1];
        double irho = 1.0 / rho;
        double u = Q[2] / rho;
        double v = Q[3] / rho;
        double E = Q[4];
        double ei = E - 0.5 * rho * (u * u + v * v);
        double G1m1 = e.g1 - 1.0;
        double G2m1 = e.g2 - 1.0;
        double p = (ei * G1m1 * G2m1 - alpha_1 * e.g1 * e.pi1 * G2m1 - alpha_2 * e.g2 * e.pi2 * G1m1) / (alpha_1 * G2m1 + alpha_2 * G1m1);
        double a1_sq = e.g1 * (p + e.pi1) / rho_1;
        double a2_sq = e.g2 * (p + e.pi2) / rho_2;
        double K = alpha_1 * alpha_2 * (rho_2 * a2_sq - rho_1 * a1_sq) / (alpha_1 * rho_2 * a2_sq + alpha_2 * rho_1 * a1_sq);
        double alpha1_x = gx[5], alpha1_y = gy[5];
        double u_x = irho * irho * (gx[2] * rho - Q[2] * (gx[0] + gx[1]));
        double v_y = irho * irho * (gy[3] * rho - Q[3] * (gy[0] + gy[1]));
        B[0] = 0.0; B[1] = 0.0; B[2] = 0.0; B[3] = 0.0; B[4] = 0.0;
        B[5] = u * alpha1_x + v * alpha1_y - K * (u_x + v_y);
    }
    static constexpr bool ncp_cons_nonzero(int c) { return c == 5; }
    // kapila_5eqn.c:247-283; its alpha test (line 278) rejects every alpha_1 != 1
    __device__ __forceinline__ static bool pad_cons(const Eos &e, const double *Q)
    {
        double alpha_1 = Q[5];
        double alpha_2 = 1.0 - alpha_1;
        double rho_1 = Q[0] / alpha_1;
        double rho_2 = Q[1] / alpha_2;
        double rho = Q[0] + Q[1];
        double u = Q[2] / rho;
        double v = Q[3] / rho;
        double E = Q[4];
        double ei = E - 0.5 * rho * (u * u + v * v);
        double G1m1 = e.g1 - 1.0;
        double G2m1 = e.g2 - 1.0;
        double p = (ei * G1m1 * G2m1 - alpha_1 * e.g1 * e.pi1 * G2m1 - alpha_2 * e.g2 * e.pi2 * G1m1) / (alpha_1 * G2m1 + alpha_2 * G1m1);
        double a1_sq = e.g1 * (p + e.pi1) / rho_1;
        double a2_sq = e.g2 * (p + e.pi2) / rho_2;
        double a_sq = (rho_1 * a1_sq * rho_2 * a2_sq) / (rho * (alpha_2 * rho_1 * a1_sq + alpha_1 * rho_2 * a2_sq));
        if (rho < RHO_FLOOR) return false;
        if (a_sq < PRS_FLOOR) return false;
        if (alpha_1 < 1.0 || alpha_1 > 1.0) return false;
        return true;
    }
};

// baer_nunziato.c: cons [a1 r1, a1 r1 u1, a1 r1 v1, a1 E1, a2 r2, a2 r2 u2, a2 r2 v2, a2 E2, a1]
//                  prim [r1, u1, v1, p1, r2, u2, v2, p2, a1]
template <> struct System<SYS_BN> {
    static constexpr int NV = 9;
    static constexpr int RX0 = 1, RX1 = 5, RY0 = 2, RY1 = 6;   // rhs_function_prim.c:115-117, 244-246
    // baer_nunziato.c:14-41; dv(a, b) = a / b (cons2prim_dv as for the Kapila system)
    __device__ __forceinline__ static void cons2prim(const Eos &e, const double *Q, double *V)
    {
        cons2prim_dv(e, Q, V, [](double a, double b) { return a / b; });
    }
    template <class Dv>
    __device__ __forceinline__ static void cons2prim_dv(const Eos &e, const double *Q, double *V, Dv dv)
    {
        double phi_1 = Q[8];
        double phi_2 = 1.0 - Q[8];
        double rho_1 = dv(Q[0], phi_1);
        double rho_2 = dv(Q[4], phi_2);
        double u_1 = dv(Q[1], Q[0]), v_1 = dv(Q[2], Q[0]);
        double u_2 = dv(Q[5], Q[4]), v_2 = dv(Q[6], Q[4]);
        double E_1 = dv(Q[3], phi_1);
        double E_2 = dv(Q[7], phi_2);
        double p_1 = (e.g1 - 1.0) * (E_1 - 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1)) - e.g1 * e.pi1;
        double p_2 = (e.g2 - 1.0) * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e.g2 * e.pi2;
        V[0] = rho_1; V[1] = u_1; V[2] = v_1; V[3] = p_1;
        V[4] = rho_2; V[5] = u_2; V[6] = v_2; V[7] = p_2;
        V[8] = phi_1;
    }
    // baer_nunziato.c:47-60
    __device__ __forceinline__ static void prim2cons(const Eos &e, const double *V, double *Q)
    {
        Q[0] = V[8] * V[0];
        Q[1] = Q[0] * V[1];
        Q[2] = Q[0] * V[2];
        Q[3] = Q[0] * (0.5 * (V[1] * V[1] + V[2] * V[2]) + (V[3] + e.g1 * e.pi1) / (V[0] * (e.g1 - 1.0)));
        Q[4] = (1.0 - V[8]) * V[4];
        Q[5] = Q[4] * V[5];
        Q[6] = Q[4] * V[6];
        Q[7] = Q[4] * (0.5 * (V[5] * V[5] + V[6] * V[6]) + (V[7] + e.g2 * e.pi2) / (V[4] * (e.g2 - 1.0)));
        Q[8] = V[8];
    }
    // baer_nunziato.c:256-321 (phase-2 flux pressure from V[8] unless fix_p2)
    template <int DIR>
    __device__ __forceinline__ static double flux(const Eos &e, const double *V, double *F, bool &bad)
    {
        constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
        double phi_1 = V[8];
        double phi_2 = 1.0 - V[8];
        double rho_1 = V[0], rho_2 = V[4];
        double u_1 = V[1], v_1 = V[2];
        double u_2 = V[5], v_2 = V[6];
        double p_1 = V[3];
        double p_2 = e.fix_p2 ? V[7] : V[8];
        double E_1 = (p_1 + e.g1 * e.pi1) / (e.g1 - 1.0) + 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1);
        double E_2 = (p_2 + e.g2 * e.pi2) / (e.g2 - 1.0) + 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2);
        double un_1 = nx * u_1 + ny * v_1;
        double un_2 = nx * u_2 + ny * v_2;
        bad |= (rho_1 < RHO_FLOOR) | (rho_2 < RHO_FLOOR) | ((p_1 + e.pi1) < PRS_FLOOR) | ((p_2 + e.pi2) < PRS_FLOOR);
        F[0] = phi_1 * rho_1 * un_1;
        F[1] = phi_1 * (rho_1 * u_1 * un_1 + nx * p_1);
        F[2] = phi_1 * (rho_1 * v_1 * un_1 + ny * p_1);
        F[3] = phi_1 * un_1 * (E_1 + p_1);
        F[4] = phi_2 * rho_2 * un_2;
        F[5] = phi_2 * (rho_2 * u_2 * un_2 + nx * p_2);
        F[6] = phi_2 * (rho_2 * v_2 * un_2 + ny * p_2);
        F[7] = phi_2 * un_2 * (E_2 + p_2);
        F[8] = 0.0;
        double s_1 = fabs(un_1) + sqrt(e.g1 * (p_1 + e.pi1) / rho_1);
        double s_2 = fabs(un_2) + sqrt(e.g2 * (p_2 + e.pi2) / rho_2);
        return (s_1 < s_2) ? s_2 : s_1;
    }
    // baer_nunziato.c:327-344
    __device__ __forceinline__ static void ncp(const Eos &, const double *V, const double *gx, const double *gy, double *B)
    {
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
    static constexpr bool ncp_nonzero(int c) { return c != 0 && c != 4; }
    // baer_nunziato.c:350-385
    __device__ __forceinline__ static bool pad(const Eos &e, const double *V)
    {
        bool ok = true;
        if (V[0] < RHO_FLOOR) ok = false;
        if (V[4] < RHO_FLOOR) ok = false;
        if ((V[3] + e.pi1) < PRS_FLOOR) ok = false;
        if ((V[7] + e.pi2) < PRS_FLOOR) ok = false;
        if (V[8] < 0.0 || V[8] > 1.0) ok = false;
        return ok;
    }

    // ---- conservative-variable path (RHSFunction, rhs_function.c) ----
    // baer_nunziato.c:66-131
    template <int DIR>
    __device__ __forceinline__ static double flux_cons(const Eos &e, const double *Q, double *F, bool &bad)
    {
        constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
        double phi_1 = Q[8];
        double phi_2 = 1.0 - Q[8];
        double rho_1 = Q[0] / phi_1;
        double rho_2 = Q[4] / phi_2;
        double u_1 = Q[1] / Q[0], v_1 = Q[2] / Q[0];
        double u_2 = Q[5] / Q[4], v_2 = Q[6] / Q[4];
        double E_1 = Q[3] / phi_1;
        double E_2 = Q[7] / phi_2;
        double p_1 = (e.g1 - 1.0) * (E_1 - 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1)) - e.g1 * e.pi1;
        double p_2 = (e.g2 - 1.0) * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e.g2 * e.pi2;
        double un_1 = nx * u_1 + ny * v_1;
        double un_2 = nx * u_2 + ny * v_2;
        bad |= (rho_1 < RHO_FLOOR) | (rho_2 < RHO_FLOOR) | ((p_1 + e.pi1) < PRS_FLOOR) | ((p_2 + e.pi2) < PRS_FLOOR);
        F[0] = phi_1 * rho_1 * un_1;
        F[1] = phi_1 * (rho_1 * u_1 * un_1 + nx * p_1);
        F[2] = phi_1 * (rho_1 * v_1 * un_1 + ny * p_1);
        F[3] = phi_1 * un_1 * (E_1 + p_1);
        F[4] = phi_2 * rho_2 * un_2;
        F[5] = phi_2 * (rho_2 * u_2 * un_2 + nx * p_2);
        F[6] = phi_2 * (rho_2 * v_2 * un_2 + ny * p_2);
        F[7] = phi_2 * un_2 * (E_2 + p_2);
        F[8] = 0.0;
        double s_1 = fabs(un_1) + sqrt(e.g1 * (p_1 + e.pi1) / rho_1);
        double s_2 = fabs(un_2) + sqrt(e.g2 * (p_2 + e.pi2) / rho_2);
        return (s_1 < s_2) ? s_2 : s_1;
    }
    // baer_nunziato.c:137-165: u_I = u_1, p_I = p_2 from the phase-2 state
    __device__ __forceinline__ static void ncp_cons(const Eos &e, const double *Q, const double *gx, const double *gy, double *B)
    {
        double phi_2 = 1.0 - Q[8];
        double rho_2 = Q[4] / phi_2;
        double u_1 = Q[1] / Q[0], v_1 = Q[2] / Q[0];
        double u_2 = Q[5] / Q[4], v_2 = Q[6] / Q[4];
        double E_2 = Q[7] / phi_2;
        double p_I = (e.g2 - 1.0) * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e.g2 * e.pi2;
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
    static constexpr bool ncp_cons_nonzero(int c) { return c != 0 && c != 4; }
    // baer_nunziato.c:207-250
    __device__ __forceinline__ static bool pad_cons(const Eos &e, const double *Q)
    {
        bool ok = true;
        double phi_1 = Q[8];
        double phi_2 = 1.0 - Q[8];
        double rho_1 = Q[0] / phi_1;
        double rho_2 = Q[4] / phi_2;
        double u_1 = Q[1] / Q[0], v_1 = Q[2] / Q[0];
        double u_2 = Q[5] / Q[4], v_2 = Q[6] / Q[4];
        double E_1 = Q[3] / phi_1;
        double E_2 = Q[7] / phi_2;
        double p_1 = (e.g1 - 1.0) * (E_1 - 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1)) - e.g1 * e.pi1;
        double p_2 = (e.g2 - 1.0) * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e.g2 * e.pi2;
        if (rho_1 < RHO_FLOOR) ok = false;
        if (rho_2 < RHO_FLOOR) ok = false;
        if ((p_1 + e.pi1) < PRS_FLOOR) ok = false;
        if ((p_2 + e.pi2) < PRS_FLOOR) ok = false;
        if (phi_1 < 0.0 || phi_1 > 1.0) ok = false;
        return ok;
    }
};

// euler.c: cons [rho, rho u, rho v, E], prim [rho, u, v, p], ideal gas GAMMA_1
template <> struct System<SYS_EULER> {
    static constexpr int NV = 4;
    static constexpr int RX0 = 1, RX1 = -1, RY0 = 2, RY1 = -1;   // rhs_function_prim.c:101-102, 230-231
    // euler.c:14-23
    __device__ __forceinline__ static void cons2prim(const Eos &e, const double *Q, double *V)
    {
        double irho = 1.0 / Q[0];
        V[0] = Q[0];
        V[1] = irho * Q[1];
        V[2] = irho * Q[2];
        V[3] = (e.g1 - 1.0) * (Q[3] - 0.5 * irho * (Q[1] * Q[1] + Q[2] * Q[2]));
    }
    // euler.c:29-38
    __device__ __forceinline__ static void prim2cons(const Eos &e, const double *V, double *Q)
    {
        double ei = (V[3]) / (e.g1 - 1.0);
        double k = 0.5 * V[0] * (V[1] * V[1] + V[2] * V[2]);
        Q[0] = V[0];
        Q[1] = V[0] * V[1];
        Q[2] = V[0] * V[2];
        Q[3] = k + ei;
    }
    // euler.c:197-236
    template <int DIR>
    __device__ __forceinline__ static double flux(const Eos &e, const double *V, double *F, bool &bad)
    {
        constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
        double rho = V[0], u = V[1], v = V[2];
        double un = nx * u + ny * v;
        double rhoun = rho * un;
        double p = V[3];
        double E = p / (e.g1 - 1.0) + 0.5 * rho * (u * u + v * v);
        bad |= (rho < RHO_FLOOR) | (p < PRS_FLOOR);
        F[0] = rhoun;
        F[1] = rhoun * u + nx * p;
        F[2] = rhoun * v + ny * p;
        F[3] = un * (E + p);
        return fabs(un) + sqrt(e.g1 * p / rho);
    }
    // euler.c:278-286
    __device__ __forceinline__ static void ncp(const Eos &, const double *, const double *, const double *, double *B)
    {
        B[0] = 0.0; B[1] = 0.0; B[2] = 0.0; B[3] = 0.0;
    }
    static constexpr bool ncp_nonzero(int) { return false; }
    // euler.c:292-310
    __device__ __forceinline__ static bool pad(const Eos &, const double *V)
    {
        bool ok = true;
        if (V[0] < RHO_FLOOR) ok = false;
        if (V[3] < PRS_FLOOR) ok = false;
        return ok;
    }

    // ---- conservative-variable path (RHSFunction, rhs_function.c) ----
    // euler.c:44-84
    template <int DIR>
    __device__ __forceinline__ static double flux_cons(const Eos &e, const double *Q, double *F, bool &bad)
    {
        constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
        double rho = Q[0];
        double irho = 1.0 / rho;
        double u = irho * Q[1];
        double v = irho * Q[2];
        double un = nx * u + ny * v;
        double rhoun = rho * un;
        double E = Q[3];
        double p = (e.g1 - 1.0) * (E - 0.5 * rho * (u * u + v * v));
        bad |= (rho < RHO_FLOOR) | (p < PRS_FLOOR);
        F[0] = rhoun;
        F[1] = rhoun * u + nx * p;
        F[2] = rhoun * v + ny * p;
        F[3] = un * (E + p);
        return fabs(un) + sqrt(e.g1 * p * irho);
    }
    __device__ __forceinline__ static void ncp_cons(const Eos &, const double *, const double *, const double *, double *B)
    {
        B[0] = 0.0; B[1] = 0.0; B[2] = 0.0; B[3] = 0.0;
    }
    static constexpr bool ncp_cons_nonzero(int) { return false; }
    // euler.c:169-191
    __device__ __forceinline__ static bool pad_cons(const Eos &e, const double *Q)
    {
        bool ok = true;
        double rho = Q[0];
        double irho = 1.0 / rho;
        double u = irho * Q[1];
        double v = irho * Q[2];
        double E = Q[3];
        double p = (e.g1 - 1.0) * (E - 0.5 * rho * (u * u + v * v));
        if (rho < RHO_FLOOR) ok = false;
        if (p < PRS_FLOOR) ok = false;
        return ok;
    }
};

// ---------------------------------------------------------------------------
// reconstruction (reconstruction.c)
// ---------------------------------------------------------------------------
struct Stencil {
    double c;
    double xm2, xm1, xp1, xp2;
    double ym2, ym1, yp1, yp2;
    double pp, pm, mp, mm;   // (i+1,j+1) (i+1,j-1) (i-1,j+1) (i-1,j-1)
};

// reconstruction.c:106-117
__device__ __forceinline__ double minmod(double a, double b)
{
    if (a * b < 0.0) return 0.0;
    return (fabs(a) < fabs(b)) ? a : b;
}
// reconstruction.c:123-127
__device__ __forceinline__ double pow4(double a) { double a2 = a * a; return a2 * a2; }

// reconstruction.c:157-178 for one direction
__device__ __forceinline__ void weno3_1d(double u_m2, double u_m1, double u_0, double u_p1, double u_p2, double &slope, double &curv)
{
    const double central_cell_wt = 100.0;
    double ux0 = -2.0 * u_m1 + 0.5 * u_m2 + 1.5 * u_0, uxx0 = 0.5 * (u_m2 - 2.0 * u_m1 + u_0);
    double ux1 = 0.5 * (u_p1 - u_m1),                  uxx1 = 0.5 * (u_m1 - 2.0 * u_0 + u_p1);
    double ux2 = -1.5 * u_0 + 2.0 * u_p1 - 0.5 * u_p2, uxx2 = 0.5 * (u_0 - 2.0 * u_p1 + u_p2);
    double IS0 = ux0 * ux0 + R13_3 * uxx0 * uxx0; double w0 = 1.0 / (pow4(IS0 + SMALL_NUM));
    double IS1 = ux1 * ux1 + R13_3 * uxx1 * uxx1; double w1 = central_cell_wt / (pow4(IS1 + SMALL_NUM));
    double IS2 = ux2 * ux2 + R13_3 * uxx2 * uxx2; double w2 = 1.0 / (pow4(IS2 + SMALL_NUM));
    double total = w0 + w1 + w2;
    w0 = w0 / total;
    w1 = w1 / total;
    w2 = w2 / total;
    slope = w0 * ux0 + w1 * ux1 + w2 * ux2;
    curv = w0 * uxx0 + w1 * uxx1 + w2 * uxx2;
}

// reconstruction.c:157-178 and :144-221 with the branch-free correctly rounded
// division of hype_div.cuh: the bits of weno3_1d / Recon<2>.  Every weight is
// gamma_k / d_k with d_k = (IS_k + 1e-12)^4 and is then divided by the weights'
// sum; with every d_k in [2^-400, 2^400] all those operands and quotients lie in
// cr_div_core's range (w_k in [2^-400, 100 2^400], w_k / sum >= 2^-810), so one
// check per stencil direction replaces one per division.  Outside it (or for a
// NaN) `special` is set and the caller recomputes with Recon<2>.
__device__ __forceinline__ bool cr_denominator_ok(double d) { return d >= 0x1p-400 && d <= 0x1p400; }

__device__ __forceinline__ void weno3_1d_cr(double u_m2, double u_m1, double u_0, double u_p1, double u_p2, double &slope,
                                            double &curv, bool &sp)
{
    const double central_cell_wt = 100.0;
    double ux0 = -2.0 * u_m1 + 0.5 * u_m2 + 1.5 * u_0, uxx0 = 0.5 * (u_m2 - 2.0 * u_m1 + u_0);
    double ux1 = 0.5 * (u_p1 - u_m1),                  uxx1 = 0.5 * (u_m1 - 2.0 * u_0 + u_p1);
    double ux2 = -1.5 * u_0 + 2.0 * u_p1 - 0.5 * u_p2, uxx2 = 0.5 * (u_0 - 2.0 * u_p1 + u_p2);
    double IS0 = ux0 * ux0 + R13_3 * uxx0 * uxx0; const double d0 = pow4(IS0 + SMALL_NUM);
    double IS1 = ux1 * ux1 + R13_3 * uxx1 * uxx1; const double d1 = pow4(IS1 + SMALL_NUM);
    double IS2 = ux2 * ux2 + R13_3 * uxx2 * uxx2; const double d2 = pow4(IS2 + SMALL_NUM);
    sp |= !(cr_denominator_ok(d0) && cr_denominator_ok(d1) && cr_denominator_ok(d2));
    double w0 = cr_div_core(1.0, d0);
    double w1 = cr_div_core(central_cell_wt, d1);
    double w2 = cr_div_core(1.0, d2);
    double total = w0 + w1 + w2;
    w0 = cr_div_core(w0, total);
    w1 = cr_div_core(w1, total);
    w2 = cr_div_core(w2, total);
    slope = w0 * ux0 + w1 * ux1 + w2 * ux2;
    curv = w0 * uxx0 + w1 * uxx1 + w2 * uxx2;
}
struct Recon2Cr {
    __device__ __forceinline__ static void run(const Stencil &s, double *c, bool &sp)
    {
        double u_0 = s.c;
        c[0] = u_0;
        weno3_1d_cr(s.xm2, s.xm1, u_0, s.xp1, s.xp2, c[1], c[3], sp);
        weno3_1d_cr(s.ym2, s.ym1, u_0, s.yp1, s.yp2, c[2], c[4], sp);
        double uxy0 =  s.pp - u_0 - c[1] - c[2] - c[3] - c[4];
        double uxy1 = -s.pm + u_0 + c[1] - c[2] + c[3] + c[4];
        double uxy2 = -s.mp + u_0 - c[1] + c[2] + c[3] + c[4];
        double uxy3 =  s.mm - u_0 + c[1] + c[2] - c[3] - c[4];
        double temp = 4.0 * (c[3] * c[3] + c[4] * c[4]);
        double IS0 = temp + uxy0 * uxy0; const double d0 = pow4(IS0 + SMALL_NUM);
        double IS1 = temp + uxy1 * uxy1; const double d1 = pow4(IS1 + SMALL_NUM);
        double IS2 = temp + uxy2 * uxy2; const double d2 = pow4(IS2 + SMALL_NUM);
        double IS3 = temp + uxy3 * uxy3; const double d3 = pow4(IS3 + SMALL_NUM);
        sp |= !(cr_denominator_ok(d0) && cr_denominator_ok(d1) && cr_denominator_ok(d2) && cr_denominator_ok(d3));
        double w0 = cr_div_core(1.0, d0), w1 = cr_div_core(1.0, d1), w2 = cr_div_core(1.0, d2), w3 = cr_div_core(1.0, d3);
        double total = w0 + w1 + w2 + w3;
        w0 = cr_div_core(w0, total); w1 = cr_div_core(w1, total); w2 = cr_div_core(w2, total); w3 = cr_div_core(w3, total);
        c[5] = w0 * uxy0 + w1 * uxy1 + w2 * uxy2 + w3 * uxy3;
    }
};

template <int N> struct Recon;
template <> struct Recon<0> {
    __device__ __forceinline__ static void run(const Stencil &s, double *c) { c[0] = s.c; }
};
// reconstruction.c:129-142
template <> struct Recon<1> {
    __device__ __forceinline__ static void run(const Stencil &s, double *c)
    {
        c[0] = s.c;
        c[1] = minmod(s.xp1 - s.c, s.c - s.xm1);
        c[2] = minmod(s.yp1 - s.c, s.c - s.ym1);
    }
};
// reconstruction.c:144-221
template <> struct Recon<2> {
    __device__ __forceinline__ static void run(const Stencil &s, double *c)
    {
        double u_0 = s.c;
        c[0] = u_0;
        weno3_1d(s.xm2, s.xm1, u_0, s.xp1, s.xp2, c[1], c[3]);
        weno3_1d(s.ym2, s.ym1, u_0, s.yp1, s.yp2, c[2], c[4]);
        double uxy0 =  s.pp - u_0 - c[1] - c[2] - c[3] - c[4];
        double uxy1 = -s.pm + u_0 + c[1] - c[2] + c[3] + c[4];
        double uxy2 = -s.mp + u_0 - c[1] + c[2] + c[3] + c[4];
        double uxy3 =  s.mm - u_0 + c[1] + c[2] - c[3] - c[4];
        double temp = 4.0 * (c[3] * c[3] + c[4] * c[4]);
        double IS0 = temp + uxy0 * uxy0; double w0 = 1.0 / (pow4(IS0 + SMALL_NUM));
        double IS1 = temp + uxy1 * uxy1; double w1 = 1.0 / (pow4(IS1 + SMALL_NUM));
        double IS2 = temp + uxy2 * uxy2; double w2 = 1.0 / (pow4(IS2 + SMALL_NUM));
        double IS3 = temp + uxy3 * uxy3; double w3 = 1.0 / (pow4(IS3 + SMALL_NUM));
        double total = w0 + w1 + w2 + w3;
        w0 = w0 / total; w1 = w1 / total; w2 = w2 / total; w3 = w3 / total;
        c[5] = w0 * uxy0 + w1 * uxy1 + w2 * uxy2 + w3 * uxy3;
    }
};
// reconstruction.c:223-357
template <> struct Recon<3> {
    __device__ __forceinline__ static void run(const Stencil &s, double *coeffs)
    {
        const double gammaHi = 0.85, gammaLo = 0.85;
        double u_0 = s.c;
        double u_ip1 = s.xp1, u_jp1 = s.yp1, u_ip1jp1 = s.pp;
        double u_im1 = s.xm1, u_jm1 = s.ym1, u_ip1jm1 = s.pm;
        double u_ip2 = s.xp2, u_jp2 = s.yp2, u_im1jp1 = s.mp;
        double u_im2 = s.xm2, u_jm2 = s.ym2, u_im1jm1 = s.mm;
        double gamma_R4 = gammaHi;
        double gamma_R3[5];
        gamma_R3[0] = (1.0 - gammaHi) * gammaLo;
        for (int i = 1; i < 5; ++i) gamma_R3[i] = 0.25 * (1 - gammaHi) * (1 - gammaLo);
        double u_xR4 = R41_60 * (-u_im1 + u_ip1) + R11_120 * (u_im2 - u_ip2);
        double u_yR4 = R41_60 * (-u_jm1 + u_jp1) + R11_120 * (u_jm2 - u_jp2);
        double u_xxR4 = -u_0 + 0.5 * (u_im1 + u_ip1);
        double u_yyR4 = -u_0 + 0.5 * (u_jm1 + u_jp1);
        double u_xyR4 = 0.25 * (u_im1jm1 - u_im1jp1 - u_ip1jm1 + u_ip1jp1);
        double u_xxxR4 = R1_6 * (u_im1 - u_ip1) + R1_12 * (u_ip2 - u_im2);
        double u_yyyR4 = R1_6 * (u_jm1 - u_jp1) + R1_12 * (u_jp2 - u_jm2);
        double u_xxyR4 = 0.25 * (-u_im1jm1 + u_im1jp1 - u_ip1jm1 + u_ip1jp1) + 0.5 * (u_jm1 - u_jp1);
        double u_xyyR4 = 0.5 * (u_im1 - u_ip1) + 0.25 * (u_ip1jp1 - u_im1jm1 - u_im1jp1 + u_ip1jm1);
        double IS_R4 = (u_xR4 + 0.1 * u_xxxR4) * (u_xR4 + 0.1 * u_xxxR4) + R13_3 * (u_xxR4 * u_xxR4 + u_yyR4 * u_yyR4) +
                       (u_yR4 + 0.1 * u_yyyR4) * (u_yR4 + 0.1 * u_yyyR4) + 39.05 * (u_xxxR4 * u_xxxR4 + u_yyyR4 * u_yyyR4) +
                       R7_6 * u_xyR4 * u_xyR4 + 4.7 * (u_xxyR4 * u_xxyR4 + u_xyyR4 * u_xyyR4);
        double w_R4 = gamma_R4 / (pow4(IS_R4 + SMALL_NUM));
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
            double IS = u_xR3[i] * u_xR3[i] + u_yR3[i] * u_yR3[i] + R13_3 * (u_xxR3[i] * u_xxR3[i] + u_yyR3[i] * u_yyR3[i]) + R7_6 * u_xyR3[i] * u_xyR3[i];
            w_R3[i] = gamma_R3[i] / (pow4(IS + SMALL_NUM));
            sum += w_R3[i];
        }
        w_R4 = w_R4 / sum;
#pragma unroll
        for (int i = 0; i < 5; ++i) w_R3[i] = w_R3[i] / sum;
        double wt_ratio = w_R4 / gamma_R4;
        coeffs[0] = u_0;
#define HYPE_W4(R4, R3) (wt_ratio * (R4 - gamma_R3[0] * R3[0] - gamma_R3[1] * R3[1] - gamma_R3[2] * R3[2] - gamma_R3[3] * R3[3] - gamma_R3[4] * R3[4]) \
                         + w_R3[0] * R3[0] + w_R3[1] * R3[1] + w_R3[2] * R3[2] + w_R3[3] * R3[3] + w_R3[4] * R3[4])
        coeffs[1] = HYPE_W4(u_xR4, u_xR3);
        coeffs[2] = HYPE_W4(u_yR4, u_yR3);
        coeffs[3] = HYPE_W4(u_xxR4, u_xxR3);
        coeffs[4] = HYPE_W4(u_yyR4, u_yyR3);
        coeffs[5] = HYPE_W4(u_xyR4, u_xyR3);
#undef HYPE_W4
        coeffs[6] = wt_ratio * u_xxxR4;
        coeffs[7] = wt_ratio * u_yyyR4;
        coeffs[8] = wt_ratio * u_xxyR4;
        coeffs[9] = wt_ratio * u_xyyR4;
    }
};

// The unlimited central coefficients (u_coeffs) Reconstruct returns beside
// the WENO ones (reconstruction.c:139-141, 172-174, 195-196, 217, 258-267);
// the VISCOUS build takes face gradients from them.  N = 0: the reference
// leaves them unset, so the viscous path starts at N = 1.
template <int N> struct UCoef;
template <> struct UCoef<1> {
    __device__ __forceinline__ static void run(const Stencil &s, double *uc)
    {
        uc[0] = s.c;
        uc[1] = 0.5 * (s.xp1 - s.xm1);
        uc[2] = 0.5 * (s.yp1 - s.ym1);
    }
};
template <> struct UCoef<2> {
    __device__ __forceinline__ static void run(const Stencil &s, double *uc)
    {
        const double u_0 = s.c;
        uc[0] = u_0;
        uc[1] = 0.5 * (s.xp1 - s.xm1);
        uc[3] = 0.5 * (s.xm1 - 2.0 * u_0 + s.xp1);
        uc[2] = 0.5 * (s.yp1 - s.ym1);
        uc[4] = 0.5 * (s.ym1 - 2.0 * u_0 + s.yp1);
        uc[5] = 0.25 * (s.pp - s.pm - s.mp + s.mm);
    }
};
template <> struct UCoef<3> {
    __device__ __forceinline__ static void run(const Stencil &s, double *uc)
    {
        const double u_0 = s.c;
        const double u_ip1 = s.xp1, u_jp1 = s.yp1, u_ip1jp1 = s.pp, u_im1 = s.xm1, u_jm1 = s.ym1, u_ip1jm1 = s.pm;
        const double u_ip2 = s.xp2, u_jp2 = s.yp2, u_im1jp1 = s.mp, u_im2 = s.xm2, u_jm2 = s.ym2, u_im1jm1 = s.mm;
        uc[0] = u_0;
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
};

}  // namespace hype
