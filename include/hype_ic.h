/*
 * hype_ic.h -- seeded initial states for the workloads the benchmarks and
 * tests run.  They stand in for HyPE-2D's hard-wired InitialCondition
 * (initialize_solution.c:12-15) and have no entry-point counterpart in the
 * reference; SmoothVortex restates kapila_5eqn.c:527-562.  Outputs are in the
 * Vec layout of hype_gpu.h (nx*ny cells, nvar interleaved), host memory.
 */
#ifndef HYPE_IC_H
#define HYPE_IC_H
#include <stdint.h>
#include "hype_gpu.h"
#ifdef __cplusplus
extern "C" {
#endif

/* Kapila: liquid (phase 1) at rest, p = 1e5, rho1 = 1000, rho2 = 1, with
 * `nbubbles` gas discs (radius U[0.1,0.2], centre U[0.4,0.6]^2 in unit-square
 * coordinates, alpha_1 = 1e-6 inside, tanh edge two cells wide) and a planar
 * shock in x < 0.1 whose pressure ratio is U[10,1000] (stiffened-gas
 * Rankine-Hugoniot state behind it). */
HYPE_API int hype_ic_shock_bubble(const hype_config *cfg, uint64_t seed, int nbubbles, double *U);

/* Baer-Nunziato: alpha_1 = 0.01 + eight tanh-edged discs, clipped to 0.99;
 * densities 0.5..2 x (1000, 1), velocities |u| <= 50, pressures 1e5..1e7, all
 * smooth random Fourier fields. */
HYPE_API int hype_ic_bn_discs(const hype_config *cfg, uint64_t seed, double *U);

/* Euler (gamma1): four constant quadrants, rho U[0.1,1.5], p U[0.03,1.5], u,v U[-1,1]. */
HYPE_API int hype_ic_euler_quadrants(const hype_config *cfg, uint64_t seed, double *U);

/* Kapila SmoothVortex (kapila_5eqn.c:527-562), 5x5 Gauss cell averages. */
HYPE_API int hype_ic_smooth_vortex(const hype_config *cfg, double *U);

#ifdef __cplusplus
}
#endif
#endif
