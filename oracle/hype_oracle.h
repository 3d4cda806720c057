/*
 * hype_oracle.h -- CPU restatement of HyPE-2D's right-hand side and SSP-RK time
 * loop.  TEST INFRASTRUCTURE ONLY: the checker that tests/, the smoke check and
 * bench.py's CPU baseline compare the sm_100a kernels against.  Nothing in the
 * product (hype-parallel_b200/) links or calls it.
 *
 * Pinned: tests/test_oracle_pin.py checks it bit for bit against the reference's
 * own sources (oracle/_ref, built by `make ref`) and against the committed
 * fixtures in tests/golden/ that were generated from them.
 */
#ifndef HYPE_ORACLE_H
#define HYPE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { HYO_EULER = 0, HYO_KAPILA = 1, HYO_BN = 2 };
/* values of HyPE-2D/hype.h:76 enum bndry_type */
enum { HYO_BC_WALL = 0, HYO_BC_INLET = 1, HYO_BC_PERIODIC = 2, HYO_BC_REFLECTIVE = 3, HYO_BC_TRANSMISSIVE = 4 };

typedef struct {
    int system;          /* HYO_EULER / HYO_KAPILA / HYO_BN */
    int order;           /* N: 0..3 (degree of the reconstruction) */
    int nx, ny;
    double x_min, x_max, y_min, y_max;
    double cfl;
    int bc_left, bc_right, bc_bottom, bc_top;
    double gamma1, gamma2, pi1, pi2;
    int bn_fixed_p2;     /* 0: Baer-Nunziato flux pressure as the reference has it (p2 = alpha1) */
    int conservative;    /* 0: RHSFunctionPrim, 1: RHSFunction (reconstruct conserved variables) */
    int viscous;         /* 1: the VISCOUS build of the reference (Kapila, N >= 1): viscous face fluxes */
    double mu1, mu2;     /* MU_1, MU_2 (hype.h:46-47) */
} hyo_config;

/* status codes */
enum { HYO_OK = 0, HYO_ERR_CONFIG = 1, HYO_ERR_INADMISSIBLE = 2 };

int hyo_nvar(int system);

/* One RHS evaluation: RHS = L(U) and *dt = CFL h / (2 s_max).  U, RHS are AoS
 * (cell-major, nvar interleaved), nx*ny*nvar doubles.  Returns HYO_OK, or
 * HYO_ERR_INADMISSIBLE where the reference would MPI_Abort. */
int hyo_rhs(const hyo_config *cfg, double t, const double *U, double *RHS, double *dt);

/* Time loop of HyPE-2D/hype.c:337-384: a first RHS call seeds dt, then SSP-RK
 * steps until t_final or max_steps, dt of each step taken from the last RHS
 * call of the previous step.  U is advanced in place. */
int hyo_solve(const hyo_config *cfg, double *U, double t0, double t_final, int max_steps,
              int *steps_out, double *t_out, double *dt_out);

/* Counters from the last hyo_rhs call in this thread: cells whose PAD check
 * failed (fallback to minmod), for tests. */
long hyo_last_pad_fallbacks(void);

/* Seeded initial states of the benchmark workloads (hype_oracle_ic.c), the same
 * bits as the product's include/hype_ic.h generators; U holds nx*ny*nvar doubles. */
int hyo_ic_shock_bubble(const hyo_config *cfg, uint64_t seed, int nbubbles, double *U);
int hyo_ic_bn_discs(const hyo_config *cfg, uint64_t seed, double *U);
int hyo_ic_euler_quadrants(const hyo_config *cfg, uint64_t seed, double *U);

#ifdef __cplusplus
}
#endif
#endif
