/*
 * hype_ref_cfg.h -- force-included (gcc -include) ahead of the reference's
 * HyPE-2D sources when oracle/Makefile compiles them into oracle/_ref.
 * TEST INFRASTRUCTURE ONLY.
 *
 * It defines the include guard of HyPE-2D/hype.h (HYPE_H_), so the sources'
 * own `#include "hype.h"` becomes empty, and restates that header's
 * declarations (HyPE-2D/hype.h:37-309) with three changes that make one set of
 * reference sources serve every configuration the oracle needs:
 *   - the PDE system (#define EULER / KAPILA_5EQN / BAER_NUNZIATO) and nVar
 *     come from the command line (hype.h:33-37 hard-codes KAPILA_5EQN, 6);
 *   - the stiffened-gas constants GAMMA_1, GAMMA_2, PI_1, PI_2 (hype.h:42-45,
 *     `static const` there) and the viscosities MU_1, MU_2 (hype.h:46-47) are
 *     run-time globals set by the driver, so the EOS of each config (e.g.
 *     PI_1 = 6e8) needs no rebuild.  Expressions in
 *     the sources evaluate identically: a constant folded at compile time and
 *     the same IEEE operation at run time round the same way;
 *   - PETSc comes from petsc_mini.h (one rank).
 * Every other constant keeps its value from hype.h:46-62.
 */
#ifndef HYPE_H_
#define HYPE_H_

#include <stdio.h>
#include <string.h>
#include "petsc_mini.h"

#ifndef HYPE_REF_NVAR
#error "HYPE_REF_NVAR must be defined (4 Euler, 6 Kapila, 9 Baer-Nunziato)"
#endif
#define nVar HYPE_REF_NVAR
#define DIM 2

extern PetscReal GAMMA_1, GAMMA_2, PI_1, PI_2;
extern PetscReal MU_1, MU_2;   /* hype.h:46-47 (1.0e-2, 0.0): run-time like the EOS constants */
static const PetscReal G_A  = 9.8;

static const PetscReal prs_floor = 1.0e-12;
static const PetscReal rho_floor = 1.0e-14;
static const PetscReal small_num = 1.0e-12;
static const PetscInt  s_width   = 5;

static const PetscReal r1_6    = 1./6.;
static const PetscReal r13_3   = 13./3.;
static const PetscReal r7_6    = 7./6.;
static const PetscReal r11_120 = 11./120.;
static const PetscReal r1_12   = 1./12.;
static const PetscReal r41_60  = 41./60.;

typedef struct { PetscReal comp[nVar]; } Field;

enum bndry_type { wall, inlet, periodic, reflective, transmissive };

PetscInt Malloc1D(PetscReal **, PetscInt);
PetscInt Free1D(PetscReal **);
PetscInt Malloc2D(PetscReal ***, PetscInt, PetscInt);
PetscInt Free2D(PetscReal ***, PetscInt);

typedef struct { PetscInt size; PetscInt nelem; PetscReal *data; } array1d;
typedef struct { PetscInt size1, size2; PetscInt nelem; PetscReal *data; } array2d;
typedef struct { PetscInt size1, size2, size3; PetscInt c1, c2, c3; PetscInt nelem; PetscReal *data; } array3d;
typedef struct { PetscInt size1, size2, size3, size4; PetscInt c1, c2, c3, c4; PetscInt nelem; PetscReal *data; } array4d;
typedef struct { PetscInt size1, size2, size3, size4, size5; PetscInt c1, c2, c3, c4, c5; PetscInt nelem; PetscReal *data; } array5d;
typedef struct { PetscInt size1, size2, size3, size4, size5, size6; PetscInt c1, c2, c3, c4, c5, c6; PetscInt nelem; PetscReal *data; } array6d;
typedef struct { PetscInt size1, size2, size3, size4, size5, size6, size7; PetscInt c1, c2, c3, c4, c5, c6, c7; PetscInt nelem; PetscReal *data; } array7d;

array1d *allocate1d(PetscInt);  array1d *copy_array1d(array1d *);  PetscInt free1d(array1d *);
void set_element_1d(array1d *, PetscInt, PetscReal);  PetscReal get_element_1d(array1d *, PetscInt);
void min_max_1d(array1d *, PetscReal *, PetscReal *);
array2d *allocate2d(PetscInt, PetscInt);  array2d *copy_array2d(array2d *);  PetscInt free2d(array2d *);
void set_element_2d(array2d *, PetscInt, PetscInt, PetscReal);  PetscReal get_element_2d(array2d *, PetscInt, PetscInt);
void min_max_2d(array2d *, PetscReal *, PetscReal *);
array3d *allocate3d(PetscInt, PetscInt, PetscInt);  array3d *copy_array3d(array3d *);  PetscInt free3d(array3d *);
void set_element_3d(array3d *, PetscInt, PetscInt, PetscInt, PetscReal);
PetscReal get_element_3d(array3d *, PetscInt, PetscInt, PetscInt);
void min_max_3d(array3d *, PetscReal *, PetscReal *);
array4d *allocate4d(PetscInt, PetscInt, PetscInt, PetscInt);  array4d *copy_array4d(array4d *);  PetscInt free4d(array4d *);
void set_element_4d(array4d *, PetscInt, PetscInt, PetscInt, PetscInt, PetscReal);
PetscReal get_element_4d(array4d *, PetscInt, PetscInt, PetscInt, PetscInt);
void min_max_4d(array4d *, PetscReal *, PetscReal *);
array5d *allocate5d(PetscInt, PetscInt, PetscInt, PetscInt, PetscInt);  array5d *copy_array5d(array5d *);  PetscInt free5d(array5d *);
void set_element_5d(array5d *, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscReal);
PetscReal get_element_5d(array5d *, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt);
void min_max_5d(array5d *, PetscReal *, PetscReal *);
array6d *allocate6d(PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt);  array6d *copy_array6d(array6d *);  PetscInt free6d(array6d *);
void set_element_6d(array6d *, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscReal);
PetscReal get_element_6d(array6d *, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt);
void min_max_6d(array6d *, PetscReal *, PetscReal *);
array7d *allocate7d(PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt);  array7d *copy_array7d(array7d *);  PetscInt free7d(array7d *);
void set_element_7d(array7d *, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscReal);
PetscReal get_element_7d(array7d *, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt);
void min_max_7d(array7d *, PetscReal *, PetscReal *);

typedef struct {
    PetscReal x_min, y_min, x_max, y_max;
    PetscInt N_x, N_y;
    PetscReal CFL, dt, h;
    PetscBool Restart;
    PetscInt InitialStep;
    PetscReal InitialTime, FinalTime;
    PetscInt WriteInterval, RestartInterval;
    PetscBool ReconsPrimitive;
    enum bndry_type LeftBoundary, RightBoundary, TopBoundary, BottomBoundary;
    PetscInt N, nDOF, Ngp_Face;
    PetscReal *xGP_Face, *wGP_Face;
    PetscInt Ngp_Vol;
    PetscReal *xGP_Vol, *yGP_Vol, *wGP_Vol;
    PetscInt N_node;
    PetscReal *x_node, *y_node;
    Vec W, localU;
    array5d *u_bnd;
    array6d *u_bnd_grad;
    array3d *F, *G, *D, *E;
    array3d *phiFace;
    array2d *phiNode, *phiVol, *gradphiVol_x, *gradphiVol_y;
    array3d *gradphiFace_x, *gradphiFace_y;
} AppCtx;

void PDECons2Prim(const PetscReal *, PetscReal *);
void PDEPrim2Cons(const PetscReal *, PetscReal *);
PetscReal PDEFlux(const PetscReal *, const PetscReal, const PetscReal, const PetscReal, const PetscReal, PetscReal *);
PetscReal PDEViscFlux(const PetscReal *, const PetscReal grad_Q[nVar][DIM], PetscReal, PetscReal, PetscReal *);
void PDENCP(const PetscReal *, const PetscReal *, const PetscReal *, PetscReal *);
void PDEmatrixB(const PetscReal *, PetscReal, PetscReal, PetscReal B[nVar][nVar]);
PetscBool PDECheckPAD(const PetscReal *);
void InletBC(PetscReal, PetscReal, PetscReal, PetscReal *);
PetscReal RiemannSolver(const PetscReal *, const PetscReal *, const PetscReal, const PetscReal, const PetscReal, const PetscReal, PetscReal *, PetscReal *);
PetscReal ViscRiemannSolver(const PetscReal *, PetscReal grad_QL[nVar][DIM], const PetscReal *, PetscReal grad_QR[nVar][DIM], const PetscReal, const PetscReal, PetscReal *);
PetscReal PDEFluxPrim(const PetscReal *, const PetscReal, const PetscReal, const PetscReal, const PetscReal, PetscReal *);
PetscReal PDEViscFluxPrim(const PetscReal *, const PetscReal grad_V[nVar][DIM], PetscReal, PetscReal, PetscReal *);
void PDENCPPrim(const PetscReal *, const PetscReal *, const PetscReal *, PetscReal *);
PetscBool PDECheckPADPrim(const PetscReal *);
PetscReal RiemannSolverPrim(const PetscReal *, const PetscReal *, const PetscReal, const PetscReal, const PetscReal, const PetscReal, PetscReal *, PetscReal *);
PetscReal ViscRiemannSolverPrim(const PetscReal *, PetscReal grad_QL[nVar][DIM], const PetscReal *, PetscReal grad_QR[nVar][DIM], const PetscReal, const PetscReal, PetscReal *);
void InletBCPrim(PetscReal, PetscReal, PetscReal, PetscReal *);

PetscReal basis(PetscReal, PetscReal, PetscInt);
void basis_grad(PetscReal, PetscReal, PetscInt, PetscReal *, PetscReal *);
PetscReal minmod(PetscReal, PetscReal);
void Reconstruct(const PetscReal *, const PetscReal *, const PetscReal *, const PetscInt, PetscReal *, PetscReal *);

void InitialCondition(PetscReal, PetscReal, PetscReal *);
PetscErrorCode InitializeSolution(Vec, DM, AppCtx);
PetscErrorCode RHSFunction(TS, PetscReal, Vec, Vec, void *);
PetscErrorCode RHSFunctionPrim(TS, PetscReal, Vec, Vec, void *);
PetscErrorCode MonitorFunction(TS, PetscInt, PetscReal, Vec, void *);
PetscErrorCode ErrorNorms(Vec, DM, AppCtx, PetscReal *, PetscReal *);
PetscErrorCode ComputePrimitiveVariables(Vec, Vec, DM);

void LidDrivenCavity(PetscReal, PetscReal, PetscReal *);
void ViscousShockTube(PetscReal, PetscReal, PetscReal *);
void SmoothVortex(PetscReal, PetscReal, PetscReal *);
void InterfaceAdvection(PetscReal, PetscReal, PetscReal *);
void AirHelium(PetscReal, PetscReal, PetscReal *);
void AirR22(PetscReal, PetscReal, PetscReal *);
void RichtmyerMeshkov(PetscReal, PetscReal, PetscReal *);
void WaterCylinder(PetscReal, PetscReal, PetscReal *);
void UnderWaterExplosion(PetscReal, PetscReal, PetscReal *);
void AirCavity(PetscReal, PetscReal, PetscReal *);
void BubbleCollapse(PetscReal, PetscReal, PetscReal *);
void AirJet(PetscReal, PetscReal, PetscReal *);
void WaterJet(PetscReal, PetscReal, PetscReal *);

#endif /* HYPE_H_ */
