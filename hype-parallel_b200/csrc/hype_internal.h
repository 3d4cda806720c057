// hype_internal.h -- host/device interface between the C ABI (hype_api.cu) and
// the kernels (hype_stage.cu, hype_aux.cu).  Not installed; not part of the ABI.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>
#include "hype_physics.cuh"
#include "../../include/hype_gpu.h"

namespace hype {

// What a stage kernel writes for each owned cell, with F = L(S) the right-hand
// side of the stage input S and X a second state (u^n):
//   OUT_RHS      out = F
//   OUT_AXPY     out = S + ((dt/kb) * F)                          PETSc VecAXPY(S, dt/kb, F)
//   OUT_ZXS      out = ((ka*X) + ((dt/kb)*F)) + (kc*S)             VecAXPBYPCZ(S, ka, dt/kb, kc, X, F)
//   OUT_ZSX      out = ((ka*S) + ((dt/kb)*F)) + (kc*X)             VecAXPBYPCZ(X, ka, dt/kb, kc, S, F)
//   OUT_RK104_5  w  = S + ((dt/6)*F); out2 = (1/25)X + (9/25)w;     fifth stage of SSPRK(10,4) and the
//                out = 15*out2 + (-5)*w                             two vector updates that follow it
enum : int { OUT_RHS = 0, OUT_AXPY = 1, OUT_ZXS = 2, OUT_ZSX = 3, OUT_RK104_5 = 4 };

// Device-resident scalars of one solve (one per instance).
struct DevScalars {
    double dt;                 // time step of the step in progress
    double t;                  // time at the start of the step in progress
    double t_final;
    double time_step;          // dt proposed by the last RHS (MonitorFunction / Ctx->dt)
    unsigned long long smax;   // bit pattern of max wave speed of the RHS being reduced
    unsigned long long smax_v; // bit pattern of max viscous eigenvalue (viscous solvers)
    double r1h_v;              // 1/h for viscous solvers, 0 otherwise: dt = CFL h / (2 (smax + (r1h_v smax_v) 2))
    unsigned int err;          // ERR_* bits
    unsigned int err_cell;     // linear index of the first cell that raised an error
    int steps, max_steps;
    int done;                  // set when the run reached t_final or max_steps
    int hold;                  // host request: skip this instance's steps for now (batch scheduling)
    int idle;                  // set by begin_step for a step this instance does not take (done or held)
    int pad_;
    double cfl_h;              // CFL*h of the instance (read by the batched step control)
};

struct StageParams {
    int nx, ny, pitch;          // row stride of a field plane, in elements (even)
    long long plane;            // elements per field plane
    int bc[4];                  // left, right, bottom, top (BC_*)
    Eos eos;
    double r1_h;                // 1/h
    double cfl_h;               // CFL*h
    const double *in;           // stage input planes (also behind the tensor map)
    const double *xn;           // second state X (u^n) for OUT_ZXS/OUT_ZSX/OUT_RK104_5
    double *out;                // output planes (or AoS when out_aos)
    double *out2;               // OUT_RK104_5 second output
    int out_aos;                // 1: write `out` interleaved (cell-major, NV per cell)
    int mode;
    double ka, kb, kc;
    DevScalars *sc;             // dt source, smax/err target, early-exit flag
    int reduce_smax;            // 1: fold this stage's max wave speed into sc->smax
    const double *inlet;        // [3][ny+6][NV] primitive ghost values for a left inlet (or null)
    int strips, runs;           // tile decomposition: column strips x row runs
    int run0, run_count;        // grid form: the launch covers runs run0 .. run0+run_count-1 (0: all runs)
    double mu1, mu2;            // viscous solvers: MU_1, MU_2 (hype.h:46-47)
    // y-slab of a decomposed grid: the planes carry row_off halo rows below row 0 and above
    // row ny-1 (the tensor map starts at row -row_off); rows 0..2 and ny-3..ny-1 of a state
    // output are also stored into the neighbouring slabs' halo rows, at row + push_shift
    // of planes push_lo / push_hi (null: no neighbour on that side)
    int row_off;
    int push_shift_lo, push_shift_hi;
    long long push_plane_lo, push_plane_hi;
    double *push_lo, *push_hi;
    // block of a grid split in x as well (a DMDA rank's block): the planes carry col_off
    // halo columns left of column 0 (and right of nx-1); the tensor map starts there
    int col_off;
    // test hook (hype_test_skip_row_loads): with skip_loads set, no row load is issued for
    // rows >= skip_loads_from, so the bounded wait on it runs out; 0 in normal operation
    int skip_loads, skip_loads_from;
};

// Tile geometry of the stage kernel: a tile is CELLS reconstruction columns
// (CELLS - 2 owned) of one strip, processed by 2*CELLS threads; CELLS is 64 or
// 128 (chosen per grid by the autotuner, 128 by default).
constexpr int STAGE_CELLS = 128;
constexpr int STAGE_SLOTS = 6;              // prim row ring
// TMA box of the FP64 stage tile: columns x0-4 .. x0+cells+1 (cells + 6), widened by
// pairs of columns until nvh * width = 8 (mod 16) doubles, nvh = (nv + 1) / 2: the two
// threads of a pair read stencil rows nvh planes apart, which then fall on disjoint halves
// of the shared-memory banks (e.g. Kapila: 136 instead of 134 for 128-cell tiles)
constexpr int stage_box_width(int cells, int nv)
{
    const int nvh = (nv + 1) / 2;
    for (int w = cells + 6; w < cells + 6 + 32; w += 2)
        if ((nvh * w) % 16 == 8) return w;
    return cells + 6;
}

size_t stage_smem_bytes(int sys, int order, int cells);
int stage_threads(int cells);
cudaError_t stage_configure(int sys, int order, int cells);   // raises the dynamic smem limit
int stage_blocks_per_sm(int sys, int order, int cells);
int stage_batch_blocks_per_sm(int sys, int order, int cells);   // resident blocks of the persistent form
cudaError_t launch_stage(int sys, int order, int cells, const CUtensorMap &tmap, const StageParams &p, cudaStream_t s);
cudaError_t launch_stage_batch(int sys, int order, int cells, const StageParams *inst, const CUtensorMap *tmaps,
                               const int2 *work, int *sched, int blocks, cudaStream_t s);
// the FP64 performance form (primitive path, HYPE_PREC_FP64_FAST): grid form, 64- or 128-column tiles
cudaError_t stage_fast_configure(int sys, int order, int cells);
int stage_fast_blocks_per_sm(int sys, int order, int cells);
cudaError_t launch_stage_fast(int sys, int order, int cells, const CUtensorMap &tmap, const StageParams &p, cudaStream_t s);
// the VISCOUS build (Kapila, N = 1..3, primitive or conservative): 128-column tiles, grid form
cudaError_t stage_visc_configure(int order, bool cons);
int stage_visc_blocks_per_sm(int order, bool cons);
cudaError_t launch_stage_visc(int order, bool cons, const CUtensorMap &tmap, const StageParams &p, cudaStream_t s);
// conservative-variable path (RHSFunction): 128-column tiles, grid form
cudaError_t stage_cons_configure(int sys, int order);
int stage_cons_blocks_per_sm(int sys, int order);
cudaError_t launch_stage_cons(int sys, int order, const CUtensorMap &tmap, const StageParams &p, cudaStream_t s);
// persistent (batched) form of the conservative path and of the viscous build: 128-column tiles
enum : int { BATCH_PATH_CONS = 0, BATCH_PATH_VISC = 1, BATCH_PATH_VISC_CONS = 2 };
cudaError_t path_batch_configure(int path, int sys, int order);
int path_batch_blocks_per_sm(int path, int sys, int order);
cudaError_t launch_path_batch(int path, int sys, int order, const StageParams *inst, const CUtensorMap *tmaps, const int2 *work,
                              int *sched, int blocks, cudaStream_t s);
// Strips of a grid: with S = ceil(nx/(cells-4)) strips and even origins
// 2*floor(s*nx/(2S)), every strip has at most 2*ceil(nx/(2S)) <= cells-4
// columns and the last one at most nx/S + 2 <= cells-2.
inline int stage_strips(int nx, int cells) { return (nx + (cells - 4) - 1) / (cells - 4); }

// One stage of an SSP-RK step over a solver's state buffers (B_U = u^n, B_S0..B_S2
// work vectors; B_NONE = unused): in -> out with OUT_* `mode` and coefficients
// ka, kb, kc; x = second state, out2 = second output; reduce = fold the max
// wave speed into DevScalars.smax (the stage whose RHS sets the next dt).
enum : int { B_NONE = -1, B_U = 0, B_S0 = 1, B_S1 = 2, B_S2 = 3 };
struct PlanStage {
    int in, out, mode;
    double ka, kb, kc;
    int x, out2, reduce;
};
constexpr int MAX_PLAN = 10;
// Stages of one step of the SSP scheme of `order` (hype.c:362-382; PETSc TSSSP
// forms); *copy_back is set when the step ends with u^n = S0 (forward Euler).
int ssp_plan(int order, PlanStage *plan, int *copy_back);

// hype_aux.cu
cudaError_t launch_aos_to_planes(const double *aos, double *planes, int nx, int ny, int nv, int pitch, long long plane, cudaStream_t s);
cudaError_t launch_planes_to_aos(const double *planes, double *aos, int nx, int ny, int nv, int pitch, long long plane, cudaStream_t s);
// the same for rows row0 .. row0+nrows-1 only (both arrays are full-grid arrays)
cudaError_t launch_aos_to_planes_rows(const double *aos, double *planes, int nx, int row0, int nrows, int nv, int pitch, long long plane,
                                      cudaStream_t s);
cudaError_t launch_planes_to_aos_rows(const double *planes, double *aos, int nx, int row0, int nrows, int nv, int pitch, long long plane,
                                      cudaStream_t s);
cudaError_t launch_begin_step(DevScalars *sc, cudaStream_t s);
cudaError_t launch_end_step(DevScalars *sc, double cfl_h, cudaStream_t s);
cudaError_t launch_seed_dt(DevScalars *sc, double cfl_h, cudaStream_t s);
// Batched step control over a member list: members[0] = count, members[1..] =
// instance indices into sc[]; each instance uses its own sc[k].cfl_h and takes
// its hold flag from hold[k].
cudaError_t launch_begin_step_batch(DevScalars *sc, const int *members, const int *hold, int max_members, cudaStream_t s);
cudaError_t launch_end_step_batch(DevScalars *sc, const int *members, int max_members, cudaStream_t s);
// u^n = S0 for every member (forward Euler), one pointer pair per instance
cudaError_t launch_copy_batch(double *const *dst, const double *const *src, const long long *n, const int *members,
                              int max_members, const DevScalars *sc, cudaStream_t s);
// writes nv sums then min/max of field acomp (acomp < 0: zeros) to red[0..nv+1];
// red must hold 64 + (512 + 1) * (nv + 2) doubles
cudaError_t launch_totals(const double *planes, double *red, int nx, int ny, int nv, int pitch, long long plane, int acomp,
                          cudaStream_t s);
constexpr size_t TOTALS_SCRATCH = 64 + 513 * 11;

// ---------------------------------------------------------------------------
// Mixed precision (N = 2, primitive path; Kapila, Baer-Nunziato, Euler).  State:
// FP32 planes for densities and momenta, FP64 planes for the energies and the
// volume fraction (MixedLayout), with one element pitch; the FP64 planes carry
// the quantities whose stiffened-gas cancellation (p from E with P_inf ~ 6e8)
// FP32 cannot resolve.
// ---------------------------------------------------------------------------
struct MixedParams {
    int nx, ny, pitch;          // element pitch of every plane (multiple of 32)
    long long plane;            // elements per plane
    int bc[4];
    Eos eos;
    double r1_h, cfl_h;
    const float *in_f; const double *in_d;     // stage input S (behind the two tensor maps)
    const float *xn_f; const double *xn_d;     // second state X (u^n)
    float *out_f; double *out_d;               // output state
    double *out_rhs;                           // OUT_RHS: interleaved FP64 RHS, 6 per cell
    int mode;
    double ka, kb, kc;
    DevScalars *sc;
    int reduce_smax;
    int strips, runs;
    int run0, run_count;        // grid form: the launch covers runs run0 .. run0+run_count-1 (0: all runs)
    // y-slab of a decomposed grid, as StageParams: row_off halo rows below and above in
    // every plane; state rows 0..2 and ny-3..ny-1 also go to the neighbours' halo rows
    int row_off;
    int push_shift_lo, push_shift_hi;
    long long push_plane_lo, push_plane_hi;
    float *push_lo_f, *push_hi_f;
    double *push_lo_d, *push_hi_d;
    int skip_loads, skip_loads_from;   // test hook, as in StageParams
};
struct MixedMaps {
    CUtensorMap f;              // FP32 planes: (nx, ny, nf), box (cells + 8, 1, nf)
    CUtensorMap d;              // FP64 planes: (nx, ny, nd), box (cells + 8, 1, nd)
};
// Which conserved components a mixed state keeps in FP64 (bit c of dmask): the
// FP32 planes hold the other components in ascending order, the FP64 planes these.
//   Kapila:         a1 rho1, a2 rho2, rho u, rho v | E, a1
//   Baer-Nunziato:  a1 rho1, a1 rho1 u1, a1 rho1 v1, a2 rho2, a2 rho2 u2, a2 rho2 v2 | a1 E1, a2 E2, a1
//   Euler:          rho, rho u, rho v | E
struct MixedLayout {
    int nf, nd;
    unsigned dmask;
};
inline MixedLayout mixed_layout(int sys)
{
    if (sys == SYS_BN) return MixedLayout{6, 3, (1u << 3) | (1u << 7) | (1u << 8)};
    if (sys == SYS_EULER) return MixedLayout{3, 1, 1u << 3};
    return MixedLayout{4, 2, (1u << 4) | (1u << 5)};
}
constexpr int MIXED_CELLS = 128;
inline int mixed_box_width(int cells) { return cells + 8; }
// strips with origins 4*floor(s*nx/(4S)) (16-byte aligned FP32 TMA origin):
// S = ceil(nx/(cells-6)) keeps every strip within cells-2 columns
inline int mixed_strips(int nx, int cells) { return (nx + (cells - 6) - 1) / (cells - 6); }
size_t mixed_smem_bytes(int sys, int cells);
int mixed_threads(int cells);
int mixed_blocks_per_sm(int sys, int cells);
int mixed_batch_blocks_per_sm(int sys, int cells);
cudaError_t launch_mixed(int sys, int cells, const MixedMaps &maps, const MixedParams &p, cudaStream_t s);
cudaError_t launch_mixed_batch(int sys, int cells, const MixedParams *inst, const MixedMaps *maps, const int2 *work, int *sched,
                               int blocks, cudaStream_t s);
// the Baer-Nunziato and Euler tiles (hype_stage_mixed_sys.cu), behind the functions above
size_t mixsys_smem_bytes(int sys, int cells);
int mixsys_blocks_per_sm(int sys, int cells, bool batch);
cudaError_t launch_mixsys(int sys, int cells, const MixedMaps &maps, const MixedParams &p, cudaStream_t s);
cudaError_t launch_mixsys_batch(int sys, int cells, const MixedParams *inst, const MixedMaps *maps, const int2 *work, int *sched,
                                int blocks, cudaStream_t s);
// layout changes between the interleaved FP64 Vec and the mixed planes of system sys
// hype_hostcopy.cu: host copies split over a small thread pool (between a caller's
// pageable arrays and pinned staging), and whether a host pointer is pageable
void host_copy(void *dst, const void *src, size_t bytes);
void host_copy_2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t rows);
bool host_is_pageable(const void *p);

cudaError_t launch_aos_to_mixed(int sys, const double *aos, float *pf, double *pd, int nx, int ny, int pitch, long long plane,
                                cudaStream_t s);
cudaError_t launch_mixed_to_aos(int sys, const float *pf, const double *pd, double *aos, int nx, int ny, int pitch, long long plane,
                                cudaStream_t s);

// hype_io.cu: PDECons2Prim of every cell, planes -> interleaved primitive variables
cudaError_t launch_cons2prim(int sys, const Eos &eos, const double *planes, double *prim_aos, int nx, int ny, int pitch,
                             long long plane, cudaStream_t s);

// hype_api.cu, shared with the batch (hype_batch.cu)
CUresult encode_planes_map(CUtensorMap *m, const void *base, bool fp32, int nx, int ny, int nplanes, int pitch, long long plane,
                           int box_w);
int validate_config(const hype_config *c, char *err, size_t errlen);
void inlet_table(const hype_config &c, double h, std::vector<double> &tab);
void inlet_to_conserved(const hype_config &c, std::vector<double> &tab);

}  // namespace hype
