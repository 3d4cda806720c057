// hype_solver.h -- the solver object behind the opaque handle of
// include/hype_gpu.h, shared by hype_api.cu (one grid) and hype_group.cu (a grid
// split into y-slabs, one solver per slab).  Internal to the library.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include "../../include/hype_gpu.h"
#include "hype_internal.h"

struct hype_solver {
    hype_config cfg;
    int nv = 0;
    int pitch = 0;
    long long plane = 0;
    double h = 0.0, r1_h = 0.0, cfl_h = 0.0;
    double *dU = nullptr, *dS0 = nullptr, *dS1 = nullptr, *dS2 = nullptr;
    double *dAosIn = nullptr, *dAosOut = nullptr, *dInlet = nullptr;
    double *dRed = nullptr;           // reduction scratch
    hype::DevScalars *dSc = nullptr;
    hype::DevScalars *hSc = nullptr;        // pinned mirror
    CUtensorMap tmU, tmS0, tmS1;
    cudaStream_t stream = nullptr;
    // banded host calls (row bands of the grid, at most MAX_BANDS)
    static constexpr int MAX_BANDS = 16;
    cudaStream_t cin = nullptr, cout = nullptr;     // host<->device copies, back to back
    cudaStream_t cvin = nullptr, cvout = nullptr;   // the layout conversions beside those copies
    cudaEvent_t ev_cp[MAX_BANDS] = {};              // per row band: host rows copied in
    cudaEvent_t ev_in[MAX_BANDS] = {};              //               converted to planes
    cudaEvent_t ev_dc[MAX_BANDS] = {};              //               result converted for the copy out
    cudaEvent_t ev_done[MAX_BANDS] = {};            //               computed
    cudaEvent_t ev_dl[MAX_BANDS] = {};              //               copied into the host staging
    // pinned host staging of the banded calls for pageable caller arrays (allocated on
    // first use, aos_bytes each)
    double *hStageIn = nullptr, *hStageOut = nullptr;
    size_t aos_bytes = 0;
    cudaEvent_t ev_fence = nullptr;                 // the compute stream's work so far
    // banded steps: stage s on compute stream s % 4 (stream, stream2, stream3, stream4),
    // band k of stage s marked by ev_sb[s * MAX_BANDS + k]
    cudaStream_t stream2 = nullptr, stream3 = nullptr, stream4 = nullptr;
    cudaEvent_t ev_sb[hype::MAX_PLAN * MAX_BANDS] = {};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t step_exec = nullptr;
    int cells = hype::STAGE_CELLS;          // tile width of the stage kernel
    int waves = 1;                    // row runs per strip = waves x (SM slots / strips)
    int sms = 0;
    int strips = 1, runs = 1;         // tile decomposition of the grid
    int bps = 0;                      // stage blocks per SM
    // mixed precision (Kapila N=2): state k = 0 (U), 1 (S0), 2 (S1) as FP32 + FP64 planes
    bool mixed = false;
    bool fast = false;                // FP64 performance form (HYPE_PREC_FP64_FAST)
    float *mf[3] = {nullptr, nullptr, nullptr};
    double *md[3] = {nullptr, nullptr, nullptr};
    hype::MixedMaps mm[3];
    // y-slab of a decomposed grid (hype_group): row_off halo rows below and above the
    // slab in every plane; nb_*[role] = the neighbouring slabs' planes of the same buffer
    // role, with their plane sizes and the row shift from this slab's rows to theirs
    int row_off = 0;
    int row0 = 0;                     // first global row of the slab
    // block of a grid split in x as well (hype_create_block): col_off halo columns left
    // and right of the block's columns in every plane, col0 its first global column
    int col_off = 0;
    int col0 = 0;
    double *nb_lo[4] = {}, *nb_hi[4] = {};
    float *nbf_lo[3] = {}, *nbf_hi[3] = {};      // the same for a mixed state: FP32 and FP64 planes
    double *nbd_lo[3] = {}, *nbd_hi[3] = {};
    long long nb_plane_lo = 0, nb_plane_hi = 0;
    int nb_shift_lo = 0, nb_shift_hi = 0;
    bool began = false;
    int test_skip_row = -1;           // hype_test_skip_row_loads: first row whose loads are not issued (-1: off)
    double last_ms = 0.0;
    char err[512] = {0};
};

namespace hype {
// hype_api.cu internals the slab group drives
int solver_fail(hype_solver *s, int code, const char *fmt, ...);
// a slab solver: rows row0 .. row0+rows-1 of the grid of `global`, with halo rows on
// the sides flagged halo_lo / halo_hi (a neighbouring slab there)
int create_slab(const hype_config *global, int row0, int rows, bool halo_lo, bool halo_hi, hype_solver **out);
// a block solver: columns col0 .. col0+cols-1 and rows row0 .. row0+rows-1 of the grid
// of `global`; halo[4] flags the sides (left, right, bottom, top) with a neighbour
int create_block(const hype_config *global, int col0, int cols, int row0, int rows, const bool halo[4], hype_solver **out);
double *solver_buf(hype_solver *s, int role);                  // B_U .. B_S2
double *solver_alloc_base(const hype_solver *s, double *buf);  // start of a padded buffer
// one stage of the plan; a state output also goes to the neighbours' halo rows
cudaError_t solver_stage(hype_solver *s, const PlanStage &q);
cudaError_t solver_seed_rhs(hype_solver *s);                    // RHS of u (reduces s_max), output discarded
int solver_reset_scalars(hype_solver *s);
int solver_read_scalars(hype_solver *s);
}  // namespace hype
