// hype_stage_tile.cuh -- the tile function of the fused FP64 stage kernel,
// shared by the primitive-variable kernels (hype_stage.cu: grid and persistent
// forms) and the conservative-variable kernels (hype_stage_cons.cu).
//
// One launch of a stage kernel evaluates HyPE-2D's right-hand side L(S)
// (RHSFunctionPrim, rhs_function_prim.c:12-626, or RHSFunction,
// rhs_function.c:12-625) on the stage input S and writes one SSP-RK stage
// combination of it, folding the CFL wave-speed maximum
// (rhs_function_prim.c:617-623) into a device scalar.
//
// Tiling.  A tile is a strip of up to CELLS-2 columns and a run of rows of one
// grid, processed by a block of 2*CELLS threads, two per column.  The block
// marches up its rows; at row r the thread pair m reconstructs the cell in
// column x0-1+m (the strip plus one ring column each side), so only two of
// CELLS reconstructions per row are repeated by the neighbouring strip.  Rows
// of the conserved state arrive by one TMA 3-D box load per row (all fields,
// columns x0-4 .. x0+CELLS+1) into a ring of STAGE_SLOTS shared-memory rows,
// are patched at domain edges with the boundary-condition copies, and are
// converted to primitive variables in place (primitive path).  Reconstruction
// coefficients go to shared memory, the x-face Riemann problem at the left of
// each column is solved by that column's pair from its own and its left
// neighbour's coefficients, the y-face problem below each cell by the cell's
// pair from its coefficients and the top-face values it kept from the row
// below.  Row r-1 is completed (y-flux difference, volume non-conservative
// term, RK combination) while row r is processed.
//
// Compiled with --fmad=false: arithmetic rounds exactly as the reference's C does.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include "hype_internal.h"
#include "hype_physics_fast.cuh"
#include "hype_tma.cuh"

namespace hype {

template <int SYS, int N, int CELLS_>
struct StageKernel {
    using S = System<SYS>;
    using QD = Quad<N>;
    static constexpr int NV = S::NV;
    static constexpr int CELLS = CELLS_;         // reconstruction columns per tile
    static constexpr int NT = 2 * CELLS;         // two threads per cell
    static constexpr int BW = stage_box_width(CELLS, NV);   // TMA box width
    static constexpr int SLOTS = STAGE_SLOTS;
    static constexpr int NDOF = QD::NDOF;
    static constexpr int NC = NDOF - 1;                    // stored coefficients (k >= 1)
    static constexpr int ROW_ELEMS = BW * NV;
    static constexpr int ROW_BYTES = ROW_ELEMS * 8;
    static constexpr int SLOT_STRIDE = ((ROW_BYTES + 127) / 128) * 128 / 8;   // doubles
    // per-cell arrays, [k][c][cell] so consecutive cells hit consecutive banks
    static constexpr int COEF_ELEMS = (NC > 2 ? NC : 2) * NV * CELLS;         // also the x-flux exchange (2 NV)
    static constexpr int YT_ELEMS = 2 * NV * CELLS;                            // top-face values, by Gauss point
    static constexpr int CARRY_ELEMS = 4 * NV * CELLS;                         // ncp, t1, G below, E below
    // the ring, the per-cell arrays and one more row slot: the conserved input of the row
    // being finished (row r-1), for the RK combination
    static constexpr size_t SMEM = 128 /* barriers */ + (size_t)(SLOTS + 1) * SLOT_STRIDE * 8 +
                                   (size_t)(COEF_ELEMS + YT_ELEMS + CARRY_ELEMS) * 8 + 64;
    // blocks the 228 KB of an SM's shared memory holds (1 KB reserved per block); the
    // launch bound asks for no more than that, so no register limit is paid for blocks
    // that could not be resident anyway (Kapila N = 3 at 128-column tiles: 1)
    static constexpr int SMEM_FIT = (int)(233472 / (SMEM + 1024));
    static constexpr int REG_TARGET = (NV <= 6 ? 2 : 1) * (128 / CELLS);
    static constexpr int MIN_BLOCKS = SMEM_FIT < 1 ? 1 : (SMEM_FIT < REG_TARGET ? SMEM_FIT : REG_TARGET);
    static constexpr size_t smem_bytes() { return SMEM; }
};

// Value of one variable's polynomial cf[0..NDOF) at Gauss point q (0/1, run
// time) of face F.  Where both Gauss points share a basis value it is folded
// at compile time (zero terms dropped, exact as in poly_eval); otherwise the
// product with the selected value is formed exactly as the reference does.
template <int N, int F>
__device__ __forceinline__ double face_val(const double *cf, int q)
{
    using QD = Quad<N>;
    double v = 0.0;
    static_for<QD::NDOF>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        constexpr double p0 = QD::phi_face(F, 0, k);
        constexpr double p1 = QD::phi_face(F, QD::NFGP > 1 ? 1 : 0, k);
        if constexpr (p0 == p1) {
            if constexpr (p0 != 0.0) {
                if constexpr (p0 == 1.0) v = v + cf[k];
                else v = v + cf[k] * p0;
            }
        } else {
            const double p = q ? p1 : p0;
            v = v + cf[k] * p;
        }
    });
    return v;
}

// Gradient component D (0: x, 1: y) of one variable at Gauss point q of face
// F from its unlimited coefficients uc: sum_k uc[k] gradphiFace_D(F, q, k) from
// 0.0 in ascending k (rhs_function_prim.c:362-369), before the 1/h factor.
// Zero basis gradients are dropped as in face_val.
template <int N, int F, int D>
__device__ __forceinline__ double face_grad(const double *uc, int q)
{
    using QD = Quad<N>;
    double v = 0.0;
    static_for<QD::NDOF>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        constexpr double p0 = QD::dphi_face(F, 0, D, k);
        constexpr double p1 = QD::dphi_face(F, QD::NFGP > 1 ? 1 : 0, D, k);
        if constexpr (p0 == p1) {
            if constexpr (p0 != 0.0) {
                if constexpr (p0 == 1.0) v = v + uc[k];
                else v = v + uc[k] * p0;
            }
        } else {
            const double p = q ? p1 : p0;
            v = v + uc[k] * p;
        }
    });
    return v;
}

// one face Gauss point with n = e_x (DIR 0) or e_y (DIR 1): riemann.c:112-140
// (RiemannSolverPrim, VL/VR primitive) or, for the conservative path,
// riemann.c:52-105 (RiemannSolver, VL/VR conserved); S is the system's physics
// (System<SYS>, or FastSystem<SYS> for the FP64 performance form)
template <class S, int DIR, bool CONS>
__device__ __forceinline__ double riemann_gp(const Eos &eos, const double *VL, const double *VR, double *F, double *D, bool &bad)
{
    constexpr int NV = S::NV;
    constexpr double nx = DIR == 0 ? 1.0 : 0.0, ny = DIR == 0 ? 0.0 : 1.0;
    if constexpr (CONS) {
        double FL[NV], FR[NV];
        const double sl = S::template flux_cons<DIR>(eos, VL, FL, bad);
        const double sr = S::template flux_cons<DIR>(eos, VR, FR, bad);
        const double s = (sl < sr) ? sr : sl;
        double Qav[NV], gx[NV], gy[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            Qav[c] = 0.5 * (VR[c] + VL[c]);
            gx[c] = nx * (VR[c] - VL[c]);
            gy[c] = ny * (VR[c] - VL[c]);
            F[c] = 0.5 * (FR[c] + FL[c] - s * (VR[c] - VL[c]));
        }
        S::ncp_cons(eos, Qav, gx, gy, D);
        return s;
    }
    double QL[NV], QR[NV], FL[NV], FR[NV];
    S::prim2cons(eos, VL, QL);
    S::prim2cons(eos, VR, QR);
    const double sl = S::template flux<DIR>(eos, VL, FL, bad);
    const double sr = S::template flux<DIR>(eos, VR, FR, bad);
    const double s = (sl < sr) ? sr : sl;
    double Vav[NV], gx[NV], gy[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        Vav[c] = 0.5 * (VR[c] + VL[c]);
        gx[c] = nx * (VR[c] - VL[c]);
        gy[c] = ny * (VR[c] - VL[c]);
        F[c] = 0.5 * (FR[c] + FL[c] - s * (QR[c] - QL[c]));
    }
    S::ncp(eos, Vav, gx, gy, D);
    return s;
}

// One tile of one grid: columns of strip `strip` (of p.strips) and rows of run
// `run` (of p.runs).  Called by every thread of a block of K::NT threads.
// CONS: the conservative-variable RHS (RHSFunction, rhs_function.c:12-625):
// no conversion of the staged rows, PDECheckPAD / PDEFlux / PDENCP on
// conserved values, and a PAD fallback that keeps only the cell mean.
// VISC: the reference's VISCOUS build (Kapila, N >= 1): walls also negate the
// tangential velocity, every face Gauss point adds the mean of the two sides'
// viscous fluxes (riemann.c:146-186) with gradients taken from the unlimited
// coefficients (rhs_function_prim.c:356-374), and the viscous eigenvalue
// maximum goes to DevScalars.smax_v for the dt (rhs_function_prim.c:617).
// FAST: the FP64 performance form (primitive path only): FastSystem / ReconFast
// of hype_physics_fast.cuh, in a translation unit built with FMA contraction;
// reads the derived constants of p.eos (Eos::derive, filled by the host).
template <int SYS, int N, int CELLS_, bool CONS, bool VISC = false, bool FAST = false>
__device__ __forceinline__ void stage_tile(const StageParams &p, const CUtensorMap *tmap, int strip, int run,
                                           unsigned char *smem_raw, double *red_s)
{
    static_assert(!(FAST && (CONS || VISC)), "the FP64 performance form covers the primitive inviscid path");
    using K = StageKernel<SYS, N, CELLS_>;
    using S = std::conditional_t<FAST, FastSystem<SYS>, typename K::S>;
    using QD = typename K::QD;
    constexpr int NV = K::NV, CELLS = K::CELLS, BW = K::BW, SLOTS = K::SLOTS, NDOF = K::NDOF;
    constexpr int NFGP = QD::NFGP, NVGP = QD::NVGP, NNODE = QD::NNODE;
    constexpr int NVH = (NV + 1) / 2;          // variables per half in the reconstruction
    constexpr unsigned FULL = 0xffffffffu;

    if (p.sc->idle) return;   // finished or held run (set by begin_step; 0 outside a time loop)

    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
    double *rows_s = reinterpret_cast<double *>(smem_raw + 128);
    double *coef_s = rows_s + (size_t)SLOTS * K::SLOT_STRIDE;   // [k-1][c][cell]; later [F|D][c][cell]
    double *yt_s = coef_s + K::COEF_ELEMS;                      // [q][c][cell]
    double *carry_s = yt_s + K::YT_ELEMS;                       // [ncp|t1|gb|eb][c][cell]
    // VISC: gradients of the variables the viscous flux reads (primitive u, v;
    // conserved a1r1, a2r2, ru, rv) at the top face, kept for the row above:
    // [q][g][d][cell], right behind the carries
    constexpr int NG = CONS ? 4 : 2, G0 = CONS ? 0 : 2;
    // conserved input of row r-1 (the row the RK combination finishes), [c][BW], its own mbarrier
    double *orow_s = carry_s + K::CARRY_ELEMS;
    double *ygt_s = orow_s + K::SLOT_STRIDE;

    const int t = threadIdx.x;
    const int m = t >> 1;            // cell of this thread's pair
    const int h = t & 1;             // which half of the pair
    // strips split the columns evenly on even boundaries (TMA x origin alignment);
    // row runs split the rows evenly
    const int x0 = 2 * (int)(((long long)strip * p.nx) / (2LL * p.strips));
    const int x1 = (strip + 1 == p.strips) ? p.nx : 2 * (int)(((long long)(strip + 1) * p.nx) / (2LL * p.strips));
    const int owc = x1 - x0;
    const int y0 = (int)(((long long)run * p.ny) / p.runs);
    const int H = (int)(((long long)(run + 1) * p.ny) / p.runs) - y0;
    if (owc > CELLS - 2 || owc < 1 || H < 1) {   // launch geometry outside what the tiling covers
        if (threadIdx.x == 0) raise_error(p.sc, ERR_BAD_LAUNCH, 0u);
        return;
    }
    const int xs = x0 - 4;                    // TMA box origin (even: x0 is even)
    const int i = x0 - 1 + m;                 // this pair's reconstruction column
    const bool active = m <= owc + 1;
    const bool owned = m >= 1 && m <= owc;
    const bool xface = m >= 1 && m <= owc + 1;
    const bool touches_x = (x0 == 0) || (x0 + owc >= p.nx);
    const int bcL = p.bc[0], bcR = p.bc[1], bcB = p.bc[2], bcT = p.bc[3];
    const bool py = (bcB == BC_PERIODIC || bcT == BC_PERIODIC);
    const double dt = (p.mode == OUT_RHS) ? 0.0 : p.sc->dt;
    const double b = dt / p.kb;   // the RK combination's dt/kb, the same for every row
    const Eos eos = p.eos;
    const double r1_h = p.r1_h;

    __syncthreads();   // the previous tile of this block is done with every buffer
    if (t == 0) {
        for (int s = 0; s <= SLOTS; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    const int row_lo = y0 - 3, row_hi = y0 + H + 2;   // rows of state this block reads
    int next_issue = row_lo, next_conv = row_lo;
    auto slot_of = [&](int row) { return (row - row_lo) % SLOTS; };
    auto row_ptr = [&](int row) { return rows_s + (size_t)slot_of(row) * K::SLOT_STRIDE; };   // [c][BW]
    auto cidx = [&](int k1, int c, int cell) { return (k1 * NV + c) * CELLS + cell; };         // coef_s index, k1 = k-1
    auto carry = [&](int which, int c) -> double & { return carry_s[(which * NV + c) * CELLS + m]; };

    double smax_loc = 0.0, smaxv_loc = 0.0;
    bool bad = false;
    unsigned bad_cell = 0xffffffffu;
    // A bounded wait ran out (ERR_TMA_TIMEOUT): thread 0 waits for the loads still in
    // flight -- ring rows issued but not yet converted, and the finish-row slot while
    // its load is outstanding -- then invalidates the barriers; the block returns.
    auto give_up = [&](bool orow_pending, unsigned orow_parity) {
        if (t != 0) return;
        raise_error(p.sc, ERR_TMA_TIMEOUT, 0u);
        const unsigned long long deadline = global_ns() + TMA_WAIT_NS;
        bool drained = true;
        for (int row = next_conv; row < next_issue; ++row)
            drained = drained && mbar_wait_until(&bars[slot_of(row)], (unsigned)(((row - row_lo) / SLOTS) & 1), deadline);
        if (orow_pending) drained = drained && mbar_wait_until(&bars[SLOTS], orow_parity, deadline);
        if (drained)
            for (int k = 0; k <= SLOTS; ++k) mbar_inval(&bars[k]);
    };

    for (int r = y0 - 1; r <= y0 + H; ++r) {
        // this iteration finishes an owned row (r-1) with an RK combination that reads its input
        const bool finish_row = r > y0 && p.mode != OUT_RHS;
        // ---------------- A. bring rows up to r+2 into the ring --------------
        if (t == 0) {
            fence_proxy_async();   // earlier generic accesses to the slots precede the TMA writes
            for (; next_issue <= min(r + 3, row_hi) && (!p.skip_loads || next_issue < p.skip_loads_from); ++next_issue) {
                const int row = next_issue;
                const int src = map_axis(row, p.ny, bcB, bcT);
                uint64_t *bar = &bars[slot_of(row)];
                mbar_expect_tx(bar, K::ROW_BYTES);
                tma_load_3d(row_ptr(row), tmap, xs + p.col_off, src + p.row_off, 0, bar);   // the map starts col_off columns left of column 0, row_off rows below row 0
            }
            if (finish_row && (!p.skip_loads || r - 1 < p.skip_loads_from)) {   // row r-1's conserved input for the RK combination in section C
                mbar_expect_tx(&bars[SLOTS], K::ROW_BYTES);
                tma_load_3d(orow_s, tmap, xs + p.col_off, (r - 1) + p.row_off, 0, &bars[SLOTS]);
            }
        }
        for (; next_conv <= r + 2; ++next_conv) {
            const int row = next_conv;
            const unsigned parity = (unsigned)(((row - row_lo) / SLOTS) & 1);
            const bool ok = mbar_wait_bounded(&bars[slot_of(row)], parity);
            if (__syncthreads_or(!ok)) {
                give_up(finish_row && (!p.skip_loads || r - 1 < p.skip_loads_from), (unsigned)((r - y0 - 1) & 1));
                return;   // block-uniform exit; the caller's next barrier is block-uniform too
            }
            double *rp = row_ptr(row);
            const int src = map_axis(row, p.ny, bcB, bcT);
            const bool yg = row < 0 || row >= p.ny;
            const bool yrefl = yg && ((row < 0 ? bcB : bcT) == BC_REFLECTIVE);
            // column cc = 1 + t; columns 1 .. owc+6 are the ones the stencils read
            const int cc = 1 + t;
            const bool conv = cc <= owc + 6;
            const int g = xs + cc;
            const bool isg = conv && (g < 0 || g >= p.nx);
            double Q[NV];
            if (touches_x) {
                // Phase 1: ghost columns fetch their conserved source values before anyone converts
                if (isg) {
                    const int gm = map_axis(g, p.nx, bcL, bcR);
                    if (gm - xs >= 0 && gm - xs < BW) {
#pragma unroll
                        for (int c = 0; c < NV; ++c) Q[c] = rp[c * BW + (gm - xs)];
                    } else {
#pragma unroll
                        for (int c = 0; c < NV; ++c) Q[c] = p.in[(long long)c * p.plane + (long long)src * p.pitch + gm];
                    }
                }
                __syncthreads();
            }
            // Phase 2: convert in place, apply reflections / inlet values
            if (conv) {
                if (!isg) {
#pragma unroll
                    for (int c = 0; c < NV; ++c) Q[c] = rp[c * BW + cc];
                }
                double V[NV];
                if constexpr (CONS) {
#pragma unroll
                    for (int c = 0; c < NV; ++c) V[c] = Q[c];
                } else if constexpr (!FAST && ((SYS == SYS_BN && (N == 1 || N == 2)) || (SYS == SYS_KAPILA && N <= 1))) {
                    // branch-free correctly rounded divisions (hype_div.cuh): the cell's
                    // independent divisions overlap instead of each waiting on the last
                    // one's slow-path branch; the compiler's division where an operand is
                    // outside their range.  Only in the tiles where it measured faster
                    // (Kapila N = 2, 3 lose to the extra registers)
                    bool special = false;
                    S::cons2prim_dv(eos, Q, V, [&special](double a, double b) { return cr_div(a, b, special); });
                    if (special) S::cons2prim(eos, Q, V);
                } else {
                    S::cons2prim(eos, Q, V);
                }
                if (isg) {
                    const int side_bc = g < 0 ? bcL : bcR;
                    if (side_bc == BC_INLET && p.inlet) {
                        const int jr = py ? row : map_axis(row, p.ny, bcB, bcT);
#pragma unroll
                        for (int c = 0; c < NV; ++c) V[c] = p.inlet[((size_t)(g + 3) * (p.ny + 6) + (jr + 3)) * NV + c];
                    } else if (side_bc == BC_REFLECTIVE) {
                        if (S::RX0 >= 0) V[S::RX0] = -V[S::RX0];
                        if (S::RX1 >= 0) V[S::RX1] = -V[S::RX1];
                        if constexpr (VISC) V[S::RXV] = -V[S::RXV];
                    }
                }
                if (yrefl) {
                    if (S::RY0 >= 0) V[S::RY0] = -V[S::RY0];
                    if (S::RY1 >= 0) V[S::RY1] = -V[S::RY1];
                    if constexpr (VISC) V[S::RYV] = -V[S::RYV];
                }
#pragma unroll
                for (int c = 0; c < NV; ++c) rp[c * BW + cc] = V[c];
            }
        }
        if (finish_row) {   // the copy of row r-1 issued at the start of this iteration
            const unsigned parity = (unsigned)((r - y0 - 1) & 1);
            const bool ok = mbar_wait_bounded(&bars[SLOTS], parity);
            if (__syncthreads_or(!ok)) {
                give_up(false, 0u);   // the finish-row load is the one that did not come
                return;   // block-uniform exit
            }
        }
        __syncthreads();   // S1: prim rows r-2 .. r+2 ready

        // ---------------- B. reconstruction of cell (r, i), split by variable ---
        const int ccm = m + 3;                                    // column of i in the ring rows
        const double *w_m2 = row_ptr(r - 2), *w_m1 = row_ptr(r - 1), *w_0 = row_ptr(r), *w_p1 = row_ptr(r + 1), *w_p2 = row_ptr(r + 2);
        if (active) {
#pragma unroll 1
            for (int kv = 0; kv < NVH; ++kv) {
                const int c = h * NVH + kv;
                if (c >= NV) break;
                Stencil st;
                const double *a0 = w_0 + c * BW + ccm;
                st.c = a0[0];
                st.xm2 = a0[-2]; st.xm1 = a0[-1]; st.xp1 = a0[1]; st.xp2 = a0[2];
                st.ym2 = w_m2[c * BW + ccm]; st.ym1 = w_m1[c * BW + ccm]; st.yp1 = w_p1[c * BW + ccm]; st.yp2 = w_p2[c * BW + ccm];
                st.pp = w_p1[c * BW + ccm + 1]; st.pm = w_m1[c * BW + ccm + 1]; st.mp = w_p1[c * BW + ccm - 1]; st.mm = w_m1[c * BW + ccm - 1];
                double cf[NDOF];
                if constexpr (FAST) {
                    ReconFast<N>::run(st, cf);
                } else if constexpr (SYS == SYS_BN && N == 2) {
                    // branch-free correctly rounded divisions let the weights' chains overlap
                    // (the Baer-Nunziato tile runs 8 warps per SM); the compiler's division
                    // where an operand is outside their range
                    bool special = false;
                    Recon2Cr::run(st, cf, special);
                    if (special) Recon<N>::run(st, cf);
                } else {
                    Recon<N>::run(st, cf);
                }
#pragma unroll
                for (int k = 1; k < NDOF; ++k) coef_s[cidx(k - 1, c, m)] = cf[k];
            }
        }
        __syncwarp();
        // own coefficients of one variable of cell `cell`, k = 0 from the ring row
        auto load_cf = [&](int c, int cell, double *cf) {
            cf[0] = w_0[c * BW + cell + 3];
#pragma unroll
            for (int k = 1; k < NDOF; ++k) cf[k] = coef_s[cidx(k - 1, c, cell)];
        };
        // VISC: unlimited coefficients of variable c of the cell `cell` of row r, from the ring rows
        auto load_uc = [&](int c, int cell, double *uc) {
            if constexpr (VISC) {
                const int col = cell + 3;
                Stencil st;
                const double *a0 = w_0 + c * BW + col;
                st.c = a0[0];
                st.xm2 = a0[-2]; st.xm1 = a0[-1]; st.xp1 = a0[1]; st.xp2 = a0[2];
                st.ym2 = w_m2[c * BW + col]; st.ym1 = w_m1[c * BW + col]; st.yp1 = w_p1[c * BW + col]; st.yp2 = w_p2[c * BW + col];
                st.pp = w_p1[c * BW + col + 1]; st.pm = w_m1[c * BW + col + 1]; st.mp = w_p1[c * BW + col - 1]; st.mm = w_m1[c * BW + col - 1];
                UCoef<N>::run(st, uc);
            }
        };
        // admissibility at the nodes (rhs_function_prim.c:382-404), nodes split between the pair
        bool ok = true;
        if (active) {
            static_for<NNODE / 2>([&](auto sq) {
                constexpr int s0 = decltype(sq)::value, s1 = NNODE / 2 + s0;
                if (!ok) return;
                double V[NV];
#pragma unroll
                for (int c = 0; c < NV; ++c) {
                    double cf[NDOF];
                    load_cf(c, m, cf);
                    double v = 0.0;
                    static_for<NDOF>([&](auto kk) {
                        constexpr int k = decltype(kk)::value;
                        constexpr double p0 = QD::phi_node(s0, k), p1 = QD::phi_node(s1, k);
                        if constexpr (p0 == p1) {
                            if constexpr (p0 != 0.0) { if constexpr (p0 == 1.0) v = v + cf[k]; else v = v + cf[k] * p0; }
                        } else {
                            v = v + cf[k] * (h ? p1 : p0);
                        }
                    });
                    V[c] = v;
                }
                if constexpr (CONS) ok = S::pad_cons(eos, V);
                else ok = S::pad(eos, V);
            });
        }
        {
            // every lane takes part in the shuffle (no short-circuit around it)
            const int ok_pair = __shfl_xor_sync(FULL, (int)ok, 1);
            ok = ok && (ok_pair != 0);
        }
        if (CONS && !ok && N >= 1 && active) {   // rhs_function.c:410-420: the slopes are zeroed from k = 1 on
#pragma unroll 1
            for (int kv = 0; kv < NVH; ++kv) {
                const int c = h * NVH + kv;
                if (c >= NV) break;
#pragma unroll
                for (int k = 1; k < NDOF; ++k) coef_s[cidx(k - 1, c, m)] = 0.0;
            }
        }
        if (!CONS && !ok && N >= 2 && active) {   // rhs_function_prim.c:407-421: [w, minmod_x, minmod_y, 0 ...]
#pragma unroll 1
            for (int kv = 0; kv < NVH; ++kv) {
                const int c = h * NVH + kv;
                if (c >= NV) break;
                const double w0 = w_0[c * BW + ccm];
                coef_s[cidx(0, c, m)] = minmod(w_0[c * BW + ccm + 1] - w0, w0 - w_0[c * BW + ccm - 1]);
                coef_s[cidx(1, c, m)] = minmod(w_p1[c * BW + ccm] - w0, w0 - w_m1[c * BW + ccm]);
#pragma unroll
                for (int k = 3; k < NDOF; ++k) coef_s[cidx(k - 1, c, m)] = 0.0;
            }
        }
        __syncwarp();

        // ---------------- C. y-face below (r, i): Gauss point q = h ----------------
        const bool in_rows = r >= y0 && r <= y0 + H;
        const int q = NFGP > 1 ? h : 0;
        {
            double G[NV], E[NV];
            const bool doit = owned && in_rows;
            double Fq[NV], Dq[NV], Vq[NV];
            if (doit) {
                double VL[NV], VR[NV];
#pragma unroll
                for (int c = 0; c < NV; ++c) {
                    double cf[NDOF];
                    load_cf(c, m, cf);
                    VR[c] = face_val<N, 2>(cf, q);
                    VL[c] = yt_s[(q * NV + c) * CELLS + m];
                }
                const double s = riemann_gp<S, 1, CONS>(eos, VL, VR, Fq, Dq, bad);
                smax_loc = fmax(smax_loc, s);
#pragma unroll
                for (int c = 0; c < NV; ++c) { Fq[c] = QD::wf(0) * Fq[c]; Dq[c] = QD::wf(0) * Dq[c]; }
                if constexpr (VISC) {
                    double gL[NV][2], gR[NV][2];
#pragma unroll
                    for (int g = 0; g < NG; ++g) {
                        const int c = G0 + g;
                        double uc[NDOF];
                        load_uc(c, m, uc);
                        gR[c][0] = r1_h * face_grad<N, 2, 0>(uc, q);
                        gR[c][1] = r1_h * face_grad<N, 2, 1>(uc, q);
                        gL[c][0] = ygt_s[((q * NG + g) * 2 + 0) * CELLS + m];
                        gL[c][1] = ygt_s[((q * NG + g) * 2 + 1) * CELLS + m];
                    }
                    double FvL[NV], FvR[NV];
                    double svl, svr;
                    if constexpr (CONS) {
                        svl = S::template visc_cons<1>(VL, gL, p.mu1, p.mu2, FvL);
                        svr = S::template visc_cons<1>(VR, gR, p.mu1, p.mu2, FvR);
                    } else {
                        svl = S::template visc_prim<1>(VL, gL, p.mu1, p.mu2, FvL);
                        svr = S::template visc_prim<1>(VR, gR, p.mu1, p.mu2, FvR);
                    }
                    smaxv_loc = fmax(smaxv_loc, (svl < svr) ? svr : svl);
#pragma unroll
                    for (int c = 0; c < NV; ++c) Vq[c] = QD::wf(0) * (0.5 * (FvR[c] + FvL[c]));
                }
            } else {
#pragma unroll
                for (int c = 0; c < NV; ++c) { Fq[c] = 0.0; Dq[c] = 0.0; Vq[c] = 0.0; }
            }
            // Flux = 0.0; Flux += w F(q0); Flux += w F(q1)   (rhs_function_prim.c:548-577),
            // VISC: Flux += w Fv(q) after each Gauss point's convective part
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                if constexpr (NFGP > 1) {
                    const double fo = __shfl_xor_sync(FULL, Fq[c], 1), d_o = __shfl_xor_sync(FULL, Dq[c], 1);
                    const double f0 = h ? fo : Fq[c], f1 = h ? Fq[c] : fo;
                    const double d0 = h ? d_o : Dq[c], d1 = h ? Dq[c] : d_o;
                    if constexpr (VISC) {
                        const double vo = __shfl_xor_sync(FULL, Vq[c], 1);
                        const double v0 = h ? vo : Vq[c], v1 = h ? Vq[c] : vo;
                        G[c] = (((0.0 + f0) + v0) + f1) + v1;
                    } else {
                        G[c] = (0.0 + f0) + f1;
                    }
                    E[c] = (0.0 + d0) + d1;
                } else {
                    if constexpr (VISC) G[c] = (0.0 + Fq[c]) + Vq[c];
                    else G[c] = 0.0 + Fq[c];
                    E[c] = 0.0 + Dq[c];
                }
            }
            if (doit && bad && bad_cell == 0xffffffffu) bad_cell = (unsigned)(r * p.nx + i);
            if (doit) {
                if (r > y0) {
                    // row r-1: rhs = ncp + ((-1/h) X - (1/h) Y)  (rhs_function_prim.c:589-602), then the RK combination
                    const int jo = r - 1;
                    const size_t gidx = (size_t)jo * p.pitch + i;
                    // the halves take alternate variables, c = 2 j + h, so every lane works in every pass
#pragma unroll
                    for (int j = 0; j < (NV + 1) / 2; ++j) {
                        if (2 * j + 1 >= NV && h) continue;   // odd NV: the last variable is half 0's alone
                        const int c = 2 * j + h;
                        const double Gc = h ? G[2 * j + 1 < NV ? 2 * j + 1 : 2 * j] : G[2 * j];
                        const double Ec = h ? E[2 * j + 1 < NV ? 2 * j + 1 : 2 * j] : E[2 * j];
                        const double Y = Gc - carry(2, c) + 0.5 * (Ec + carry(3, c));
                        const double ty = r1_h * Y;
                        const double rhs = carry(0, c) + (carry(1, c) - ty);
                        if (p.mode == OUT_RHS) {
                            if (p.out_aos) p.out[((size_t)jo * p.nx + i) * NV + c] = rhs;
                            else p.out[(size_t)c * p.plane + gidx] = rhs;
                            continue;
                        }
                        const double Sv = orow_s[c * BW + ccm];   // = p.in[c * plane + gidx], staged by TMA
                        const double bF = b * rhs;
                        double o;
                        if (p.mode == OUT_AXPY) {
                            o = Sv + bF;
                        } else if (p.mode == OUT_ZXS) {
                            const double Xv = p.xn[(size_t)c * p.plane + gidx];
                            const double s0 = p.ka * Xv + bF;
                            o = s0 + p.kc * Sv;
                        } else if (p.mode == OUT_ZSX) {
                            const double Xv = p.xn[(size_t)c * p.plane + gidx];
                            const double s0 = p.ka * Sv + bF;
                            o = s0 + p.kc * Xv;
                        } else {   // OUT_RK104_5
                            const double Xv = p.xn[(size_t)c * p.plane + gidx];
                            const double w = Sv + bF;
                            const double w1 = (1. / 25) * Xv + (9. / 25) * w;
                            p.out2[(size_t)c * p.plane + gidx] = w1;
                            o = 15.0 * w1 + (-5.0) * w;
                        }
                        p.out[(size_t)c * p.plane + gidx] = o;
                        // a y-slab's edge rows are the neighbours' halo rows: store them there too
                        if (p.push_lo && jo < 3)
                            p.push_lo[(long long)c * p.push_plane_lo + (long long)(jo + p.push_shift_lo) * p.pitch + i] = o;
                        if (p.push_hi && jo >= p.ny - 3)
                            p.push_hi[(long long)c * p.push_plane_hi + (long long)(jo + p.push_shift_hi) * p.pitch + i] = o;
                    }
                }
#pragma unroll
                for (int j = 0; j < (NV + 1) / 2; ++j) {
                    if (2 * j + 1 >= NV && h) continue;
                    const int c = 2 * j + h;
                    carry(2, c) = h ? G[2 * j + 1 < NV ? 2 * j + 1 : 2 * j] : G[2 * j];
                    carry(3, c) = h ? E[2 * j + 1 < NV ? 2 * j + 1 : 2 * j] : E[2 * j];
                }
            }
        }

        // ---------------- D. keep the top-face values (Gauss point q) for row r+1 --
        if (owned && r >= y0 - 1 && r < y0 + H && (NFGP > 1 || h == 0)) {
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                double cf[NDOF];
                load_cf(c, m, cf);
                yt_s[(q * NV + c) * CELLS + m] = face_val<N, 3>(cf, q);
            }
            if constexpr (VISC) {
#pragma unroll
                for (int g = 0; g < NG; ++g) {
                    double uc[NDOF];
                    load_uc(G0 + g, m, uc);
                    ygt_s[((q * NG + g) * 2 + 0) * CELLS + m] = r1_h * face_grad<N, 3, 0>(uc, q);
                    ygt_s[((q * NG + g) * 2 + 1) * CELLS + m] = r1_h * face_grad<N, 3, 1>(uc, q);
                }
            }
        }

        // ---------------- E. volume non-conservative term (rhs_function_prim.c:459-479)
        const bool full_row = r >= y0 && r < y0 + H;
        {
            // rhs = 0.0; rhs += -w_q B_q for q = 0..NVGP-1; the pair holds q = 2h, 2h+1
            constexpr int QH = NVGP > 1 ? NVGP / 2 : 1;
            double tq[QH][NV];
#pragma unroll
            for (int a = 0; a < QH; ++a)
#pragma unroll
                for (int c = 0; c < NV; ++c) tq[a][c] = 0.0;
            const bool doit = owned && full_row && (NVGP > 1 || h == 0);
            if (doit) {
                static_for<QH>([&](auto sa) {
                    constexpr int a = decltype(sa)::value;
                    constexpr int q0 = a, q1 = (NVGP > 1 ? QH : 0) + a;   // half 0 -> q0, half 1 -> q1
                    double V[NV], gx[NV], gy[NV], B[NV];
#pragma unroll
                    for (int c = 0; c < NV; ++c) {
                        double cf[NDOF];
                        load_cf(c, m, cf);
                        double v = 0.0, dx = 0.0, dy = 0.0;
                        static_for<NDOF>([&](auto kk) {
                            constexpr int k = decltype(kk)::value;
                            constexpr double pv0 = QD::phi_vol(q0, k), pv1 = QD::phi_vol(q1, k);
                            constexpr double px0 = QD::dphi_vol_x(q0, k), px1 = QD::dphi_vol_x(q1, k);
                            constexpr double py0 = QD::dphi_vol_y(q0, k), py1 = QD::dphi_vol_y(q1, k);
                            if constexpr (pv0 == pv1) { if constexpr (pv0 != 0.0) { if constexpr (pv0 == 1.0) v = v + cf[k]; else v = v + cf[k] * pv0; } }
                            else v = v + cf[k] * (h ? pv1 : pv0);
                            if constexpr (px0 == px1) { if constexpr (px0 != 0.0) { if constexpr (px0 == 1.0) dx = dx + cf[k]; else dx = dx + cf[k] * px0; } }
                            else dx = dx + cf[k] * (h ? px1 : px0);
                            if constexpr (py0 == py1) { if constexpr (py0 != 0.0) { if constexpr (py0 == 1.0) dy = dy + cf[k]; else dy = dy + cf[k] * py0; } }
                            else dy = dy + cf[k] * (h ? py1 : py0);
                        });
                        V[c] = v; gx[c] = r1_h * dx; gy[c] = r1_h * dy;
                    }
                    if constexpr (CONS) S::ncp_cons(eos, V, gx, gy, B);
                    else S::ncp(eos, V, gx, gy, B);
#pragma unroll
                    for (int c = 0; c < NV; ++c) tq[a][c] = -QD::wv(0) * B[c];
                });
            }
            static_for<NV>([&](auto cc_) {
                constexpr int c = decltype(cc_)::value;
                if constexpr (!(CONS ? S::ncp_cons_nonzero(c) : S::ncp_nonzero(c))) {
                    // B[c] is the constant 0.0 for every Gauss point: ((0 + -0) + -0) ... = +0
                    if (owned && full_row && (c & 1) == h) carry(0, c) = 0.0;
                } else if constexpr (NVGP > 1) {
                    double parts[NVGP];
#pragma unroll
                    for (int a = 0; a < QH; ++a) {
                        const double o = __shfl_xor_sync(FULL, tq[a][c], 1);
                        parts[a] = h ? o : tq[a][c];
                        parts[QH + a] = h ? tq[a][c] : o;
                    }
                    double acc = 0.0;
#pragma unroll
                    for (int a = 0; a < NVGP; ++a) acc += parts[a];
                    if (owned && full_row && (c & 1) == h) carry(0, c) = acc;
                } else {
                    const double o = __shfl_xor_sync(FULL, tq[0][c], 1);
                    const double acc = 0.0 + (h ? o : tq[0][c]);
                    if (owned && full_row && (c & 1) == h) carry(0, c) = acc;
                }
            });
        }
        __syncthreads();   // S2: every column's coefficients of row r visible

        // ---------------- F. x-face at the left of column i: Gauss point q ----------
        double Fx[NV], Dx[NV];
        {
            const bool doit = xface && full_row;
            double Fq[NV], Dq[NV], Vq[NV];
            if (doit) {
                double VL[NV], VR[NV];
#pragma unroll
                for (int c = 0; c < NV; ++c) {
                    double cl[NDOF], cr[NDOF];
                    load_cf(c, m - 1, cl);
                    load_cf(c, m, cr);
                    VL[c] = face_val<N, 1>(cl, q);
                    VR[c] = face_val<N, 0>(cr, q);
                }
                const double s = riemann_gp<S, 0, CONS>(eos, VL, VR, Fq, Dq, bad);
                smax_loc = fmax(smax_loc, s);
#pragma unroll
                for (int c = 0; c < NV; ++c) { Fq[c] = QD::wf(0) * Fq[c]; Dq[c] = QD::wf(0) * Dq[c]; }
                if constexpr (VISC) {
                    double gL[NV][2], gR[NV][2];
#pragma unroll
                    for (int g = 0; g < NG; ++g) {
                        const int c = G0 + g;
                        double ul[NDOF], ur[NDOF];
                        load_uc(c, m - 1, ul);
                        load_uc(c, m, ur);
                        gL[c][0] = r1_h * face_grad<N, 1, 0>(ul, q);
                        gL[c][1] = r1_h * face_grad<N, 1, 1>(ul, q);
                        gR[c][0] = r1_h * face_grad<N, 0, 0>(ur, q);
                        gR[c][1] = r1_h * face_grad<N, 0, 1>(ur, q);
                    }
                    double FvL[NV], FvR[NV];
                    double svl, svr;
                    if constexpr (CONS) {
                        svl = S::template visc_cons<0>(VL, gL, p.mu1, p.mu2, FvL);
                        svr = S::template visc_cons<0>(VR, gR, p.mu1, p.mu2, FvR);
                    } else {
                        svl = S::template visc_prim<0>(VL, gL, p.mu1, p.mu2, FvL);
                        svr = S::template visc_prim<0>(VR, gR, p.mu1, p.mu2, FvR);
                    }
                    smaxv_loc = fmax(smaxv_loc, (svl < svr) ? svr : svl);
#pragma unroll
                    for (int c = 0; c < NV; ++c) Vq[c] = QD::wf(0) * (0.5 * (FvR[c] + FvL[c]));
                }
                if (bad && bad_cell == 0xffffffffu) bad_cell = (unsigned)(r * p.nx + i);
            } else {
#pragma unroll
                for (int c = 0; c < NV; ++c) { Fq[c] = 0.0; Dq[c] = 0.0; Vq[c] = 0.0; }
            }
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                if constexpr (NFGP > 1) {
                    const double fo = __shfl_xor_sync(FULL, Fq[c], 1), d_o = __shfl_xor_sync(FULL, Dq[c], 1);
                    const double f0 = h ? fo : Fq[c], f1 = h ? Fq[c] : fo;
                    const double d0 = h ? d_o : Dq[c], d1 = h ? Dq[c] : d_o;
                    if constexpr (VISC) {
                        const double vo = __shfl_xor_sync(FULL, Vq[c], 1);
                        const double v0 = h ? vo : Vq[c], v1 = h ? Vq[c] : vo;
                        Fx[c] = (((0.0 + f0) + v0) + f1) + v1;
                    } else {
                        Fx[c] = (0.0 + f0) + f1;
                    }
                    Dx[c] = (0.0 + d0) + d1;
                } else {
                    if constexpr (VISC) Fx[c] = (0.0 + Fq[c]) + Vq[c];
                    else Fx[c] = 0.0 + Fq[c];
                    Dx[c] = 0.0 + Dq[c];
                }
            }
        }
        __syncthreads();   // S3: coefficient reads done; the buffer now carries face fluxes
        if (xface && full_row) {
#pragma unroll
            for (int j = 0; j < (NV + 1) / 2; ++j) {
                if (2 * j + 1 >= NV && h) continue;
                const int c = 2 * j + h;
                coef_s[c * CELLS + m] = h ? Fx[2 * j + 1 < NV ? 2 * j + 1 : 2 * j] : Fx[2 * j];
                coef_s[(NV + c) * CELLS + m] = h ? Dx[2 * j + 1 < NV ? 2 * j + 1 : 2 * j] : Dx[2 * j];
            }
        }
        __syncthreads();   // S4
        if (owned && full_row) {
#pragma unroll
            for (int j = 0; j < (NV + 1) / 2; ++j) {
                if (2 * j + 1 >= NV && h) continue;
                const int c = 2 * j + h;
                const double Fc = h ? Fx[2 * j + 1 < NV ? 2 * j + 1 : 2 * j] : Fx[2 * j];
                const double Dc = h ? Dx[2 * j + 1 < NV ? 2 * j + 1 : 2 * j] : Dx[2 * j];
                const double F1 = coef_s[c * CELLS + m + 1], D1 = coef_s[(NV + c) * CELLS + m + 1];
                const double X = F1 - Fc + 0.5 * (D1 + Dc);
                carry(1, c) = -r1_h * X;
            }
        }
    }

    // ---------------- CFL maximum: warp shuffle, block, one atomic ------------
    if (bad) raise_error(p.sc, ERR_INADMISSIBLE_FACE, bad_cell);
    __syncthreads();   // red_s is reused tile after tile
    if (p.reduce_smax) {
        double mx = smax_loc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
        if ((t & 31) == 0) red_s[t >> 5] = mx;
        __syncthreads();
        if (t == 0) {
            double b = red_s[0];
#pragma unroll
            for (int w = 1; w < K::NT / 32; ++w) b = fmax(b, red_s[w]);
            if (b > 0.0) atomicMax(&p.sc->smax, (unsigned long long)__double_as_longlong(b));
        }
        if constexpr (VISC) {   // the same for the viscous eigenvalue
            __syncthreads();
            double mv = smaxv_loc;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mv = fmax(mv, __shfl_xor_sync(FULL, mv, o));
            if ((t & 31) == 0) red_s[t >> 5] = mv;
            __syncthreads();
            if (t == 0) {
                double b = red_s[0];
#pragma unroll
                for (int w = 1; w < K::NT / 32; ++w) b = fmax(b, red_s[w]);
                if (b > 0.0) atomicMax(&p.sc->smax_v, (unsigned long long)__double_as_longlong(b));
            }
        }
    }
    for (int k = t; k <= SLOTS; k += K::NT) mbar_inval(&bars[k]);
}

}  // namespace hype
