// hype_stage_mixed.cu -- the mixed-precision stage kernel for the Kapila
// five-equation model at N = 2: same tiling, TMA row staging and face
// bookkeeping as the FP64 kernel (hype_stage.cu), with
//   FP32: state a1 rho1, a2 rho2, rho u, rho v; primitives rho1, rho2, u, v;
//         WENO reconstruction; mass/momentum fluxes; wave speeds; the
//         non-conservative alpha terms;
//   FP64: state E and a1; the pressure recovery from the stiffened-gas EOS
//         (kapila_5eqn.c:14-35, where P_inf*gamma ~ 2.6e9 cancels against
//         rho e); face pressure and volume fraction; the energy flux and its
//         dissipation; the cell totals (RHS assembly and RK combination); dt.
// Reconstruction works on deviations from the cell value and normalises the
// WENO weights by their smallest denominator, which gives the weights of
// reconstruction.c:163-170 exactly in real arithmetic and stays inside FP32
// range for any data.  Not bit-compatible with the reference by design; its
// error against the FP64 path is measured in tests/test_gpu_mixed.py.
#include <cuda.h>
#include <cuda_runtime.h>
#include "hype_internal.h"
#include "hype_tma.cuh"
#include "hype_mixed_common.cuh"

namespace hype {

template <int CELLS_>
struct MixedKernel {
    using QD = Quad<2>;
    static constexpr int NV = 6;
    static constexpr int CELLS = CELLS_;
    static constexpr int NT = 2 * CELLS;
    static constexpr int BW = CELLS + 8;               // multiple of 4 floats (16 B)
    static constexpr int SLOTS = STAGE_SLOTS;
    static constexpr int F_ROW_BYTES = 4 * BW * 4;      // FP32 planes of one row
    static constexpr int D_ROW_BYTES = 2 * BW * 8;      // FP64 planes of one row
    static constexpr int F_REGION = (F_ROW_BYTES + 127) / 128 * 128;
    static constexpr int D_REGION = (D_ROW_BYTES + 127) / 128 * 128;
    static constexpr int SLOT_BYTES = F_REGION + D_REGION;
    // reconstruction coefficients: k = 1..4 as one float4 per (cell, variable), cells 7
    // float4 apart (quarter-warp float4 loads fall on disjoint banks), then k = 5 as
    // [c][cell]; later 7 FP64 flux values per cell
    static constexpr int CV_STRIDE = 7;
    static constexpr int COEF_FLOATS = 4 * CV_STRIDE * CELLS + NV * CELLS;
    static constexpr int YTF_FLOATS = 2 * 4 * CELLS;     // top-face rho1 rho2 u v, by Gauss point
    static constexpr int YTD_DOUBLES = 2 * 2 * CELLS;    // top-face p, a1
    static constexpr int CARRY_DOUBLES = 14 * CELLS;     // t1[6], G below[6], E5 below, ncp5
    static constexpr int MIN_BLOCKS = 3 * (128 / CELLS);
    static constexpr size_t smem_bytes()
    {
        // the ring plus one more slot: the stage input of the row being finished (row r-1)
        return 128 + (size_t)(SLOTS + 1) * SLOT_BYTES + (size_t)COEF_FLOATS * 4 + (size_t)YTF_FLOATS * 4 +
               (size_t)YTD_DOUBLES * 8 + (size_t)CARRY_DOUBLES * 8 + 64;
    }
};

// Kapila EOS constants in the forms the mixed kernel uses
struct MixedEos {
    double g1, g2, pi1, pi2, G1m1, G2m1, c1, c2, inv_G12;
    float g1f, g2f;
    __device__ __forceinline__ explicit MixedEos(const Eos &e)
    {
        g1 = e.g1; g2 = e.g2; pi1 = e.pi1; pi2 = e.pi2;
        G1m1 = g1 - 1.0; G2m1 = g2 - 1.0;
        c1 = g1 * pi1 * G2m1; c2 = g2 * pi2 * G1m1;
        inv_G12 = 1.0 / (G1m1 * G2m1);
        g1f = (float)g1; g2f = (float)g2;
    }
};

// primitive state at a point: FP32 rho1 rho2 u v, FP64 p a1
struct PrimM {
    float r1, r2, u, v;
    double p, a;
};

// sum_{k>=1} c[k-1] phi(k) at face F, Gauss point q (run time 0/1)
template <int F>
__device__ __forceinline__ float face_poly(const float *c, int q)
{
    using QD = Quad<2>;
    float v = 0.0f;
    static_for<5>([&](auto kk) {
        constexpr int k = decltype(kk)::value + 1;
        constexpr float p0 = (float)QD::phi_face(F, 0, k), p1 = (float)QD::phi_face(F, 1, k);
        if constexpr (p0 == p1) {
            if constexpr (p0 != 0.0f) v += c[k - 1] * p0;
        } else {
            v += c[k - 1] * (q ? p1 : p0);
        }
    });
    return v;
}

// Kapila admissibility (kapila_5eqn.c:450-479) on a mixed primitive state
__device__ __forceinline__ bool pad_mixed(const MixedEos &e, const PrimM &V)
{
    const double a2 = 1.0 - V.a;
    const float af = (float)V.a, a2f = (float)a2;
    const float rho = af * V.r1 + a2f * V.r2;
    const float a1sq = fdiv(e.g1f * (float)(V.p + e.pi1), V.r1);
    const float a2sq = fdiv(e.g2f * (float)(V.p + e.pi2), V.r2);
    const float asq = fdiv(V.r1 * a1sq * V.r2 * a2sq, rho * (a2f * V.r1 * a1sq + af * V.r2 * a2sq));
    if (rho < 1.0e-14f) return false;
    if (asq < 1.0e-12f) return false;
    if (V.a < 0.0 || V.a > 1.0) return false;
    return true;
}

// K = a1 a2 (rho2 a2^2 - rho1 a1^2) / (a1 rho2 a2^2 + a2 rho1 a1^2)  (kapila_5eqn.c:432-434)
__device__ __forceinline__ float kapila_K(const MixedEos &e, float r1, float r2, double p, double a)
{
    const float af = (float)a, a2f = (float)(1.0 - a);
    const float r1a1 = e.g1f * (float)(p + e.pi1);   // rho1 a1^2
    const float r2a2 = e.g2f * (float)(p + e.pi2);   // rho2 a2^2
    (void)r1; (void)r2;
    return fdiv(af * a2f * (r2a2 - r1a1), af * r2a2 + a2f * r1a1);
}

// Rusanov flux and fluctuation at one face Gauss point (riemann.c:112-140).
// F[0..3] from FP32 arithmetic, F[4] (energy) and F[5] (alpha) in FP64.
template <int DIR>
__device__ __forceinline__ float riemann_mixed(const MixedEos &e, const PrimM &L, const PrimM &R, double *F, float &D5, bool &bad)
{
    float FL[4], FR[4], QL[4], QR[4];
    double EL, ER, F4L, F4R;
    auto side = [&](const PrimM &V, float *Fs, float *Qs, double &Es, double &F4s) -> float {
        const double a2 = 1.0 - V.a;
        const float af = (float)V.a, a2f = (float)a2;
        const float rho = af * V.r1 + a2f * V.r2;
        const float un = DIR == 0 ? V.u : V.v;
        const double ei = (V.p * (V.a * e.G2m1 + a2 * e.G1m1) + V.a * e.c1 + a2 * e.c2) * e.inv_G12;
        Es = ei + (double)(0.5f * rho * (V.u * V.u + V.v * V.v));
        const float pf = (float)V.p;
        const float a1sq = fdiv(e.g1f * (float)(V.p + e.pi1), V.r1);
        const float a2sq = fdiv(e.g2f * (float)(V.p + e.pi2), V.r2);
        const float asq = fdiv(V.r1 * a1sq * V.r2 * a2sq, rho * (a2f * V.r1 * a1sq + af * V.r2 * a2sq));
        bad |= (asq < 1.0e-12f);
        Fs[0] = af * V.r1 * un;
        Fs[1] = a2f * V.r2 * un;
        Fs[2] = rho * V.u * un + (DIR == 0 ? pf : 0.0f);
        Fs[3] = rho * V.v * un + (DIR == 1 ? pf : 0.0f);
        F4s = (Es + V.p) * (double)un;
        Qs[0] = af * V.r1; Qs[1] = a2f * V.r2; Qs[2] = rho * V.u; Qs[3] = rho * V.v;
        return fabsf(un) + sqrtf(asq);
    };
    const float sl = side(L, FL, QL, EL, F4L);
    const float sr = side(R, FR, QR, ER, F4R);
    const float s = (sl < sr) ? sr : sl;
#pragma unroll
    for (int c = 0; c < 4; ++c) F[c] = (double)(0.5f * (FR[c] + FL[c] - s * (QR[c] - QL[c])));
    F[4] = 0.5 * (F4R + F4L - (double)s * (ER - EL));
    F[5] = -0.5 * (double)s * (R.a - L.a);
    // fluctuation of the alpha equation at the face average (kapila_5eqn.c:417-444)
    const float uav = 0.5f * (R.u + L.u), vav = 0.5f * (R.v + L.v);
    const double pav = 0.5 * (R.p + L.p), aav = 0.5 * (R.a + L.a);
    const float K = kapila_K(e, 0.5f * (R.r1 + L.r1), 0.5f * (R.r2 + L.r2), pav, aav);
    const float da = (float)(R.a - L.a);
    D5 = DIR == 0 ? (uav * da - K * (R.u - L.u)) : (vav * da - K * (R.v - L.v));
    return s;
}

// SLAB: a y-slab of a decomposed grid (row offset, edge rows stored into the
// neighbours' halo rows); the single-grid and batched kernels compile without it.
template <int CELLS_, bool SLAB = false>
__device__ __forceinline__ void mixed_tile(const MixedParams &p, const MixedMaps *maps, int strip, int run,
                                           unsigned char *smem, double *red_s)
{
    using K = MixedKernel<CELLS_>;
    using QD = Quad<2>;
    constexpr int NV = 6, CELLS = K::CELLS, BW = K::BW, SLOTS = K::SLOTS;
    constexpr unsigned FULL = 0xffffffffu;
    if (p.sc->idle) return;   // finished or held run (set by begin_step; 0 outside a time loop)

    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    unsigned char *rows = smem + 128;
    // stage input of row r-1 (the row the RK combination finishes): FP32 then FP64 planes
    unsigned char *orow = rows + (size_t)SLOTS * K::SLOT_BYTES;
    const float *orowf = reinterpret_cast<const float *>(orow);
    const double *orowd = reinterpret_cast<const double *>(orow + K::F_REGION);
    float *coef_f = reinterpret_cast<float *>(rows + (size_t)(SLOTS + 1) * K::SLOT_BYTES);
    double *exch = reinterpret_cast<double *>(coef_f);                  // x-face fluxes after S3: [7][cell]
    float *ytf = coef_f + K::COEF_FLOATS;                                 // [q][4][cell]
    double *ytd = reinterpret_cast<double *>(ytf + K::YTF_FLOATS);        // [q][2][cell]
    double *carry = ytd + K::YTD_DOUBLES;                                 // [14][cell]

    const int t = threadIdx.x, m = t >> 1, h = t & 1;
    const int x0 = 4 * (int)(((long long)strip * p.nx) / (4LL * p.strips));
    const int x1 = (strip + 1 == p.strips) ? p.nx : 4 * (int)(((long long)(strip + 1) * p.nx) / (4LL * p.strips));
    const int owc = x1 - x0;
    const int y0 = (int)(((long long)run * p.ny) / p.runs);
    const int H = (int)(((long long)(run + 1) * p.ny) / p.runs) - y0;
    if (owc > CELLS - 2 || owc < 1 || H < 1) {
        if (t == 0) raise_error(p.sc, ERR_BAD_LAUNCH, 0u);
        return;
    }
    const int xs = x0 - 4;
    const int i = x0 - 1 + m;
    const bool active = m <= owc + 1, owned = m >= 1 && m <= owc, xface = m >= 1 && m <= owc + 1;
    const bool touches_x = (x0 == 0) || (x1 >= p.nx);
    const int bcL = p.bc[0], bcR = p.bc[1], bcB = p.bc[2], bcT = p.bc[3];
    const double dt = (p.mode == OUT_RHS) ? 0.0 : p.sc->dt;
    const double b = dt / p.kb;
    const MixedEos e(p.eos);
    const double r1_h = p.r1_h;

    __syncthreads();
    if (t == 0) {
        for (int k = 0; k <= SLOTS; ++k) mbar_init(&bars[k], 1);
        fence_mbar_init();
    }
    __syncthreads();

    const int row_lo = y0 - 3, row_hi = y0 + H + 2;
    int next_issue = row_lo, next_conv = row_lo;
    auto slot_of = [&](int row) { return (row - row_lo) % SLOTS; };
    auto rowf = [&](int row) { return reinterpret_cast<float *>(rows + (size_t)slot_of(row) * K::SLOT_BYTES); };
    auto rowd = [&](int row) { return reinterpret_cast<double *>(rows + (size_t)slot_of(row) * K::SLOT_BYTES + K::F_REGION); };
    float4 *coef_v = reinterpret_cast<float4 *>(coef_f);                   // [cell][c] k = 1..4
    float *coef_5 = coef_f + 4 * K::CV_STRIDE * CELLS;                      // [c][cell] k = 5
    auto cf_store = [&](int c, int cell, const float *cf) {
        coef_v[cell * K::CV_STRIDE + c] = make_float4(cf[0], cf[1], cf[2], cf[3]);
        coef_5[c * CELLS + cell] = cf[4];
    };
    // the five coefficients of (cell, c) as an accessor for pair_poly (k1 = 0..4)
    auto cf_of = [&](int c, int cell) {
        const float4 v = coef_v[cell * K::CV_STRIDE + c];
        const float *p5 = &coef_5[c * CELLS + cell];
        return [v, p5](int k1) -> float { return k1 == 0 ? v.x : k1 == 1 ? v.y : k1 == 2 ? v.z : k1 == 3 ? v.w : *p5; };
    };

    float smax_loc = 0.0f;
    bool bad = false;
    unsigned bad_cell = 0xffffffffu;
    // a bounded wait ran out: thread 0 waits for the loads in flight, then the block returns
    // (the same as the FP64 tile, hype_stage_tile.cuh)
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
        // ---------------- A. rows up to r+2: two TMA loads (FP32, FP64 planes) per row
        if (t == 0) {
            fence_proxy_async();
            for (; next_issue <= min(r + 3, row_hi) && (!p.skip_loads || next_issue < p.skip_loads_from); ++next_issue) {
                const int row = next_issue;
                const int src = map_axis(row, p.ny, bcB, bcT);
                uint64_t *bar = &bars[slot_of(row)];
                mbar_expect_tx(bar, K::F_ROW_BYTES + K::D_ROW_BYTES);
                const int ty = SLAB ? src + p.row_off : src;   // a slab's maps start row_off rows below row 0
                tma_load_3d(rowf(row), &maps->f, xs, ty, 0, bar);
                tma_load_3d(rowd(row), &maps->d, xs, ty, 0, bar);
            }
            if (finish_row && (!p.skip_loads || r - 1 < p.skip_loads_from)) {   // row r-1's stage input for the RK combination
                const int ty = SLAB ? (r - 1) + p.row_off : r - 1;
                mbar_expect_tx(&bars[SLOTS], K::F_ROW_BYTES + K::D_ROW_BYTES);
                tma_load_3d(orow, &maps->f, xs, ty, 0, &bars[SLOTS]);
                tma_load_3d(orow + K::F_REGION, &maps->d, xs, ty, 0, &bars[SLOTS]);
            }
        }
        for (; next_conv <= r + 2; ++next_conv) {
            const int row = next_conv;
            const unsigned parity = (unsigned)(((row - row_lo) / SLOTS) & 1);
            const bool ok = mbar_wait_bounded(&bars[slot_of(row)], parity);
            if (__syncthreads_or(!ok)) {
                give_up(finish_row && (!p.skip_loads || r - 1 < p.skip_loads_from), (unsigned)((r - y0 - 1) & 1));
                return;
            }
            float *rf = rowf(row);
            double *rd = rowd(row);
            const int src = map_axis(row, p.ny, bcB, bcT);
            const bool yrefl = (row < 0 || row >= p.ny) && ((row < 0 ? bcB : bcT) == BC_REFLECTIVE);
            const int cc = 1 + t;
            const bool conv = cc <= owc + 6;
            const int g = xs + cc;
            const bool isg = conv && (g < 0 || g >= p.nx);
            float q[4];
            double E = 0.0, a1 = 0.0;
            if (touches_x) {
                if (isg) {
                    const int gm = map_axis(g, p.nx, bcL, bcR);
                    if (gm - xs >= 0 && gm - xs < BW) {
#pragma unroll
                        for (int c = 0; c < 4; ++c) q[c] = rf[c * BW + (gm - xs)];
                        E = rd[gm - xs]; a1 = rd[BW + (gm - xs)];
                    } else {
                        const long long gi = (long long)src * p.pitch + gm;
#pragma unroll
                        for (int c = 0; c < 4; ++c) q[c] = p.in_f[(long long)c * p.plane + gi];
                        E = p.in_d[gi]; a1 = p.in_d[p.plane + gi];
                    }
                }
                __syncthreads();
            }
            if (conv) {
                if (!isg) {
#pragma unroll
                    for (int c = 0; c < 4; ++c) q[c] = rf[c * BW + cc];
                    E = rd[cc]; a1 = rd[BW + cc];
                }
                // kapila_5eqn.c:14-35, pressure in FP64
                const double a2 = 1.0 - a1;
                const double rho = (double)q[0] + (double)q[1];
                const double irho = 1.0 / rho;
                double u = (double)q[2] * irho, v = (double)q[3] * irho;
                const double ei = E - 0.5 * rho * (u * u + v * v);
                const double pr = (ei * e.G1m1 * e.G2m1 - a1 * e.c1 - a2 * e.c2) / (a1 * e.G2m1 + a2 * e.G1m1);
                if (isg && (g < 0 ? bcL : bcR) == BC_REFLECTIVE) u = -u;
                if (yrefl) v = -v;
                rf[cc] = fdiv(q[0], (float)a1);
                rf[BW + cc] = fdiv(q[1], (float)a2);
                rf[2 * BW + cc] = (float)u;
                rf[3 * BW + cc] = (float)v;
                rd[cc] = pr;
                rd[BW + cc] = a1;
            }
        }
        if (finish_row) {   // the copy of row r-1 issued at the start of this iteration
            const unsigned parity = (unsigned)((r - y0 - 1) & 1);
            const bool ok = mbar_wait_bounded(&bars[SLOTS], parity);
            if (__syncthreads_or(!ok)) {
                give_up(false, 0u);
                return;
            }
        }
        __syncthreads();   // S1

        // ---------------- B. reconstruction: half 0 takes rho1 rho2 u, half 1 v p a1
        const int ccm = m + 3;
        const float *f_m2 = rowf(r - 2), *f_m1 = rowf(r - 1), *f_0 = rowf(r), *f_p1 = rowf(r + 1), *f_p2 = rowf(r + 2);
        const double *d_m2 = rowd(r - 2), *d_m1 = rowd(r - 1), *d_0 = rowd(r), *d_p1 = rowd(r + 1), *d_p2 = rowd(r + 2);
        auto center = [&](int c, int cell) -> float { return f_0[c * BW + cell + 3]; };
        if (active) {
#pragma unroll 1
            for (int kv = 0; kv < 3; ++kv) {
                const int c = kv < 2 ? 2 * h + kv : 4 + h;   // half 0: rho1 rho2 p, half 1: u v a1 (no FP32/FP64 split in a pass)
                float d[12];
                if (c < 4) {
                    const int o = c * BW + ccm;
                    const float w0 = f_0[o];
                    d[0] = f_0[o - 2] - w0; d[1] = f_0[o - 1] - w0; d[2] = f_0[o + 1] - w0; d[3] = f_0[o + 2] - w0;
                    d[4] = f_m2[o] - w0; d[5] = f_m1[o] - w0; d[6] = f_p1[o] - w0; d[7] = f_p2[o] - w0;
                    d[8] = f_p1[o + 1] - w0; d[9] = f_m1[o + 1] - w0; d[10] = f_p1[o - 1] - w0; d[11] = f_m1[o - 1] - w0;
                } else {
                    const int o = (c - 4) * BW + ccm;
                    const double w0 = d_0[o];
                    d[0] = (float)(d_0[o - 2] - w0); d[1] = (float)(d_0[o - 1] - w0); d[2] = (float)(d_0[o + 1] - w0); d[3] = (float)(d_0[o + 2] - w0);
                    d[4] = (float)(d_m2[o] - w0); d[5] = (float)(d_m1[o] - w0); d[6] = (float)(d_p1[o] - w0); d[7] = (float)(d_p2[o] - w0);
                    d[8] = (float)(d_p1[o + 1] - w0); d[9] = (float)(d_m1[o + 1] - w0); d[10] = (float)(d_p1[o - 1] - w0); d[11] = (float)(d_m1[o - 1] - w0);
                }
                float cf[5];
                weno3_f(d, cf);
                cf_store(c, m, cf);
            }
        }
        __syncwarp();
        // point value of the reconstruction of cell `cell` with basis values phi[k] (k = 1..5)
        auto prim_at = [&](int cell, auto b0, auto b1) -> PrimM {
            using B0 = decltype(b0);
            using B1 = decltype(b1);
            float pv[NV];
#pragma unroll
            for (int c = 0; c < NV; ++c) pv[c] = pair_poly<B0, B1>(cf_of(c, cell), h);
            PrimM V;
            V.r1 = center(0, cell) + pv[0];
            V.r2 = center(1, cell) + pv[1];
            V.u = center(2, cell) + pv[2];
            V.v = center(3, cell) + pv[3];
            V.p = d_0[cell + 3] + (double)pv[4];
            V.a = d_0[BW + cell + 3] + (double)pv[5];
            return V;
        };
        // admissibility at the nodes: half 0 nodes 0-3 (x = +-1/2), half 1 nodes 4-7 (y = +-1/2)
        bool ok = true;
        if (active) {
            static_for<4>([&](auto sq) {
                constexpr int s0 = decltype(sq)::value, s1 = 4 + s0;
                if (!ok) return;
                const PrimM V = prim_at(m, PhiNode<2, s0>{}, PhiNode<2, s1>{});
                ok = pad_mixed(e, V);
            });
        }
        {
            const int ok_pair = __shfl_xor_sync(FULL, (int)ok, 1);
            ok = ok && (ok_pair != 0);
        }
        if (!ok && active) {   // rhs_function_prim.c:407-421 in deviation form
#pragma unroll 1
            for (int kv = 0; kv < 3; ++kv) {
                const int c = kv < 2 ? 2 * h + kv : 4 + h;   // half 0: rho1 rho2 p, half 1: u v a1 (no FP32/FP64 split in a pass)
                float dxp, dxm, dyp, dym;
                if (c < 4) {
                    const int o = c * BW + ccm;
                    const float w0 = f_0[o];
                    dxp = f_0[o + 1] - w0; dxm = w0 - f_0[o - 1]; dyp = f_p1[o] - w0; dym = w0 - f_m1[o];
                } else {
                    const int o = (c - 4) * BW + ccm;
                    const double w0 = d_0[o];
                    dxp = (float)(d_0[o + 1] - w0); dxm = (float)(w0 - d_0[o - 1]); dyp = (float)(d_p1[o] - w0); dym = (float)(w0 - d_m1[o]);
                }
                const float cf[5] = {minmod_f(dxp, dxm), minmod_f(dyp, dym), 0.0f, 0.0f, 0.0f};
                cf_store(c, m, cf);
            }
        }
        __syncwarp();
        (void)d_m2; (void)d_p2; (void)f_m2; (void)f_p2;
        // ---------------- C. y-face below (r, i), Gauss point q = h; complete row r-1
        const bool in_rows = r >= y0 && r <= y0 + H;
        const bool full_row = r >= y0 && r < y0 + H;
        const int q = h;
        {
            double Fq[NV];
            float Dq = 0.0f;
            const bool doit = owned && in_rows;
            if (doit) {
                PrimM VR = prim_at(m, PhiFace<2, 2, 0>{}, PhiFace<2, 2, 1>{});
                PrimM VL;
                VL.r1 = ytf[(q * 4 + 0) * CELLS + m]; VL.r2 = ytf[(q * 4 + 1) * CELLS + m];
                VL.u = ytf[(q * 4 + 2) * CELLS + m]; VL.v = ytf[(q * 4 + 3) * CELLS + m];
                VL.p = ytd[(q * 2 + 0) * CELLS + m]; VL.a = ytd[(q * 2 + 1) * CELLS + m];
                const float sp = riemann_mixed<1>(e, VL, VR, Fq, Dq, bad);
                smax_loc = fmaxf(smax_loc, sp);
                if (bad && bad_cell == 0xffffffffu) bad_cell = (unsigned)(r * p.nx + i);
            } else {
#pragma unroll
                for (int c = 0; c < NV; ++c) Fq[c] = 0.0;
            }
            double G[NV];
#pragma unroll
            for (int c = 0; c < NV; ++c) G[c] = 0.5 * Fq[c] + 0.5 * __shfl_xor_sync(FULL, Fq[c], 1);
            const double E5 = 0.5 * (double)Dq + 0.5 * (double)__shfl_xor_sync(FULL, Dq, 1);
            if (doit) {
                if (r > y0) {
                    const int jo = r - 1;
                    const size_t gidx = (size_t)jo * p.pitch + i;
                    // the halves take alternate variables, c = 2 j + h, so every lane works in every pass
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const int c = 2 * j + h;
                        double Y = (h ? G[2 * j + 1] : G[2 * j]) - carry[(6 + c) * CELLS + m];
                        if (c == 5) Y += 0.5 * (E5 + carry[12 * CELLS + m]);
                        const double rhs = (c == 5 ? carry[13 * CELLS + m] : 0.0) + (carry[c * CELLS + m] - r1_h * Y);
                        if (p.mode == OUT_RHS) {
                            p.out_rhs[((size_t)jo * p.nx + i) * NV + c] = rhs;
                            continue;
                        }
                        // = the stage input at (row r-1, i), staged by TMA
                        const double Sv = c < 4 ? (double)orowf[c * BW + ccm] : orowd[(c - 4) * BW + ccm];
                        double o;
                        if (p.mode == OUT_AXPY) {
                            o = Sv + b * rhs;
                        } else {
                            const double Xv = c < 4 ? (double)p.xn_f[(size_t)c * p.plane + gidx] : p.xn_d[(size_t)(c - 4) * p.plane + gidx];
                            o = (p.mode == OUT_ZXS) ? (p.ka * Xv + b * rhs) + p.kc * Sv : (p.ka * Sv + b * rhs) + p.kc * Xv;
                        }
                        if (c < 4) p.out_f[(size_t)c * p.plane + gidx] = (float)o;
                        else p.out_d[(size_t)(c - 4) * p.plane + gidx] = o;
                        if constexpr (SLAB) {   // a y-slab's edge rows are the neighbours' halo rows: store them there too
                            if (p.push_lo_f && jo < 3) {
                                const long long at = (long long)(jo + p.push_shift_lo) * p.pitch + i;
                                if (c < 4) p.push_lo_f[c * p.push_plane_lo + at] = (float)o;
                                else p.push_lo_d[(c - 4) * p.push_plane_lo + at] = o;
                            }
                            if (p.push_hi_f && jo >= p.ny - 3) {
                                const long long at = (long long)(jo + p.push_shift_hi) * p.pitch + i;
                                if (c < 4) p.push_hi_f[c * p.push_plane_hi + at] = (float)o;
                                else p.push_hi_d[(c - 4) * p.push_plane_hi + at] = o;
                            }
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < 3; ++j) carry[(6 + 2 * j + h) * CELLS + m] = h ? G[2 * j + 1] : G[2 * j];
                if (h == 1) carry[12 * CELLS + m] = E5;
            }
        }

        // ---------------- D. top-face values at Gauss point q for row r+1
        if (owned && r >= y0 - 1 && r < y0 + H) {
            const PrimM VT = prim_at(m, PhiFace<2, 3, 0>{}, PhiFace<2, 3, 1>{});
            ytf[(q * 4 + 0) * CELLS + m] = VT.r1; ytf[(q * 4 + 1) * CELLS + m] = VT.r2;
            ytf[(q * 4 + 2) * CELLS + m] = VT.u; ytf[(q * 4 + 3) * CELLS + m] = VT.v;
            ytd[(q * 2 + 0) * CELLS + m] = VT.p; ytd[(q * 2 + 1) * CELLS + m] = VT.a;
        }

        // ---------------- E. volume term of the alpha equation at Gauss points 2h, 2h+1
        {
            float tsum = 0.0f;
            if (owned && full_row) {
                static_for<2>([&](auto sa) {
                    constexpr int qa = decltype(sa)::value, qb = 2 + qa;
                    const PrimM V = prim_at(m, PhiVol<2, qa>{}, PhiVol<2, qb>{});
                    using GX0 = DPhiVolX<2, qa>;
                    using GX1 = DPhiVolX<2, qb>;
                    using GY0 = DPhiVolY<2, qa>;
                    using GY1 = DPhiVolY<2, qb>;
                    const auto c2 = cf_of(2, m), c3 = cf_of(3, m), c5 = cf_of(5, m);
                    float ux = pair_poly<GX0, GX1>(c2, h);
                    float vy = pair_poly<GY0, GY1>(c3, h);
                    float ax = pair_poly<GX0, GX1>(c5, h);
                    float ay = pair_poly<GY0, GY1>(c5, h);
                    const float r1hf = (float)r1_h;
                    ux *= r1hf; vy *= r1hf; ax *= r1hf; ay *= r1hf;
                    const float K = kapila_K(e, V.r1, V.r2, V.p, V.a);
                    tsum += -0.25f * (V.u * ax + V.v * ay - K * (ux + vy));
                });
            }
            const float other = __shfl_xor_sync(FULL, tsum, 1);
            if (owned && full_row && h == 1) carry[13 * CELLS + m] = (double)other + (double)tsum;
        }
        __syncthreads();   // S2: every column's coefficients of row r visible

        // ---------------- F. x-face at the left of column i, Gauss point q
        double Fx[NV];
        double Dx5;
        {
            double Fq[NV];
            float Dq = 0.0f;
            if (xface && full_row) {
                const PrimM VL = prim_at(m - 1, PhiFace<2, 1, 0>{}, PhiFace<2, 1, 1>{});
                const PrimM VR = prim_at(m, PhiFace<2, 0, 0>{}, PhiFace<2, 0, 1>{});
                const float sp = riemann_mixed<0>(e, VL, VR, Fq, Dq, bad);
                smax_loc = fmaxf(smax_loc, sp);
                if (bad && bad_cell == 0xffffffffu) bad_cell = (unsigned)(r * p.nx + i);
            } else {
#pragma unroll
                for (int c = 0; c < NV; ++c) Fq[c] = 0.0;
            }
#pragma unroll
            for (int c = 0; c < NV; ++c) Fx[c] = 0.5 * Fq[c] + 0.5 * __shfl_xor_sync(FULL, Fq[c], 1);
            Dx5 = 0.5 * (double)Dq + 0.5 * (double)__shfl_xor_sync(FULL, Dq, 1);
        }
        __syncthreads();   // S3
        if (xface && full_row) {
#pragma unroll
            for (int j = 0; j < 3; ++j) exch[(2 * j + h) * CELLS + m] = h ? Fx[2 * j + 1] : Fx[2 * j];
            if (h == 1) exch[6 * CELLS + m] = Dx5;
        }
        __syncthreads();   // S4
        if (owned && full_row) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int c = 2 * j + h;
                double X = exch[c * CELLS + m + 1] - (h ? Fx[2 * j + 1] : Fx[2 * j]);
                if (c == 5) X += 0.5 * (exch[6 * CELLS + m + 1] + Dx5);
                carry[c * CELLS + m] = -r1_h * X;
            }
        }
    }
    if (bad) raise_error(p.sc, ERR_INADMISSIBLE_FACE, bad_cell);
    __syncthreads();
    if (p.reduce_smax) {
        float mx = smax_loc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
        if ((t & 31) == 0) red_s[t >> 5] = (double)mx;
        __syncthreads();
        if (t == 0) {
            double b = red_s[0];
            for (int w = 1; w < K::NT / 32; ++w) b = fmax(b, red_s[w]);
            if (b > 0.0) atomicMax(&p.sc->smax, (unsigned long long)__double_as_longlong(b));
        }
    }
    for (int k = t; k <= SLOTS; k += K::NT) mbar_inval(&bars[k]);
}

template <int CELLS, bool SLAB>
__global__ void __launch_bounds__(2 * CELLS, (MixedKernel<CELLS>::MIN_BLOCKS))
mixed_kernel(const __grid_constant__ MixedMaps maps, const MixedParams p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * CELLS / 32];
    mixed_tile<CELLS, SLAB>(p, &maps, blockIdx.x, p.run0 + (int)blockIdx.y, smem_raw, red_s);
}

template <int CELLS>
__global__ void __launch_bounds__(2 * CELLS, (MixedKernel<CELLS>::MIN_BLOCKS))
mixed_batch_kernel(const MixedParams *__restrict__ inst, const MixedMaps *__restrict__ maps, const int2 *__restrict__ work,
                   int *__restrict__ sched)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * CELLS / 32];
    __shared__ int item_s;
    __shared__ MixedParams p_s;   // re-read after each barrier instead of held in registers
    const int nwork = sched[0];
    const DevScalars *last = nullptr;
    for (;;) {
        const int w = work_take(sched, nwork, last, &item_s);
        if (w >= nwork) break;
        const int2 it = work[w];
        if (threadIdx.x == 0) {
            p_s = inst[it.x];
            p_s.runs *= item_refine(it.y);
            fence_tensormap_acquire(&maps[it.x].f);
            fence_tensormap_acquire(&maps[it.x].d);
        }
        __syncthreads();
        const int tile = item_tile(it.y);
        mixed_tile<CELLS>(p_s, &maps[it.x], tile % p_s.strips, tile / p_s.strips, smem_raw, red_s);
        last = p_s.sc;
    }
    work_finish(sched);
}

struct MixedEntry {
    const void *single, *batch, *slab;
    size_t smem;
    int threads;
};
template <int CELLS>
static MixedEntry mixed_entry_of()
{
    return MixedEntry{reinterpret_cast<const void *>(mixed_kernel<CELLS, false>), reinterpret_cast<const void *>(mixed_batch_kernel<CELLS>),
                      reinterpret_cast<const void *>(mixed_kernel<CELLS, true>), MixedKernel<CELLS>::smem_bytes(), 2 * CELLS};
}
static MixedEntry mixed_entry(int cells) { return cells == 64 ? mixed_entry_of<64>() : mixed_entry_of<128>(); }

size_t mixed_smem_bytes(int sys, int cells) { return sys == SYS_KAPILA ? mixed_entry(cells).smem : mixsys_smem_bytes(sys, cells); }
int mixed_threads(int cells) { return 2 * cells; }

static cudaError_t mixed_configure(int cells)
{
    const MixedEntry e = mixed_entry(cells);
    cudaError_t r = cudaFuncSetAttribute(e.single, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(e.slab, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
    if (r != cudaSuccess) return r;
    return cudaFuncSetAttribute(e.batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
}

int mixed_blocks_per_sm(int sys, int cells)
{
    if (sys != SYS_KAPILA) return mixsys_blocks_per_sm(sys, cells, false);
    const MixedEntry e = mixed_entry(cells);
    int nb = 0;
    if (mixed_configure(cells) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.single, e.threads, e.smem) != cudaSuccess) return 0;
    return nb;
}

int mixed_batch_blocks_per_sm(int sys, int cells)
{
    if (sys != SYS_KAPILA) return mixsys_blocks_per_sm(sys, cells, true);
    const MixedEntry e = mixed_entry(cells);
    int nb = 0;
    if (mixed_configure(cells) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.batch, e.threads, e.smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_mixed(int sys, int cells, const MixedMaps &maps, const MixedParams &p, cudaStream_t s)
{
    if (sys != SYS_KAPILA) return launch_mixsys(sys, cells, maps, p, s);
    const MixedEntry e = mixed_entry(cells);
    MixedMaps mm = maps;
    MixedParams pp = p;
    void *args[] = {&mm, &pp};
    const unsigned gy = (unsigned)(p.run_count > 0 ? p.run_count : p.runs);
    return cudaLaunchKernel(p.row_off ? e.slab : e.single, dim3((unsigned)p.strips, gy, 1), dim3((unsigned)e.threads, 1, 1), args, e.smem, s);
}

cudaError_t launch_mixed_batch(int sys, int cells, const MixedParams *inst, const MixedMaps *maps, const int2 *work, int *sched,
                               int blocks, cudaStream_t s)
{
    if (sys != SYS_KAPILA) return launch_mixsys_batch(sys, cells, inst, maps, work, sched, blocks, s);
    const MixedEntry e = mixed_entry(cells);
    void *args[] = {&inst, &maps, &work, &sched};
    return cudaLaunchKernel(e.batch, dim3((unsigned)blocks, 1, 1), dim3((unsigned)e.threads, 1, 1), args, e.smem, s);
}

// interleaved FP64 Vec (nv per cell) <-> mixed planes: component c goes to FP64
// plane popc(dmask below c) where bit c of dmask is set, else to FP32 plane
// popc(~dmask below c) (MixedLayout)
__global__ void aos_to_mixed_kernel(const double *__restrict__ aos, float *__restrict__ pf, double *__restrict__ pd, int nx,
                                    int ny, int pitch, long long plane, int nv, unsigned dmask)
{
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n * nv; k += (long long)gridDim.x * blockDim.x) {
        const long long cell = k / nv;
        const int c = (int)(k % nv);
        const long long gi = (cell / nx) * pitch + cell % nx;
        const unsigned below = (1u << c) - 1u;
        if ((dmask >> c) & 1u) pd[__popc(dmask & below) * plane + gi] = aos[k];
        else pf[__popc(~dmask & below) * plane + gi] = (float)aos[k];
    }
}
__global__ void mixed_to_aos_kernel(const float *__restrict__ pf, const double *__restrict__ pd, double *__restrict__ aos, int nx,
                                    int ny, int pitch, long long plane, int nv, unsigned dmask)
{
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n * nv; k += (long long)gridDim.x * blockDim.x) {
        const long long cell = k / nv;
        const int c = (int)(k % nv);
        const long long gi = (cell / nx) * pitch + cell % nx;
        const unsigned below = (1u << c) - 1u;
        aos[k] = ((dmask >> c) & 1u) ? pd[__popc(dmask & below) * plane + gi] : (double)pf[__popc(~dmask & below) * plane + gi];
    }
}
cudaError_t launch_aos_to_mixed(int sys, const double *aos, float *pf, double *pd, int nx, int ny, int pitch, long long plane,
                                cudaStream_t s)
{
    const MixedLayout L = mixed_layout(sys);
    aos_to_mixed_kernel<<<1184, 256, 0, s>>>(aos, pf, pd, nx, ny, pitch, plane, L.nf + L.nd, L.dmask);
    return cudaGetLastError();
}
cudaError_t launch_mixed_to_aos(int sys, const float *pf, const double *pd, double *aos, int nx, int ny, int pitch, long long plane,
                                cudaStream_t s)
{
    const MixedLayout L = mixed_layout(sys);
    mixed_to_aos_kernel<<<1184, 256, 0, s>>>(pf, pd, aos, nx, ny, pitch, plane, L.nf + L.nd, L.dmask);
    return cudaGetLastError();
}

}  // namespace hype
