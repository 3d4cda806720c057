// hype_stage_mixed_sys.cu -- mixed-precision stage kernels of the
// Baer-Nunziato and Euler systems at N = 2 (primitive path): the tiling, TMA
// row staging, pair split and face bookkeeping of the Kapila mixed tile
// (hype_stage_mixed.cu), over a per-system description (MixSys<SYS>) of
//   - which conserved and primitive components live in FP64 (mixed_layout:
//     the energies and the volume fraction, where the stiffened-gas pressure
//     recovery cancels P_inf ~ 6e8 against rho e) and which in FP32
//     (densities, momenta, velocities);
//   - the conversion to primitives (baer_nunziato.c:14-41, euler.c:14-23),
//     the admissibility check (baer_nunziato.c:350-385, euler.c:292-310),
//     the Rusanov flux with its path fluctuation (riemann.c:112-140 over
//     baer_nunziato.c:47-60, 256-344 and euler.c:29-38, 197-286) and the
//     volume non-conservative term (rhs_function_prim.c:459-479).
// Reconstruction (reconstruction.c:144-221) runs in FP32 on deviations from the
// cell value, the FP64 components' point values being their FP64 cell value
// plus the FP32 deviation; fluxes of FP32 components in FP32, of FP64 components
// in FP64; cell totals, the RK combination and dt in FP64.  Not bit-compatible
// with the reference by design; its error against the FP64 path is measured in
// tests/test_gpu_mixed.py.
#include <cuda.h>
#include <cuda_runtime.h>
#include "hype_internal.h"
#include "hype_tma.cuh"
#include "hype_mixed_common.cuh"

namespace hype {

namespace {

// EOS constants of both phases in the forms the kernels use
struct MixEos {
    double g1, g2, pi1, pi2, g1m1, g2m1, i1, i2, g1pi1, g2pi2;
    float g1f, g2f;
    int fix_p2;
    __device__ __forceinline__ explicit MixEos(const Eos &e)
    {
        g1 = e.g1; g2 = e.g2; pi1 = e.pi1; pi2 = e.pi2;
        g1m1 = g1 - 1.0; g2m1 = g2 - 1.0;
        i1 = 1.0 / g1m1; i2 = 1.0 / g2m1;
        g1pi1 = g1 * pi1; g2pi2 = g2 * pi2;
        g1f = (float)g1; g2f = (float)g2;
        fix_p2 = e.fix_p2;
    }
};

template <int SYS> struct MixSys;

// euler.c: cons [rho, rho u, rho v | E], prim [rho, u, v | p]; ideal gas GAMMA_1
template <> struct MixSys<SYS_EULER> {
    static constexpr int NV = 4, NF = 3, ND = 1, NNCP = 0, NG = 0;
    static constexpr unsigned DMASK = 1u << 3;
    static constexpr int MIN_BLOCKS = 3;
    struct Pt { float f[NF]; double d[ND]; };
    static constexpr int ncp_comp(int) { return -1; }
    static constexpr int grad_comp(int) { return -1; }
    // euler.c:14-23; reflx / refly: a wall ghost (rhs_function_prim.c:101-102, 230-231)
    __device__ __forceinline__ static void conv(const MixEos &e, const float *q, const double *dq, float *vf, double *vd,
                                                bool reflx, bool refly)
    {
        const double rho = (double)q[0];
        const double irho = 1.0 / rho;
        double u = (double)q[1] * irho, v = (double)q[2] * irho;
        vd[0] = e.g1m1 * (dq[0] - 0.5 * rho * (u * u + v * v));
        if (reflx) u = -u;
        if (refly) v = -v;
        vf[0] = q[0];
        vf[1] = (float)u;
        vf[2] = (float)v;
    }
    // euler.c:292-310
    __device__ __forceinline__ static bool pad(const MixEos &, const Pt &V)
    {
        return !(V.f[0] < 1.0e-14f) && !(V.d[0] < PRS_FLOOR);
    }
    // riemann.c:112-140 with euler.c:29-38 (conserved values) and euler.c:197-236 (flux)
    template <int DIR>
    __device__ __forceinline__ static float riemann(const MixEos &e, const Pt &L, const Pt &R, double *F, double *, bool &bad)
    {
        float FL[3], FR[3], QL[3], QR[3];
        double EL, ER, F3L, F3R;
        auto side = [&](const Pt &V, float *Fs, float *Qs, double &Es, double &F3s) -> float {
            const float rho = V.f[0], u = V.f[1], v = V.f[2];
            const float un = DIR == 0 ? u : v;
            const double p = V.d[0];
            Es = p * e.i1 + (double)(0.5f * rho * (u * u + v * v));
            bad |= (rho < 1.0e-14f) | (p < PRS_FLOOR);
            const float pf = (float)p, rhoun = rho * un;
            Fs[0] = rhoun;
            Fs[1] = rhoun * u + (DIR == 0 ? pf : 0.0f);
            Fs[2] = rhoun * v + (DIR == 1 ? pf : 0.0f);
            F3s = (double)un * (Es + p);
            Qs[0] = rho; Qs[1] = rho * u; Qs[2] = rho * v;
            return fabsf(un) + sqrtf(fdiv((float)(e.g1 * p), rho));
        };
        const float sl = side(L, FL, QL, EL, F3L);
        const float sr = side(R, FR, QR, ER, F3R);
        const float s = (sl < sr) ? sr : sl;
#pragma unroll
        for (int c = 0; c < 3; ++c) F[c] = (double)(0.5f * (FR[c] + FL[c] - s * (QR[c] - QL[c])));
        F[3] = 0.5 * (F3R + F3L - (double)s * (ER - EL));
        return s;
    }
    __device__ __forceinline__ static void vol_ncp(const MixEos &, const Pt &, const float *, const float *, double *) {}
};

// baer_nunziato.c: cons [a1 r1, a1 r1 u1, a1 r1 v1, a1 E1, a2 r2, a2 r2 u2, a2 r2 v2, a2 E2, a1]
//                  prim [r1, u1, v1, p1, r2, u2, v2, p2, a1]
// FP32 slots: r1 u1 v1 r2 u2 v2 (components 0 1 2 4 5 6); FP64 slots: p1 p2 a1 (3 7 8).
// Non-conservative components 1 2 3 5 6 7 8 (baer_nunziato.c:327-344: u_I = u1, p_I = p2).
template <> struct MixSys<SYS_BN> {
    static constexpr int NV = 9, NF = 6, ND = 3, NNCP = 7, NG = 1;
    static constexpr unsigned DMASK = (1u << 3) | (1u << 7) | (1u << 8);
    static constexpr int MIN_BLOCKS = 2;
    struct Pt { float f[NF]; double d[ND]; };
    static constexpr int ncp_comp(int j) { return j < 3 ? j + 1 : j + 2; }
    static constexpr int grad_comp(int) { return 8; }   // the volume term needs grad a1 only
    // baer_nunziato.c:14-41; reflx / refly: a wall ghost (rhs_function_prim.c:115-117, 244-246)
    __device__ __forceinline__ static void conv(const MixEos &e, const float *q, const double *dq, float *vf, double *vd,
                                                bool reflx, bool refly)
    {
        const double phi_1 = dq[2], phi_2 = 1.0 - dq[2];
        const double q0 = (double)q[0], q3 = (double)q[3];
        const double rho_1 = q0 / phi_1, rho_2 = q3 / phi_2;
        const double iq0 = 1.0 / q0, iq3 = 1.0 / q3;
        double u_1 = (double)q[1] * iq0, v_1 = (double)q[2] * iq0;
        double u_2 = (double)q[4] * iq3, v_2 = (double)q[5] * iq3;
        const double E_1 = dq[0] / phi_1, E_2 = dq[1] / phi_2;
        vd[0] = e.g1m1 * (E_1 - 0.5 * rho_1 * (u_1 * u_1 + v_1 * v_1)) - e.g1pi1;
        vd[1] = e.g2m1 * (E_2 - 0.5 * rho_2 * (u_2 * u_2 + v_2 * v_2)) - e.g2pi2;
        vd[2] = phi_1;
        if (reflx) { u_1 = -u_1; u_2 = -u_2; }
        if (refly) { v_1 = -v_1; v_2 = -v_2; }
        vf[0] = (float)rho_1; vf[1] = (float)u_1; vf[2] = (float)v_1;
        vf[3] = (float)rho_2; vf[4] = (float)u_2; vf[5] = (float)v_2;
    }
    // baer_nunziato.c:350-385
    __device__ __forceinline__ static bool pad(const MixEos &e, const Pt &V)
    {
        bool ok = true;
        if (V.f[0] < 1.0e-14f) ok = false;
        if (V.f[3] < 1.0e-14f) ok = false;
        if ((V.d[0] + e.pi1) < PRS_FLOOR) ok = false;
        if ((V.d[1] + e.pi2) < PRS_FLOOR) ok = false;
        if (V.d[2] < 0.0 || V.d[2] > 1.0) ok = false;
        return ok;
    }
    // riemann.c:112-140 with baer_nunziato.c:47-60 (conserved values, p2 = V[7]) and
    // :256-321 (flux; its phase-2 pressure is V[8] as written, V[7] with fix_p2), the
    // fluctuation B(V_avg) (V_R - V_L) n of :327-344
    template <int DIR>
    __device__ __forceinline__ static float riemann(const MixEos &e, const Pt &L, const Pt &R, double *F, double *D, bool &bad)
    {
        float FL[6], FR[6], QL[6], QR[6];
        double GL[3], GR[3], CL[3], CR[3];   // FP64 components 3 7 8: flux, conserved value
        auto side = [&](const Pt &V, float *Fs, float *Qs, double *Gs, double *Cs) -> float {
            const double phi_1 = V.d[2], phi_2 = 1.0 - V.d[2];
            const float f1 = (float)phi_1, f2 = (float)phi_2;
            const float rho_1 = V.f[0], u_1 = V.f[1], v_1 = V.f[2];
            const float rho_2 = V.f[3], u_2 = V.f[4], v_2 = V.f[5];
            const double p_1 = V.d[0];
            const double p_2 = e.fix_p2 ? V.d[1] : V.d[2];   // the flux's phase-2 pressure
            const float un_1 = DIR == 0 ? u_1 : v_1, un_2 = DIR == 0 ? u_2 : v_2;
            const double k_1 = (double)(0.5f * rho_1 * (u_1 * u_1 + v_1 * v_1));
            const double k_2 = (double)(0.5f * rho_2 * (u_2 * u_2 + v_2 * v_2));
            const double E_1 = (p_1 + e.g1pi1) * e.i1 + k_1;
            const double E_2 = (p_2 + e.g2pi2) * e.i2 + k_2;
            bad |= (rho_1 < 1.0e-14f) | (rho_2 < 1.0e-14f) | ((p_1 + e.pi1) < PRS_FLOOR) | ((p_2 + e.pi2) < PRS_FLOOR);
            const float p1f = (float)p_1, p2f = (float)p_2;
            Fs[0] = f1 * rho_1 * un_1;
            Fs[1] = f1 * (rho_1 * u_1 * un_1 + (DIR == 0 ? p1f : 0.0f));
            Fs[2] = f1 * (rho_1 * v_1 * un_1 + (DIR == 1 ? p1f : 0.0f));
            Fs[3] = f2 * rho_2 * un_2;
            Fs[4] = f2 * (rho_2 * u_2 * un_2 + (DIR == 0 ? p2f : 0.0f));
            Fs[5] = f2 * (rho_2 * v_2 * un_2 + (DIR == 1 ? p2f : 0.0f));
            Gs[0] = phi_1 * (double)un_1 * (E_1 + p_1);
            Gs[1] = phi_2 * (double)un_2 * (E_2 + p_2);
            Gs[2] = 0.0;
            Qs[0] = f1 * rho_1; Qs[1] = Qs[0] * u_1; Qs[2] = Qs[0] * v_1;
            Qs[3] = f2 * rho_2; Qs[4] = Qs[3] * u_2; Qs[5] = Qs[3] * v_2;
            Cs[0] = phi_1 * E_1;
            Cs[1] = phi_2 * ((V.d[1] + e.g2pi2) * e.i2 + k_2);   // prim2cons takes p2 = V[7]
            Cs[2] = phi_1;
            const float s_1 = fabsf(un_1) + sqrtf(fdiv((float)(e.g1 * (p_1 + e.pi1)), rho_1));
            const float s_2 = fabsf(un_2) + sqrtf(fdiv((float)(e.g2 * (p_2 + e.pi2)), rho_2));
            return (s_1 < s_2) ? s_2 : s_1;
        };
        const float sl = side(L, FL, QL, GL, CL);
        const float sr = side(R, FR, QR, GR, CR);
        const float s = (sl < sr) ? sr : sl;
        constexpr int fc[6] = {0, 1, 2, 4, 5, 6}, dc[3] = {3, 7, 8};
#pragma unroll
        for (int k = 0; k < 6; ++k) F[fc[k]] = (double)(0.5f * (FR[k] + FL[k] - s * (QR[k] - QL[k])));
#pragma unroll
        for (int k = 0; k < 3; ++k) F[dc[k]] = 0.5 * (GR[k] + GL[k] - (double)s * (CR[k] - CL[k]));
        // fluctuation at the face average: u_I, v_I = phase-1 velocity, p_I = phase-2 pressure (V[7])
        const double uI = 0.5 * ((double)R.f[1] + (double)L.f[1]), vI = 0.5 * ((double)R.f[2] + (double)L.f[2]);
        const double pI = 0.5 * (R.d[1] + L.d[1]);
        const double da = R.d[2] - L.d[2];
        const double ph_x = DIR == 0 ? da : 0.0, ph_y = DIR == 1 ? da : 0.0;
        const double un = uI * ph_x + vI * ph_y;
        D[0] = -pI * ph_x; D[1] = -pI * ph_y; D[2] = -pI * un;
        D[3] = pI * ph_x;  D[4] = pI * ph_y;  D[5] = pI * un;
        D[6] = un;
        return s;
    }
    // B(V) grad V at a volume Gauss point (baer_nunziato.c:327-344): gx[0], gy[0] = grad a1
    __device__ __forceinline__ static void vol_ncp(const MixEos &, const Pt &V, const float *gx, const float *gy, double *B)
    {
        const double uI = (double)V.f[1], vI = (double)V.f[2], pI = V.d[1];
        const double ax = (double)gx[0], ay = (double)gy[0];
        const double un = uI * ax + vI * ay;
        B[0] = -pI * ax; B[1] = -pI * ay; B[2] = -pI * un;
        B[3] = pI * ax;  B[4] = pI * ay;  B[5] = pI * un;
        B[6] = un;
    }
};

// component c of the system: FP64 or FP32, and its slot among those planes
template <class M> __host__ __device__ constexpr bool is_d(int c) { return (M::DMASK >> c) & 1u; }
template <class M> __host__ __device__ constexpr int slot_of_comp(int c)
{
    int k = 0;
    for (int j = 0; j < c; ++j) k += (is_d<M>(j) == is_d<M>(c)) ? 1 : 0;
    return k;
}
// the non-conservative slot of component c, or -1
template <class M> __host__ __device__ constexpr int ncp_slot(int c)
{
    for (int j = 0; j < M::NNCP; ++j)
        if (M::ncp_comp(j) == c) return j;
    return -1;
}

}  // namespace

template <int SYS, int CELLS_>
struct MixSysKernel {
    using M = MixSys<SYS>;
    static constexpr int NV = M::NV, NF = M::NF, ND = M::ND, NNCP = M::NNCP;
    static constexpr int CELLS = CELLS_;
    static constexpr int NT = 2 * CELLS;
    static constexpr int BW = CELLS + 8;                 // multiple of 4 floats (16 B)
    static constexpr int SLOTS = STAGE_SLOTS;
    static constexpr int F_ROW_BYTES = NF * BW * 4;
    static constexpr int D_ROW_BYTES = ND * BW * 8;
    static constexpr int F_REGION = (F_ROW_BYTES + 127) / 128 * 128;
    static constexpr int D_REGION = (D_ROW_BYTES + 127) / 128 * 128;
    static constexpr int SLOT_BYTES = F_REGION + D_REGION;
    static constexpr int COEF_FLOATS = 5 * NV * CELLS;   // [k-1][c][cell]; after S3 the x-face exchange
    static_assert(2 * (NV + NNCP) <= 5 * NV, "x-face exchange exceeds the coefficient buffer");
    static constexpr int YTF_FLOATS = 2 * NF * CELLS;    // top-face FP32 values, by Gauss point
    static constexpr int YTD_DOUBLES = 2 * ND * CELLS;   // top-face FP64 values
    // pre[NV] (volume term + x-flux difference of the row), G below[NV], E below[NNCP]
    static constexpr int CARRY_DOUBLES = (2 * NV + NNCP) * CELLS;
    static constexpr int MIN_BLOCKS = M::MIN_BLOCKS * (128 / CELLS);
    static constexpr size_t smem_bytes()
    {
        return 128 + (size_t)(SLOTS + 1) * SLOT_BYTES + (size_t)COEF_FLOATS * 4 + (size_t)YTF_FLOATS * 4 +
               (size_t)YTD_DOUBLES * 8 + (size_t)CARRY_DOUBLES * 8 + 64;
    }
};

// SLAB: a y-slab of a decomposed grid (row offset, edge rows stored into the
// neighbours' halo rows); the single-grid and batched kernels compile without it.
template <int SYS, int CELLS_, bool SLAB = false>
__device__ __forceinline__ void mixsys_tile(const MixedParams &p, const MixedMaps *maps, int strip, int run,
                                            unsigned char *smem, double *red_s)
{
    using K = MixSysKernel<SYS, CELLS_>;
    using M = typename K::M;
    using Pt = typename M::Pt;
    using QD = Quad<2>;
    constexpr int NV = K::NV, NF = K::NF, ND = K::ND, NNCP = K::NNCP, NG = M::NG;
    constexpr int CELLS = K::CELLS, BW = K::BW, SLOTS = K::SLOTS;
    constexpr int NVH = (NV + 1) / 2;
    constexpr unsigned FULL = 0xffffffffu;
    if (p.sc->idle) return;

    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    unsigned char *rows = smem + 128;
    unsigned char *orow = rows + (size_t)SLOTS * K::SLOT_BYTES;   // stage input of row r-1: FP32 then FP64 planes
    const float *orowf = reinterpret_cast<const float *>(orow);
    const double *orowd = reinterpret_cast<const double *>(orow + K::F_REGION);
    float *coef_f = reinterpret_cast<float *>(rows + (size_t)(SLOTS + 1) * K::SLOT_BYTES);
    double *exch = reinterpret_cast<double *>(coef_f);                  // x-face fluxes after S3: [NV + NNCP][cell]
    float *ytf = coef_f + K::COEF_FLOATS;                                 // [q][NF][cell]
    double *ytd = reinterpret_cast<double *>(ytf + K::YTF_FLOATS);        // [q][ND][cell]
    double *carry = ytd + K::YTD_DOUBLES;                                 // [2 NV + NNCP][cell]
    double *pre = carry, *gbelow = carry + NV * CELLS, *ebelow = carry + 2 * NV * CELLS;

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
    const MixEos e(p.eos);
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
    auto cf_at = [&](int k1, int c, int cell) -> float & { return coef_f[(k1 * NV + c) * CELLS + cell]; };

    float smax_loc = 0.0f;
    bool bad = false;
    unsigned bad_cell = 0xffffffffu;
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
        const bool finish_row = r > y0 && p.mode != OUT_RHS;
        // ---------------- A. rows up to r+2: two TMA loads (FP32, FP64 planes) per row
        if (t == 0) {
            fence_proxy_async();
            for (; next_issue <= min(r + 3, row_hi) && (!p.skip_loads || next_issue < p.skip_loads_from); ++next_issue) {
                const int row = next_issue;
                const int src = map_axis(row, p.ny, bcB, bcT);
                uint64_t *bar = &bars[slot_of(row)];
                mbar_expect_tx(bar, K::F_ROW_BYTES + K::D_ROW_BYTES);
                const int ty = SLAB ? src + p.row_off : src;
                tma_load_3d(rowf(row), &maps->f, xs, ty, 0, bar);
                tma_load_3d(rowd(row), &maps->d, xs, ty, 0, bar);
            }
            if (finish_row && (!p.skip_loads || r - 1 < p.skip_loads_from)) {
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
            float q[NF];
            double dq[ND];
            if (touches_x) {
                if (isg) {
                    const int gm = map_axis(g, p.nx, bcL, bcR);
                    if (gm - xs >= 0 && gm - xs < BW) {
#pragma unroll
                        for (int c = 0; c < NF; ++c) q[c] = rf[c * BW + (gm - xs)];
#pragma unroll
                        for (int c = 0; c < ND; ++c) dq[c] = rd[c * BW + (gm - xs)];
                    } else {
                        const long long gi = (long long)src * p.pitch + gm;
#pragma unroll
                        for (int c = 0; c < NF; ++c) q[c] = p.in_f[(long long)c * p.plane + gi];
#pragma unroll
                        for (int c = 0; c < ND; ++c) dq[c] = p.in_d[(long long)c * p.plane + gi];
                    }
                }
                __syncthreads();
            }
            if (conv) {
                if (!isg) {
#pragma unroll
                    for (int c = 0; c < NF; ++c) q[c] = rf[c * BW + cc];
#pragma unroll
                    for (int c = 0; c < ND; ++c) dq[c] = rd[c * BW + cc];
                }
                float vf[NF];
                double vd[ND];
                M::conv(e, q, dq, vf, vd, isg && (g < 0 ? bcL : bcR) == BC_REFLECTIVE, yrefl);
#pragma unroll
                for (int c = 0; c < NF; ++c) rf[c * BW + cc] = vf[c];
#pragma unroll
                for (int c = 0; c < ND; ++c) rd[c * BW + cc] = vd[c];
            }
        }
        if (finish_row) {
            const unsigned parity = (unsigned)((r - y0 - 1) & 1);
            const bool ok = mbar_wait_bounded(&bars[SLOTS], parity);
            if (__syncthreads_or(!ok)) {
                give_up(false, 0u);
                return;
            }
        }
        __syncthreads();   // S1

        // ---------------- B. reconstruction: half h takes components h*NVH ..
        const int ccm = m + 3;
        const float *f_m2 = rowf(r - 2), *f_m1 = rowf(r - 1), *f_0 = rowf(r), *f_p1 = rowf(r + 1), *f_p2 = rowf(r + 2);
        const double *d_m2 = rowd(r - 2), *d_m1 = rowd(r - 1), *d_0 = rowd(r), *d_p1 = rowd(r + 1), *d_p2 = rowd(r + 2);
        if (active) {
#pragma unroll 1
            for (int kv = 0; kv < NVH; ++kv) {
                const int c = h * NVH + kv;
                if (c >= NV) break;
                const bool dcomp = (M::DMASK >> c) & 1u;
                const int sl = __popc(dcomp ? (M::DMASK & ((1u << c) - 1u)) : (~M::DMASK & ((1u << c) - 1u)));
                float d[12];
                if (!dcomp) {
                    const int o = sl * BW + ccm;
                    const float w0 = f_0[o];
                    d[0] = f_0[o - 2] - w0; d[1] = f_0[o - 1] - w0; d[2] = f_0[o + 1] - w0; d[3] = f_0[o + 2] - w0;
                    d[4] = f_m2[o] - w0; d[5] = f_m1[o] - w0; d[6] = f_p1[o] - w0; d[7] = f_p2[o] - w0;
                    d[8] = f_p1[o + 1] - w0; d[9] = f_m1[o + 1] - w0; d[10] = f_p1[o - 1] - w0; d[11] = f_m1[o - 1] - w0;
                } else {
                    const int o = sl * BW + ccm;
                    const double w0 = d_0[o];
                    d[0] = (float)(d_0[o - 2] - w0); d[1] = (float)(d_0[o - 1] - w0); d[2] = (float)(d_0[o + 1] - w0); d[3] = (float)(d_0[o + 2] - w0);
                    d[4] = (float)(d_m2[o] - w0); d[5] = (float)(d_m1[o] - w0); d[6] = (float)(d_p1[o] - w0); d[7] = (float)(d_p2[o] - w0);
                    d[8] = (float)(d_p1[o + 1] - w0); d[9] = (float)(d_m1[o + 1] - w0); d[10] = (float)(d_p1[o - 1] - w0); d[11] = (float)(d_m1[o - 1] - w0);
                }
                float cf[5];
                weno3_f(d, cf);
#pragma unroll
                for (int k = 0; k < 5; ++k) cf_at(k, c, m) = cf[k];
            }
        }
        __syncwarp();
        // point value of the reconstruction of cell `cell` with basis values phi_of(k), k = 1..5
        auto prim_at = [&](int cell, auto b0, auto b1) -> Pt {
            using B0 = decltype(b0);
            using B1 = decltype(b1);
            Pt V;
            static_for<NV>([&](auto cc_) {
                constexpr int c = decltype(cc_)::value;
                constexpr int sl = slot_of_comp<M>(c);
                const float v = pair_poly<B0, B1>([&](int k1) { return cf_at(k1, c, cell); }, h);
                if constexpr (is_d<M>(c)) V.d[sl] = d_0[sl * BW + cell + 3] + (double)v;
                else V.f[sl] = f_0[sl * BW + cell + 3] + v;
            });
            return V;
        };
        // admissibility at the nodes: half 0 nodes 0-3 (x = +-1/2), half 1 nodes 4-7 (y = +-1/2)
        bool ok = true;
        if (active) {
            static_for<4>([&](auto sq) {
                constexpr int s0 = decltype(sq)::value, s1 = 4 + s0;
                if (!ok) return;
                const Pt V = prim_at(m, PhiNode<2, s0>{}, PhiNode<2, s1>{});
                ok = M::pad(e, V);
            });
        }
        {
            const int ok_pair = __shfl_xor_sync(FULL, (int)ok, 1);
            ok = ok && (ok_pair != 0);
        }
        if (!ok && active) {   // rhs_function_prim.c:407-421 in deviation form
#pragma unroll 1
            for (int kv = 0; kv < NVH; ++kv) {
                const int c = h * NVH + kv;
                if (c >= NV) break;
                const bool dcomp = (M::DMASK >> c) & 1u;
                const int sl = __popc(dcomp ? (M::DMASK & ((1u << c) - 1u)) : (~M::DMASK & ((1u << c) - 1u)));
                const int o = sl * BW + ccm;
                float dxp, dxm, dyp, dym;
                if (!dcomp) {
                    const float w0 = f_0[o];
                    dxp = f_0[o + 1] - w0; dxm = w0 - f_0[o - 1]; dyp = f_p1[o] - w0; dym = w0 - f_m1[o];
                } else {
                    const double w0 = d_0[o];
                    dxp = (float)(d_0[o + 1] - w0); dxm = (float)(w0 - d_0[o - 1]); dyp = (float)(d_p1[o] - w0); dym = (float)(w0 - d_m1[o]);
                }
                cf_at(0, c, m) = minmod_f(dxp, dxm);
                cf_at(1, c, m) = minmod_f(dyp, dym);
                cf_at(2, c, m) = 0.0f; cf_at(3, c, m) = 0.0f; cf_at(4, c, m) = 0.0f;
            }
        }
        __syncwarp();
        (void)d_m2; (void)d_p2; (void)f_m2; (void)f_p2;
        // ---------------- C. y-face below (r, i), Gauss point q = h; complete row r-1
        const bool in_rows = r >= y0 && r <= y0 + H;
        const bool full_row = r >= y0 && r < y0 + H;
        const int q = h;
        {
            double Fq[NV], Dq[NNCP > 0 ? NNCP : 1];
            const bool doit = owned && in_rows;
            if (doit) {
                const Pt VR = prim_at(m, PhiFace<2, 2, 0>{}, PhiFace<2, 2, 1>{});
                Pt VL;
#pragma unroll
                for (int c = 0; c < NF; ++c) VL.f[c] = ytf[(q * NF + c) * CELLS + m];
#pragma unroll
                for (int c = 0; c < ND; ++c) VL.d[c] = ytd[(q * ND + c) * CELLS + m];
                const float sp = M::template riemann<1>(e, VL, VR, Fq, Dq, bad);
                smax_loc = fmaxf(smax_loc, sp);
                if (bad && bad_cell == 0xffffffffu) bad_cell = (unsigned)(r * p.nx + i);
            } else {
#pragma unroll
                for (int c = 0; c < NV; ++c) Fq[c] = 0.0;
#pragma unroll
                for (int j = 0; j < NNCP; ++j) Dq[j] = 0.0;
            }
            double G[NV], E[NNCP > 0 ? NNCP : 1];
#pragma unroll
            for (int c = 0; c < NV; ++c) G[c] = 0.5 * Fq[c] + 0.5 * __shfl_xor_sync(FULL, Fq[c], 1);
#pragma unroll
            for (int j = 0; j < NNCP; ++j) E[j] = 0.5 * Dq[j] + 0.5 * __shfl_xor_sync(FULL, Dq[j], 1);
            if (doit) {
                if (r > y0) {
                    const int jo = r - 1;
                    const size_t gidx = (size_t)jo * p.pitch + i;
                    // one variable of row r-1: c, its plane kind and slot, its non-conservative slot jn
                    auto finish_one = [&](int c, auto dcomp_, auto ncp_, int sl, int jn, double Gc, double Ec) {
                        constexpr bool dcomp = decltype(dcomp_)::value != 0, has_ncp = decltype(ncp_)::value != 0;
                        double Y = Gc - gbelow[c * CELLS + m];
                        if constexpr (has_ncp) Y += 0.5 * (Ec + ebelow[jn * CELLS + m]);
                        const double rhs = pre[c * CELLS + m] - r1_h * Y;
                        if (p.mode == OUT_RHS) {
                            p.out_rhs[((size_t)jo * p.nx + i) * NV + c] = rhs;
                            return;
                        }
                        const double Sv = dcomp ? orowd[sl * BW + ccm] : (double)orowf[sl * BW + ccm];
                        double o;
                        if (p.mode == OUT_AXPY) {
                            o = Sv + b * rhs;
                        } else {
                            const double Xv = dcomp ? p.xn_d[(size_t)sl * p.plane + gidx] : (double)p.xn_f[(size_t)sl * p.plane + gidx];
                            o = (p.mode == OUT_ZXS) ? (p.ka * Xv + b * rhs) + p.kc * Sv : (p.ka * Sv + b * rhs) + p.kc * Xv;
                        }
                        if (dcomp) p.out_d[(size_t)sl * p.plane + gidx] = o;
                        else p.out_f[(size_t)sl * p.plane + gidx] = (float)o;
                        if constexpr (SLAB) {
                            if (p.push_lo_f && jo < 3) {
                                const long long at = (long long)(jo + p.push_shift_lo) * p.pitch + i;
                                if (dcomp) p.push_lo_d[sl * p.push_plane_lo + at] = o;
                                else p.push_lo_f[sl * p.push_plane_lo + at] = (float)o;
                            }
                            if (p.push_hi_f && jo >= p.ny - 3) {
                                const long long at = (long long)(jo + p.push_shift_hi) * p.pitch + i;
                                if (dcomp) p.push_hi_d[sl * p.push_plane_hi + at] = o;
                                else p.push_hi_f[sl * p.push_plane_hi + at] = (float)o;
                            }
                        }
                    };
                    // the halves take variables 2 j and 2 j + 1 of pair j: one code path when
                    // the two are of one kind (plane type, non-conservative term), so that
                    // every lane works in the same pass
                    static_for<(NV + 1) / 2>([&](auto jj_) {
                        constexpr int c0 = 2 * decltype(jj_)::value, c1 = c0 + 1;
                        constexpr bool two = c1 < NV;
                        constexpr bool d0 = is_d<M>(c0), d1 = is_d<M>(c1);
                        constexpr int n0 = ncp_slot<M>(c0), n1 = two ? ncp_slot<M>(c1) : -1;
                        constexpr int s0 = slot_of_comp<M>(c0), s1 = slot_of_comp<M>(c1);
                        constexpr int e0 = n0 >= 0 ? n0 : 0, e1 = n1 >= 0 ? n1 : 0;
                        constexpr int g1 = two ? c1 : c0;
                        if constexpr (two && d0 == d1 && ((n0 >= 0) == (n1 >= 0))) {
                            finish_one(h ? c1 : c0, ic<d0 ? 1 : 0>{}, ic<(n0 >= 0) ? 1 : 0>{}, h ? s1 : s0, h ? n1 : n0,
                                       h ? G[g1] : G[c0], h ? E[e1] : E[e0]);
                        } else {
                            if (h == 0) finish_one(c0, ic<d0 ? 1 : 0>{}, ic<(n0 >= 0) ? 1 : 0>{}, s0, n0, G[c0], E[e0]);
                            else if (two) finish_one(c1, ic<d1 ? 1 : 0>{}, ic<(n1 >= 0) ? 1 : 0>{}, s1, n1, G[g1], E[e1]);
                        }
                    });
                }
                static_for<(NV + 1) / 2>([&](auto jj_) {
                    constexpr int c0 = 2 * decltype(jj_)::value, c1 = c0 + 1;
                    constexpr bool two = c1 < NV;
                    constexpr int g1 = two ? c1 : c0;
                    constexpr int n0 = ncp_slot<M>(c0), n1 = two ? ncp_slot<M>(c1) : -1;
                    if (h == 0 || two) gbelow[(h ? g1 : c0) * CELLS + m] = h ? G[g1] : G[c0];
                    if constexpr (n0 >= 0) if (h == 0) ebelow[n0 * CELLS + m] = E[n0];
                    if constexpr (n1 >= 0) if (h == 1) ebelow[n1 * CELLS + m] = E[n1];
                });
            }
        }

        // ---------------- D. top-face values at Gauss point q for row r+1
        if (owned && r >= y0 - 1 && r < y0 + H) {
            const Pt VT = prim_at(m, PhiFace<2, 3, 0>{}, PhiFace<2, 3, 1>{});
#pragma unroll
            for (int c = 0; c < NF; ++c) ytf[(q * NF + c) * CELLS + m] = VT.f[c];
#pragma unroll
            for (int c = 0; c < ND; ++c) ytd[(q * ND + c) * CELLS + m] = VT.d[c];
        }

        // ---------------- E. volume non-conservative term at Gauss points 2h, 2h+1
        if constexpr (NNCP > 0) {
            double tsum[NNCP];
#pragma unroll
            for (int j = 0; j < NNCP; ++j) tsum[j] = 0.0;
            if (owned && full_row) {
                static_for<2>([&](auto sa) {
                    constexpr int qa = decltype(sa)::value, qb = 2 + qa;
                    const Pt V = prim_at(m, PhiVol<2, qa>{}, PhiVol<2, qb>{});
                    float gx[NG], gy[NG];
#pragma unroll
                    for (int gg = 0; gg < NG; ++gg) {
                        const int c = M::grad_comp(gg);
                        const float ax = pair_poly<DPhiVolX<2, qa>, DPhiVolX<2, qb>>([&](int k1) { return cf_at(k1, c, m); }, h);
                        const float ay = pair_poly<DPhiVolY<2, qa>, DPhiVolY<2, qb>>([&](int k1) { return cf_at(k1, c, m); }, h);
                        gx[gg] = ax * (float)r1_h;
                        gy[gg] = ay * (float)r1_h;
                    }
                    double B[NNCP];
                    M::vol_ncp(e, V, gx, gy, B);
#pragma unroll
                    for (int j = 0; j < NNCP; ++j) tsum[j] += -0.25 * B[j];
                });
            }
            static_for<NNCP>([&](auto jj_) {
                constexpr int j = decltype(jj_)::value;
                constexpr int c = M::ncp_comp(j);
                const double other = __shfl_xor_sync(FULL, tsum[j], 1);
                if (owned && full_row && (c & 1) == h) pre[c * CELLS + m] = tsum[j] + other;
            });
        }
        __syncthreads();   // S2: every column's coefficients of row r visible

        // ---------------- F. x-face at the left of column i, Gauss point q
        double Fx[NV], Dx[NNCP > 0 ? NNCP : 1];
        {
            double Fq[NV], Dq[NNCP > 0 ? NNCP : 1];
            if (xface && full_row) {
                const Pt VL = prim_at(m - 1, PhiFace<2, 1, 0>{}, PhiFace<2, 1, 1>{});
                const Pt VR = prim_at(m, PhiFace<2, 0, 0>{}, PhiFace<2, 0, 1>{});
                const float sp = M::template riemann<0>(e, VL, VR, Fq, Dq, bad);
                smax_loc = fmaxf(smax_loc, sp);
                if (bad && bad_cell == 0xffffffffu) bad_cell = (unsigned)(r * p.nx + i);
            } else {
#pragma unroll
                for (int c = 0; c < NV; ++c) Fq[c] = 0.0;
#pragma unroll
                for (int j = 0; j < NNCP; ++j) Dq[j] = 0.0;
            }
#pragma unroll
            for (int c = 0; c < NV; ++c) Fx[c] = 0.5 * Fq[c] + 0.5 * __shfl_xor_sync(FULL, Fq[c], 1);
#pragma unroll
            for (int j = 0; j < NNCP; ++j) Dx[j] = 0.5 * Dq[j] + 0.5 * __shfl_xor_sync(FULL, Dq[j], 1);
        }
        __syncthreads();   // S3
        if (xface && full_row) {
            static_for<(NV + 1) / 2>([&](auto jj_) {
                constexpr int c0 = 2 * decltype(jj_)::value, c1 = c0 + 1;
                constexpr bool two = c1 < NV;
                constexpr int g1 = two ? c1 : c0;
                constexpr int n0 = ncp_slot<M>(c0), n1 = two ? ncp_slot<M>(c1) : -1;
                if (h == 0 || two) exch[(h ? g1 : c0) * CELLS + m] = h ? Fx[g1] : Fx[c0];
                if constexpr (n0 >= 0) if (h == 0) exch[(NV + n0) * CELLS + m] = Dx[n0];
                if constexpr (n1 >= 0) if (h == 1) exch[(NV + n1) * CELLS + m] = Dx[n1];
            });
        }
        __syncthreads();   // S4
        if (owned && full_row) {
            static_for<NV>([&](auto cc_) {
                constexpr int c = decltype(cc_)::value;
                if ((c & 1) != h) return;
                double X = exch[c * CELLS + m + 1] - Fx[c];
                constexpr int jn = ncp_slot<M>(c);
                if constexpr (jn >= 0) {
                    X += 0.5 * (exch[(NV + jn) * CELLS + m + 1] + Dx[jn]);
                    pre[c * CELLS + m] = pre[c * CELLS + m] + (-r1_h * X);
                } else {
                    pre[c * CELLS + m] = -r1_h * X;
                }
            });
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

template <int SYS, int CELLS, bool SLAB>
__global__ void __launch_bounds__(2 * CELLS, (MixSysKernel<SYS, CELLS>::MIN_BLOCKS))
mixsys_kernel(const __grid_constant__ MixedMaps maps, const MixedParams p)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_s[2 * CELLS / 32];
    mixsys_tile<SYS, CELLS, SLAB>(p, &maps, blockIdx.x, p.run0 + (int)blockIdx.y, smem_raw, red_s);
}

template <int SYS, int CELLS>
__global__ void __launch_bounds__(2 * CELLS, (MixSysKernel<SYS, CELLS>::MIN_BLOCKS))
mixsys_batch_kernel(const MixedParams *__restrict__ inst, const MixedMaps *__restrict__ maps, const int2 *__restrict__ work,
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
        mixsys_tile<SYS, CELLS>(p_s, &maps[it.x], tile % p_s.strips, tile / p_s.strips, smem_raw, red_s);
        last = p_s.sc;
    }
    work_finish(sched);
}

namespace {
struct MixSysEntry {
    const void *single, *batch, *slab;
    size_t smem;
    int threads;
};
template <int SYS, int CELLS>
MixSysEntry mixsys_entry_of()
{
    return MixSysEntry{reinterpret_cast<const void *>(mixsys_kernel<SYS, CELLS, false>),
                       reinterpret_cast<const void *>(mixsys_batch_kernel<SYS, CELLS>),
                       reinterpret_cast<const void *>(mixsys_kernel<SYS, CELLS, true>), MixSysKernel<SYS, CELLS>::smem_bytes(),
                       2 * CELLS};
}
template <int SYS>
MixSysEntry mixsys_entry_sys(int cells) { return cells == 64 ? mixsys_entry_of<SYS, 64>() : mixsys_entry_of<SYS, 128>(); }
MixSysEntry mixsys_entry(int sys, int cells)
{
    return sys == SYS_BN ? mixsys_entry_sys<SYS_BN>(cells) : mixsys_entry_sys<SYS_EULER>(cells);
}
cudaError_t mixsys_configure(const MixSysEntry &e)
{
    cudaError_t r = cudaFuncSetAttribute(e.single, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(e.slab, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(e.batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
    return r;
}
}  // namespace

size_t mixsys_smem_bytes(int sys, int cells) { return mixsys_entry(sys, cells).smem; }

int mixsys_blocks_per_sm(int sys, int cells, bool batch)
{
    const MixSysEntry e = mixsys_entry(sys, cells);
    int nb = 0;
    if (mixsys_configure(e) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch ? e.batch : e.single, e.threads, e.smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_mixsys(int sys, int cells, const MixedMaps &maps, const MixedParams &p, cudaStream_t s)
{
    const MixSysEntry e = mixsys_entry(sys, cells);
    MixedMaps mm = maps;
    MixedParams pp = p;
    void *args[] = {&mm, &pp};
    const unsigned gy = (unsigned)(p.run_count > 0 ? p.run_count : p.runs);
    return cudaLaunchKernel(p.row_off ? e.slab : e.single, dim3((unsigned)p.strips, gy, 1), dim3((unsigned)e.threads, 1, 1), args,
                            e.smem, s);
}

cudaError_t launch_mixsys_batch(int sys, int cells, const MixedParams *inst, const MixedMaps *maps, const int2 *work, int *sched,
                                int blocks, cudaStream_t s)
{
    const MixSysEntry e = mixsys_entry(sys, cells);
    void *args[] = {&inst, &maps, &work, &sched};
    return cudaLaunchKernel(e.batch, dim3((unsigned)blocks, 1, 1), dim3((unsigned)e.threads, 1, 1), args, e.smem, s);
}

}  // namespace hype
