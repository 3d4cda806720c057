// hype_mixed_common.cuh -- FP32 pieces shared by the mixed-precision stage
// tiles (hype_stage_mixed.cu: Kapila; hype_stage_mixed_sys.cu: Baer-Nunziato
// and Euler): the WENO3 reconstruction of reconstruction.c:144-221 on
// deviations from the cell value, and minmod.
#pragma once
#include <cuda_runtime.h>
#include "hype_physics.cuh"

namespace hype {

__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

// One direction of WENO3 (reconstruction.c:157-178) on deviations from the cell
// value, weights gamma_k / (IS_k + eps)^4 scaled by min_k (IS_k + eps)^4: slope and
// curvature from the deviations at -2, -1, +1, +2.  The x and the y direction run at
// once as the two lanes of packed FP32 operations (sm_100 f32x2: lane .x the x
// direction, lane .y the y direction), half the FP32 instructions of two scalar
// passes; minima and the fast reciprocals stay per lane.
__device__ __forceinline__ void weno3_xy_f2(float2 dm2, float2 dm1, float2 dp1, float2 dp2, float2 &slope, float2 &curv)
{
    const float2 k2 = make_float2(2.0f, 2.0f), km2 = make_float2(-2.0f, -2.0f), kh = make_float2(0.5f, 0.5f);
    const float2 kmh = make_float2(-0.5f, -0.5f), k13 = make_float2(13.0f / 3.0f, 13.0f / 3.0f);
    const float2 keps = make_float2(1.0e-12f, 1.0e-12f), k100 = make_float2(100.0f, 100.0f);
    const float2 ux0 = __ffma2_rn(km2, dm1, __fmul2_rn(kh, dm2));
    const float2 uxx0 = __fmul2_rn(kh, __ffma2_rn(km2, dm1, dm2));
    const float2 ux1 = __fmul2_rn(kh, __ffma2_rn(make_float2(-1.0f, -1.0f), dm1, dp1));
    const float2 uxx1 = __fmul2_rn(kh, __fadd2_rn(dm1, dp1));
    const float2 ux2 = __ffma2_rn(k2, dp1, __fmul2_rn(kmh, dp2));
    const float2 uxx2 = __fmul2_rn(kh, __ffma2_rn(km2, dp1, dp2));
    const float2 a0 = __ffma2_rn(ux0, ux0, __ffma2_rn(__fmul2_rn(k13, uxx0), uxx0, keps));
    const float2 a1 = __ffma2_rn(ux1, ux1, __ffma2_rn(__fmul2_rn(k13, uxx1), uxx1, keps));
    const float2 a2 = __ffma2_rn(ux2, ux2, __ffma2_rn(__fmul2_rn(k13, uxx2), uxx2, keps));
    const float2 mn = make_float2(fminf(a0.x, fminf(a1.x, a2.x)), fminf(a0.y, fminf(a1.y, a2.y)));
    auto rcp2 = [](float2 v) { return make_float2(__fdividef(1.0f, v.x), __fdividef(1.0f, v.y)); };   // fast reciprocals
    float2 q0 = __fmul2_rn(mn, rcp2(a0));
    float2 q1 = __fmul2_rn(mn, rcp2(a1));
    float2 q2 = __fmul2_rn(mn, rcp2(a2));
    q0 = __fmul2_rn(q0, q0); q1 = __fmul2_rn(q1, q1); q2 = __fmul2_rn(q2, q2);
    const float2 w0 = __fmul2_rn(q0, q0), w1 = __fmul2_rn(k100, __fmul2_rn(q1, q1)), w2 = __fmul2_rn(q2, q2);
    const float2 sum = __fadd2_rn(__fadd2_rn(w0, w1), w2);
    const float2 inv = rcp2(sum);
    slope = __fmul2_rn(__ffma2_rn(w2, ux2, __ffma2_rn(w1, ux1, __fmul2_rn(w0, ux0))), inv);
    curv = __fmul2_rn(__ffma2_rn(w2, uxx2, __ffma2_rn(w1, uxx1, __fmul2_rn(w0, uxx0))), inv);
}

// reconstruction.c:144-221 on deviations (u_0 = 0): coefficients k = 1..5
__device__ __forceinline__ void weno3_f(const float *d, float *c)
{
    // d: xm2 xm1 xp1 xp2 ym2 ym1 yp1 yp2 pp pm mp mm
    float2 sl, cu;
    weno3_xy_f2(make_float2(d[0], d[4]), make_float2(d[1], d[5]), make_float2(d[2], d[6]), make_float2(d[3], d[7]), sl, cu);
    c[0] = sl.x; c[1] = sl.y; c[2] = cu.x; c[3] = cu.y;
    const float c1 = c[0], c2 = c[1], c3 = c[2], c4 = c[3];
    const float x0 = d[8] - c1 - c2 - c3 - c4;
    const float x1 = -d[9] + c1 - c2 + c3 + c4;
    const float x2 = -d[10] - c1 + c2 + c3 + c4;
    const float x3 = d[11] + c1 + c2 - c3 - c4;
    const float tmp = 4.0f * (c3 * c3 + c4 * c4) + 1.0e-12f;
    const float a0 = tmp + x0 * x0, a1 = tmp + x1 * x1, a2 = tmp + x2 * x2, a3 = tmp + x3 * x3;
    const float mn = fminf(fminf(a0, a1), fminf(a2, a3));
    float q0 = fdiv(mn, a0), q1 = fdiv(mn, a1), q2 = fdiv(mn, a2), q3 = fdiv(mn, a3);
    q0 *= q0; q1 *= q1; q2 *= q2; q3 *= q3;
    const float w0 = q0 * q0, w1 = q1 * q1, w2 = q2 * q2, w3 = q3 * q3;
    c[4] = (w0 * x0 + w1 * x1 + w2 * x2 + w3 * x3) * fdiv(1.0f, w0 + w1 + w2 + w3);
}

// sum over k = 1..5 of cf(k-1) phi(k) for the two halves of a thread pair: half 0
// takes the basis values of B0, half 1 those of B1 (PhiFace, PhiNode, PhiVol,
// DPhiVolX, DPhiVolY of Quad<2>).  A term whose basis value is below 1e-9 in both
// halves is dropped (y^2 - 1/12 at y = +-1/(2 sqrt 3) and the like: below FP32
// resolution of the sum), and a value both halves share needs no selection.
constexpr double cabs_c(double x) { return x < 0.0 ? -x : x; }
template <class B0, class B1, class CF>
__device__ __forceinline__ float pair_poly(CF cf, int h)
{
    float v = 0.0f;
    static_for<5>([&](auto kk) {
        constexpr int k = decltype(kk)::value + 1;
        constexpr double a0 = B0::template at<k>(), a1 = B1::template at<k>();
        if constexpr (cabs_c(a0) < 1e-9 && cabs_c(a1) < 1e-9) {
        } else if constexpr (a0 == a1) {
            v += cf(k - 1) * (float)a0;
        } else {
            v += cf(k - 1) * (h ? (float)a1 : (float)a0);
        }
    });
    return v;
}

__device__ __forceinline__ float minmod_f(float a, float b)
{
    if (a * b < 0.0f) return 0.0f;
    return (fabsf(a) < fabsf(b)) ? a : b;
}

}  // namespace hype
