// hype_mixed_common.cuh -- FP32 pieces shared by the mixed-precision stage
// tiles (hype_stage_mixed.cu: Kapila; hype_stage_mixed_sys.cu: Baer-Nunziato
// and Euler): the WENO3 reconstruction of reconstruction.c:144-221 on
// deviations from the cell value, and minmod.
#pragma once
#include <cuda_runtime.h>
#include "hype_physics.cuh"

namespace hype {

__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

// One direction of WENO3 (reconstruction.c:157-178) on deviations from the
// cell value, weights gamma_k / (IS_k + eps)^4 scaled by min_k (IS_k + eps)^4.
__device__ __forceinline__ void weno3_1d_f(float dm2, float dm1, float dp1, float dp2, float &slope, float &curv)
{
    const float ux0 = -2.0f * dm1 + 0.5f * dm2, uxx0 = 0.5f * (dm2 - 2.0f * dm1);
    const float ux1 = 0.5f * (dp1 - dm1), uxx1 = 0.5f * (dm1 + dp1);
    const float ux2 = 2.0f * dp1 - 0.5f * dp2, uxx2 = 0.5f * (dp2 - 2.0f * dp1);
    const float r13 = 13.0f / 3.0f, eps = 1.0e-12f;
    const float a0 = ux0 * ux0 + r13 * uxx0 * uxx0 + eps;
    const float a1 = ux1 * ux1 + r13 * uxx1 * uxx1 + eps;
    const float a2 = ux2 * ux2 + r13 * uxx2 * uxx2 + eps;
    const float mn = fminf(a0, fminf(a1, a2));
    float q0 = fdiv(mn, a0), q1 = fdiv(mn, a1), q2 = fdiv(mn, a2);
    q0 *= q0; q1 *= q1; q2 *= q2;
    const float w0 = q0 * q0, w1 = 100.0f * (q1 * q1), w2 = q2 * q2;
    const float inv = fdiv(1.0f, w0 + w1 + w2);
    slope = (w0 * ux0 + w1 * ux1 + w2 * ux2) * inv;
    curv = (w0 * uxx0 + w1 * uxx1 + w2 * uxx2) * inv;
}

// reconstruction.c:144-221 on deviations (u_0 = 0): coefficients k = 1..5
__device__ __forceinline__ void weno3_f(const float *d, float *c)
{
    // d: xm2 xm1 xp1 xp2 ym2 ym1 yp1 yp2 pp pm mp mm
    weno3_1d_f(d[0], d[1], d[2], d[3], c[0], c[2]);
    weno3_1d_f(d[4], d[5], d[6], d[7], c[1], c[3]);
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
