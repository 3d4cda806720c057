// hype_div.cuh -- IEEE round-to-nearest-even FP64 division a / b as a straight
// line of fused multiply-adds, for the bit-exact kernels.
//
// The compiler's division ends in a branch to its own slow path, which keeps
// independent divisions from overlapping; this one has no branch, so the WENO
// weights of a reconstruction (reconstruction.c:163-170, 186-193, 207-215)
// issue as interleaved chains.  Method (Markstein's Newton-Raphson division,
// IBM J. Res. Dev. 34 (1990); P. Markstein, "IA-64 and Elementary Functions",
// 2000, ch. 8; the exact-remainder property in J.-M. Muller et al., "Handbook
// of Floating-Point Arithmetic", 2010, sec. 4.3):
//   y  ~ 1/b: the hardware approximation (PTX rcp.approx.ftz.f64), two
//            Newton-Raphson steps y += y (1 - b y);
//   q0 = a y, r0 = a - b q0 (fma), q1 = q0 + r0 y (fma): |q1 - a/b| < 1 ulp;
//   r1 = a - b q1 is then exact (fma), and so is rn = a - b qn for the
//   neighbour qn of q1 on the side of a/b (the sign of r1 / b); the quotient
//   is whichever of q1, qn leaves the smaller |remainder|.  A tie would need
//   a/b to be a midpoint of two doubles, impossible for a quotient of doubles
//   that is not exact.
// Valid while a, b, the quotient and the remainders are normal numbers: the
// operands' and the quotient's binary exponents in [-900, 1000] (b: [-1000,
// 1000]), or a = 0.  Outside that `special` is set and the caller recomputes
// with the compiler's division.  tests/test_gpu_division.py compares it with
// IEEE division on 2^30 operand pairs per run (hype_test_division).
#pragma once
#include <cuda_runtime.h>

namespace hype {

__device__ __forceinline__ unsigned biased_exp(double x) { return (unsigned)((__double_as_longlong(x) >> 52) & 0x7ff); }

// a / b for operands the caller has checked: a, b, a / b nonzero, finite, with
// binary exponents in [-900, 1000]
__device__ __forceinline__ double cr_div_core(double a, double b)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    double e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    double q = a * y;
    double r = fma(-b, q, a);
    q = fma(r, y, q);
    r = fma(-b, q, a);   // exact
    const bool up = (r > 0.0) == (b > 0.0);
    const long long qi = __double_as_longlong(q);
    const double qn = __longlong_as_double(qi + ((up == (q >= 0.0)) ? 1LL : -1LL));
    const double rn = fma(-b, qn, a);   // exact
    return (fabs(rn) < fabs(r)) ? qn : q;
}

// a / b for any operands; `special` is set where they are outside the range above
__device__ __forceinline__ double cr_div(double a, double b, bool &special)
{
    const double q = cr_div_core(a, b);
    const unsigned eb = biased_exp(b), ea = biased_exp(a), eq = biased_exp(q);
    const bool ok_b = eb >= 1023u - 1000u && eb <= 1023u + 1000u;
    const bool ok_a = ea >= 1023u - 900u && ea <= 1023u + 1000u && eq >= 1023u - 900u && eq <= 1023u + 1000u;
    special |= !(ok_b && (a == 0.0 || ok_a));
    return (a == 0.0) ? a * copysign(1.0, b) : q;   // a signed zero keeps the IEEE sign
}

}  // namespace hype
