/*
 * flops.cpp -- TEST INFRASTRUCTURE ONLY.  The oracle (hype_oracle.c) compiled
 * as C++ with every `double` replaced by a counting type, to count the
 * floating-point operations of one RHS evaluation: the algorithmic FLOPs per
 * cell of HyPE-2D's RHSFunctionPrim / RHSFunction, which it follows operation
 * for operation.  Additions (and subtractions), multiplications, divisions and
 * square roots are counted separately; comparisons, absolute values, negations
 * and transcendental calls are counted apart from the FLOPs.  The values
 * computed are the oracle's own (the type wraps an IEEE double and rounds every
 * operation on its own, as -ffp-contract=off does).
 *
 * Built by `make -C oracle flops` into _build/libhype_oracle_flops.so; it
 * exports the oracle's C API plus hyo_flops_reset / hyo_flops_read.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

namespace flopcount {
enum { ADD = 0, MUL = 1, DIV = 2, SQRT = 3, CMP = 4, ABS = 5, NEG = 6, TRANS = 7, NCOUNT = 8 };
static unsigned long long count[NCOUNT];

struct fd {
    double v;
    fd() = default;
    fd(double x) : v(x) {}
    explicit operator double() const { return v; }
};
static_assert(sizeof(fd) == sizeof(double), "fd must have the layout of a double");

inline fd operator+(fd a, fd b) { ++count[ADD]; return fd(a.v + b.v); }
inline fd operator-(fd a, fd b) { ++count[ADD]; return fd(a.v - b.v); }
inline fd operator*(fd a, fd b) { ++count[MUL]; return fd(a.v * b.v); }
inline fd operator/(fd a, fd b) { ++count[DIV]; return fd(a.v / b.v); }
inline fd operator-(fd a) { ++count[NEG]; return fd(-a.v); }
inline fd operator+(fd a) { return a; }
inline fd &operator+=(fd &a, fd b) { a = a + b; return a; }
inline fd &operator-=(fd &a, fd b) { a = a - b; return a; }
inline fd &operator*=(fd &a, fd b) { a = a * b; return a; }
inline fd &operator/=(fd &a, fd b) { a = a / b; return a; }
inline bool operator<(fd a, fd b) { ++count[CMP]; return a.v < b.v; }
inline bool operator>(fd a, fd b) { ++count[CMP]; return a.v > b.v; }
inline bool operator<=(fd a, fd b) { ++count[CMP]; return a.v <= b.v; }
inline bool operator>=(fd a, fd b) { ++count[CMP]; return a.v >= b.v; }
inline bool operator==(fd a, fd b) { ++count[CMP]; return a.v == b.v; }
inline bool operator!=(fd a, fd b) { ++count[CMP]; return a.v != b.v; }
inline fd sqrt(fd a) { ++count[SQRT]; return fd(::sqrt(a.v)); }
inline fd fabs(fd a) { ++count[ABS]; return fd(::fabs(a.v)); }
inline fd tanh(fd a) { ++count[TRANS]; return fd(::tanh(a.v)); }
}  // namespace flopcount

using flopcount::fd;
using flopcount::sqrt;
using flopcount::fabs;
using flopcount::tanh;

#define double fd
#include "hype_oracle.c"
#undef double

extern "C" {
__attribute__((visibility("default"))) void hyo_flops_reset(void)
{
    memset(flopcount::count, 0, sizeof(flopcount::count));
}
/* out[0..7]: add/sub, mul, div, sqrt, compare, abs, neg, transcendental */
__attribute__((visibility("default"))) void hyo_flops_read(unsigned long long *out)
{
    memcpy(out, flopcount::count, sizeof(flopcount::count));
}
}
