"""The branch-free correctly rounded FP64 division of the bit-exact
Baer-Nunziato reconstruction (csrc/hype_div.cuh) against IEEE division.

Per seed 2^30 operand pairs on the GPU (hype_test_division): raw bit patterns
(zeros, subnormals, infinities, NaNs), operands of every exponent, quotients
next to a midpoint of two doubles (the hard rounding cases) and divisors with
an all-ones significand.  Wherever the function reports its operands in range
its result must be the IEEE quotient bit for bit; out of range its caller
divides with IEEE division instead (Recon<2>), so bit-exactness of the kernels
rests on this test together with the parity tests.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 0x9E3779B97F4A7C15])
def test_branch_free_division_equals_ieee(hp, seed):
    n = 1 << 30
    mism, spec = ctypes.c_longlong(-1), ctypes.c_longlong(-1)
    assert hp.lib().hype_test_division(0, n, seed, ctypes.byref(mism), ctypes.byref(spec)) == hp.OK
    print("pairs", n, "mismatches", mism.value, "out of range", spec.value)
    assert mism.value == 0
    # the raw-bit and wide-exponent quarters fall partly outside the range; most pairs do not
    assert 0 < spec.value < n // 2
