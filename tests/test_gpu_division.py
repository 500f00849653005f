"""The kernels divide a 3-vector by one divisor through one correctly rounded reciprocal and an exact FMA remainder
(Markstein's theorem) instead of three divisions; the result must be bit-identical to the correctly rounded division
for every operand (2^28 random triples over all finite bit patterns plus cloth-like operands)."""
import ctypes as C

import pytest

from bevy_xpbd_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 0xC0FFEE])
def test_shared_reciprocal_division_is_correctly_rounded(seed):
    L = N.load()
    bad = C.c_uint64(123)
    assert L.xpbd_selftest_division(0, 1 << 28, seed, C.byref(bad)) == 0
    assert bad.value == 0
