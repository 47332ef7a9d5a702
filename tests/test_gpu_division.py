"""The kernels divide by constants (3, 6, 12, 36, W) and by per-cell values
(rho, |grad C|, tau) with an FMA correction of q = a*RN(1/b) (Markstein's
theorem) instead of the IEEE division the reference uses. The results must
be bit-identical to IEEE division: checked on the device on 2^27 random
operands per divisor spread over the binades [2^-1000, 2^1000]."""
import ctypes as ct

import pytest

import amrlbm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("divisor", [3.0, 6.0, 12.0, 36.0, 5.0, 4.0, 0.0])
def test_division_matches_ieee(divisor):
    lib = amrlbm.load_library()
    bad = ct.c_uint64(123)
    assert lib.amrlbm_selftest_division(1 << 27, 20261203 + int(divisor), divisor,
                                        ct.byref(bad)) == 0
    assert bad.value == 0, f"{bad.value} results differ from IEEE division by {divisor}"
