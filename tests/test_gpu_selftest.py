"""Device arithmetic the FP64 kernels rely on, checked bit for bit against
IEEE division on the GPU."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def test_division_by_known_constants(lib):
    bad = C.c_longlong(-1)
    assert lib.adc_selftest_div_const(1 << 30, 20261203, C.byref(bad)) == 0
    assert bad.value == 0, f"{bad.value} mismatches"
