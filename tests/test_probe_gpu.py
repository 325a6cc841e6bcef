"""The texture-rate probe that the fast propagate kernel's roofline is quoted against."""
import ctypes as C

import pytest

from luvas3d import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [_lib.DTYPE_U8, _lib.DTYPE_F16, _lib.DTYPE_F32])
def test_texture_rate_is_measured(dtype):
    lib = _lib.load()
    rates = []
    for checker in (0, 1):
        r = C.c_double()
        _lib.check(lib.l3d_measure_texture_rate(dtype, checker, C.byref(r)))
        rates.append(r.value)
    # 148 SMs near 2 GHz: between 0.1 and 16 bilinear samples per SM per clock
    for r in rates:
        assert 148 * 1.0e9 * 0.1 < r < 148 * 2.0e9 * 16
