"""The line-FFT building block of every pass (psg_fft.cuh) against numpy."""
import ctypes as C

import numpy as np
import pytest

import psgpu_b200 as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512])
@pytest.mark.parametrize("sign", [-1, 1])
@pytest.mark.parametrize("swap", [0, 1])
def test_linefft(n, sign, swap):
    L = P.lib()
    rng = np.random.default_rng(n)
    lines = 37
    x = (rng.standard_normal((lines, n)) + 1j * rng.standard_normal((lines, n))).astype(np.complex128)
    y = np.zeros_like(x)
    dp = C.POINTER(C.c_double)
    rc = L.psg_debug_linefft(n, sign, swap, x.ctypes.data_as(dp), y.ctypes.data_as(dp), lines)
    assert rc == 0, L.psg_last_error()
    ref = np.fft.fft(x, axis=1) if sign < 0 else np.fft.ifft(x, axis=1) * n
    assert np.abs(y - ref).max() / np.abs(ref).max() < 1e-14
