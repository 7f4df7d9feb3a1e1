"""Failure detection without a GPU fault: a bounded device wait that cannot
succeed runs out, the kernel leaves PSG_DEVICE_TIMEOUT in its status word and
returns, the host reads it, and the context stays usable (a step afterwards
gives the same result as on a fresh engine)."""
import ctypes

import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.fields import random_vorticity3d

pytestmark = pytest.mark.gpu

PSG_DEVICE_TIMEOUT = 0x7E01


def test_bounded_wait_reports_timeout_and_context_survives():
    L = P.lib()
    L.psg_debug_wait_timeout.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    st = ctypes.c_int(-1)
    assert L.psg_debug_wait_timeout(1000, ctypes.byref(st)) == 0
    assert st.value == PSG_DEVICE_TIMEOUT
    # the context is intact: an engine steps as it does on a fresh context
    xi, et, zt = random_vorticity3d(16, 4)
    a = P.NS3D(16, P.SCHEME_NS_RK4, precision=64, nu=0.02)
    a.upload(xi, et, zt)
    a.step(1e-3, 3)
    a.sync()
    r1 = a.download()
    b = P.NS3D(16, P.SCHEME_NS_RK4, precision=64, nu=0.02)
    b.upload(xi, et, zt)
    b.step(1e-3, 3)
    for x, y in zip(r1, b.download()):
        np.testing.assert_array_equal(x, y)


def test_bad_arguments_are_refused_on_the_host():
    L = P.lib()
    L.psg_debug_wait_timeout.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    st = ctypes.c_int(0)
    assert L.psg_debug_wait_timeout(0, ctypes.byref(st)) != 0
    assert b"bad arguments" in L.psg_last_error()
