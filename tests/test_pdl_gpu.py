"""Programmatic dependent launch of the 3D passes.

Each pass of a right-hand side launches with the programmatic-serialisation
attribute after the pass before it (and pass A after the previous right-hand
side's pass E), and waits on the previous grid before its first global access.
The arithmetic is the same with and without it, so every scheme must give
bit-identical states in every PSG_PDL mode (1: every pass, 2: every pass but the
x-pass, the default) and with it off (0), over one call of several steps (the
steps chained) and over single-step calls, and the energetics reduction between
calls must see the finished state.  The set-up autotuner's choices (x-pass
variant, scalar or packed pass A) round differently, so the engines compared
here pin them.
"""
import os

import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.fields import taylor_green3d

pytestmark = pytest.mark.gpu


PINS = {"PSG_XPASS_VARIANT": "0", "PSG_PASSA_PACKED": "0"}


def _run(pdl, n, scheme, prec, calls):
    os.environ.update(PINS, PSG_PDL=str(pdl))
    try:
        e = P.NS3D(n, scheme, precision=prec, nu=1.0 / 400.0)
    finally:
        for k in list(PINS) + ["PSG_PDL"]:
            os.environ.pop(k, None)
    xi, et, zt = taylor_green3d(n, 7, amp=1e-2)
    comps = [xi, et, zt]
    if scheme == P.SCHEME_BOUS_RK4:
        e.set_params(1.0 / 400.0, ri=1.0)
        comps.append(0.1 * xi)
    e.upload(*comps)
    en = []
    for k in calls:
        e.step(2e-3, k)
        en.append(tuple(e.energetics()))
    out = e.download()
    e.close()
    return out, en


@pytest.mark.parametrize("scheme,prec,n", [
    (P.SCHEME_NS_RK4, 32, 64), (P.SCHEME_NS_RK4, 64, 32), (P.SCHEME_BOUS_RK4, 32, 64),
    (P.SCHEME_BOUS_RK4, 64, 32), (P.SCHEME_NS_HEUN, 32, 32), (P.SCHEME_EULER_HEUN, 64, 32)])
def test_pdl_steps_bit_identical(scheme, prec, n):
    calls = [3, 1, 1, 2]  # chained steps in one call, and steps in calls of their own
    b, eb = _run(0, n, scheme, prec, calls)
    assert all(np.isfinite(v).all() for v in b)
    for mode in (1, 2):
        a, ea = _run(mode, n, scheme, prec, calls)
        for x, y in zip(a, b):
            assert np.array_equal(x, y), mode
        assert ea == eb, mode
