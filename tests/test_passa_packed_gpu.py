"""Pass A (z-inverse with the velocity formed in registers) on packed f32x2
transforms, two output fields per instruction, against the scalar kernel.

The packed kernel runs the same butterflies and twiddles on the pair of fields,
with its complex products in a fixed fused-multiply-add form, so the two agree
to FP32 rounding (not bit for bit).  Pinned by PSG_PASSA_PACKED at set-up:

* Navier-Stokes and Boussinesq RK4/CN FP32 engines, 64^3 and 32^3, 5 steps:
  relative L2 difference of the states <= 1e-6;
* the packed engine against the FP64 engine on the same input, within the
  FP32 parity tolerance of the fixtures (2e-5, max-norm relative);
* the autotuner reports the pinned choice, and FP64 engines never take it.
"""
import os

import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.fields import taylor_green3d

pytestmark = pytest.mark.gpu


def _run(pin, n, scheme, prec, steps=5):
    if pin is not None:
        os.environ["PSG_PASSA_PACKED"] = str(pin)
    try:
        e = P.NS3D(n, scheme, precision=prec, nu=1.0 / 400.0)
    finally:
        os.environ.pop("PSG_PASSA_PACKED", None)
    xi, et, zt = taylor_green3d(n, 3, amp=1e-2)
    comps = [xi, et, zt]
    if scheme == P.SCHEME_BOUS_RK4:
        e.set_params(1.0 / 400.0, ri=1.0)
        comps.append(0.1 * et)
    e.upload(*comps)
    e.step(2e-3, steps)
    out = np.stack(e.download())
    tun = e.pass_a_tuning()
    e.close()
    return out, tun


@pytest.mark.parametrize("scheme", [P.SCHEME_NS_RK4, P.SCHEME_BOUS_RK4])
@pytest.mark.parametrize("n", [32, 64])
def test_packed_pass_a_matches_scalar(scheme, n):
    a, ta = _run(1, n, scheme, 32)
    b, tb = _run(0, n, scheme, 32)
    assert ta[0] is True and tb[0] is False
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-6
    c, tc = _run(None, n, scheme, 64)
    assert tc[0] is False and tc[1] == (-1.0, -1.0)
    assert np.abs(a - c).max() / np.abs(c).max() <= 2e-5
