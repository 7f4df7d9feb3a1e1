"""Every x-pass schedule the autotuner can pick (PSG_XPASS_VARIANT pins one;
a variant that does not fit the device at that size is skipped) gives the
same step as variant 1, for the RK4/CN and the Heun/CN (with the physical
vorticity it keeps) schemes and the Boussinesq RK4/CN scheme (nine fields
through the x-pass): 1e-12 in FP64, 2e-6 in FP32 (max-norm relative).  The
FP32 variants 4-7 and 12, 14 transform two lines per packed f32x2
instruction (their products round in another order: 2e-6 holds them too);
variants 8-14 (even) run blocks of half the rows."""
import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.fields import random_vorticity3d

pytestmark = pytest.mark.gpu

TOL = {64: 1e-12, 32: 2e-6}


def _run(monkeypatch, v, n, scheme, prec):
    monkeypatch.setenv("PSG_XPASS_VARIANT", str(v))
    bous = scheme == P.SCHEME_BOUS_RK4
    kw = dict(ri=1.0, sc=1.0, theta=np.pi / 2) if bous else {}
    e = P.NS3D(n, scheme, precision=prec, nu=0.01, ampfor=-1.0, kf=4.0, **kw)
    if e.autotune(rerun=False)[0] != v:
        return None, None  # the variant does not fit: the pin is not taken
    comps = list(random_vorticity3d(n, 12))
    if bous:
        comps.append(random_vorticity3d(n, 13)[0])
    e.upload(*comps)
    e.step(2e-3, 3, dump_last=(scheme == P.SCHEME_NS_HEUN))
    st = np.stack(e.download())
    ph = e.physical() if scheme == P.SCHEME_NS_HEUN else None
    return st, ph


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("scheme", [P.SCHEME_NS_RK4, P.SCHEME_NS_HEUN, P.SCHEME_BOUS_RK4])
@pytest.mark.parametrize("n", [32, 64])
def test_xpass_variants_agree(monkeypatch, prec, scheme, n):
    ref, ref_ph = _run(monkeypatch, 1, n, scheme, prec)
    assert ref is not None
    for v in (0, 2, 3, 4, 5, 6, 7, 8, 10, 12, 14):
        st, ph = _run(monkeypatch, v, n, scheme, prec)
        if st is None:
            continue
        assert _rel(st, ref) < TOL[prec], v
        if ph is not None:
            assert _rel(ph, ref_ph) < TOL[prec], v
