"""The Boussinesq DNS build's step (libpsg_bous3d_dns.so) against the
reference's own DNS build (3D_Boussinesq/src/cuda.cu, oracle/_ref/
libref_bous3d_dns.so) on the same inputs, through the same C ABI.

32^3, Re = 100, Ri = 1, Sc = 1, gravity along z (theta = pi/2), forcing on
zeta at (0, kf, 0), output every NOUT = 5 steps with statsFLAG = 1:
* adaptFLAG = 1 and Dtarget != 0: the CFL-adaptive step
  (3D_Boussinesq/src/out_low.h:11-16) and the forcing throttle
  (functions.h:364-368, cuda.cu:104-106) change the run, and both builds
  change it the same way: state to 1e-10 (max-norm relative), time to 1e-12;
* adaptFLAG = 0, Dtarget = 0: the plain DNS loop (steps while t <= Tstep);
* the run with both features differs from the plain one (they act).
TSTART = 1 keeps the reference from writing raw volumes at t = 0
(out_low.h:79-80 fires when t < dt).
"""
import os

import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.abi import TimestepLibrary
from psgpu_b200.fields import random_vorticity3d
from tests.golden_cases import relerr

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_bous3d_dns.so")
N, NU, DT, KF = 32, 0.01, 0.01, 1.0


def _state():
    xi, et, zt = random_vorticity3d(N, 21, solenoidal=True)
    rho = 0.1 * random_vorticity3d(N, 22)[0]
    return xi, et, zt, rho


def _run(lib, adapt, dtarget):
    xi, et, zt, rho = _state()
    return lib.bous3d_dns(xi, et, zt, rho, N, NU, DT, 1.0 + 40 * DT, ri=1.0, sc=1.0,
                          theta=np.pi / 2, ampfor=-0.5 * KF, kf=KF, dtarget=dtarget, adapt=adapt,
                          stats=1, nout=5, tstart=1.0, time0=1.0)


@pytest.mark.parametrize("adapt,dtarget", [(1, 0.05), (0, 0.0), (1, 0.0), (0, 0.05)])
def test_dns_build_matches_reference(adapt, dtarget, monkeypatch):
    if not os.path.exists(REF):
        pytest.skip("reference Boussinesq DNS build not built (oracle/build_ref.sh)")
    monkeypatch.delenv("PSG_PRECISION", raising=False)
    P.lib()
    ours = _run(TimestepLibrary(P.dropin_path("bous3d_dns"), "bous3d_dns"), adapt, dtarget)
    ref = _run(TimestepLibrary(REF, "bous3d_dns"), adapt, dtarget)
    for a, b, name in zip(ours[:4], ref[:4], ("xii", "eta", "zet", "rho")):
        assert np.isfinite(a).all()
        assert relerr(a, b) < 1e-10, name
    assert ours[4] == pytest.approx(ref[4], rel=1e-12)


def test_adaptive_step_and_throttle_act(monkeypatch):
    monkeypatch.delenv("PSG_PRECISION", raising=False)
    P.lib()
    lib = TimestepLibrary(P.dropin_path("bous3d_dns"), "bous3d_dns")
    plain = _run(lib, 0, 0.0)
    both = _run(lib, 1, 0.05)
    assert plain[4] != both[4]  # the step changed the time reached
    assert relerr(both[0], plain[0]) > 1e-6
