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
* the run with both features differs from the plain one (they act);
* RecFLAG = 1: the recurrence search writes the same guesses to
  JOB0/UPO_ZK.out as the reference's build (3D_Boussinesq/src/
  functions.h:592-609) at a threshold the run crosses, and the run ends at
  the same state and time.  The flow there recurs: small internal gravity
  waves with horizontal wavevectors (|k| <= 1.5, kz = 0, gravity along z)
  at Ri = 100 oscillate at the buoyancy frequency N = 10 (period 0.63 > the
  check's 0.5 minimum) around a steady vortical part, unforced.
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


def _records(path, nkt):
    raw = np.fromfile(path, dtype=np.float64)
    rec = 7 + 8 * nkt
    assert raw.size % rec == 0
    return raw.reshape(-1, rec)


def test_recurrence_guesses_match_reference(monkeypatch, tmp_path):
    """RecFLAG = 1: at a threshold the run crosses, our DNS drop-in writes the
    same guesses to JOB0/UPO_ZK.out as the reference's DNS build (record
    layout of 3D_Boussinesq/src/functions.h:596-606: start time, v2, period,
    shifts, residual, four fields) and reaches the same final state and time.
    The reference's check reassigns the loop's time variable
    (functions.h:501), which adds NOUT steps to the run; the drop-in does the
    same."""
    if not os.path.exists(REF):
        pytest.skip("reference Boussinesq DNS build not built (oracle/build_ref.sh)")
    monkeypatch.delenv("PSG_PRECISION", raising=False)
    P.lib()
    ours_lib = TimestepLibrary(P.dropin_path("bous3d_dns"), "bous3d_dns")
    ref_lib = TimestepLibrary(REF, "bous3d_dns")
    g = P.Grid3D(N)
    nkt = g.nkt
    hz = g.wavenumbers()[2] == 0
    xi, et, zt = (0.05 * a * hz for a in random_vorticity3d(N, 21, kmin=0.5, kmax=1.5,
                                                             solenoidal=True))
    rho = 0.05 * random_vorticity3d(N, 22, kmin=0.5, kmax=1.5)[0] * hz
    kw = dict(ri=100.0, sc=1.0, theta=np.pi / 2, ampfor=0.0, kf=KF, stats=1, nout=2,
              tstart=1.0, time0=1.0, rec=1)
    tend = 1.0 + 200 * DT
    found = None
    for thr in (0.8, 0.5, 0.3, 0.2, 0.12, 0.08, 0.05, 0.03):
        wd = tmp_path / f"ours_{thr}"
        out = ours_lib.bous3d_dns(xi, et, zt, rho, N, NU, DT, tend, resthresh=thr,
                                  workdir=str(wd), **kw)
        r = _records(wd / "JOB0" / "UPO_ZK.out", nkt)
        lines = (wd / "JOB0" / "UPOinfo_ts.dat").read_text().splitlines()
        assert len(lines) == 1 + len(r)
        if len(r):
            found = (thr, r, out)
            break
    assert found is not None, "no threshold emitted a guess"
    thr, ours, out = found
    assert (ours[:, 6] < thr).all() and (ours[:, 2] >= 0.5 - 1e-12).all()
    wd = tmp_path / "ref"
    ref_out = ref_lib.bous3d_dns(xi, et, zt, rho, N, NU, DT, tend, resthresh=thr,
                                 workdir=str(wd), **kw)
    ref = _records(wd / "JOB0" / "UPO_ZK.out", nkt)
    assert ours.shape == ref.shape
    np.testing.assert_allclose(ours[:, :6], ref[:, :6], rtol=1e-12, atol=1e-12)  # time .. shift z
    np.testing.assert_allclose(ours[:, 6], ref[:, 6], rtol=1e-9)                # residual
    assert np.abs(ours[:, 7:] - ref[:, 7:]).max() <= 1e-10 * np.abs(ref[:, 7:]).max()
    for a, b in zip(out[:4], ref_out[:4]):
        assert relerr(a, b) < 1e-10
    assert out[4] == pytest.approx(ref_out[4], rel=1e-12)
