"""The Newton-solver build's 3D step (18-argument timestep_cuda_, its own
forcing form) through libpsg_ns3d_newton.so.

* against the oracle's restatement at 32^3 with the forcing on (FP64 1e-10,
  FP32 2e-5, max-norm relative);
* the oracle pinned against the reference build itself (oracle/_ref, grid
  fixed at 128^3 by its kernels.h), 2 steps, and the drop-in against it too.
"""
import os

import numpy as np
import pytest

import psgpu_b200 as P
from oracle import pyoracle as O
from psgpu_b200.abi import TimestepLibrary
from psgpu_b200.fields import random_vorticity3d
from tests.golden_cases import relerr

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_ns3d_gmres.so")
TOL = {64: 1e-10, 32: 2e-5}
NU, DT, AMP, KF = 1.0 / 20.0, 0.01, -4.0, 4


@pytest.fixture(params=[64, 32], ids=["fp64", "fp32"])
def precision(request, monkeypatch):
    monkeypatch.setenv("PSG_PRECISION", str(request.param))
    return request.param


def test_dropin_matches_oracle(precision, monkeypatch):
    n = 32
    monkeypatch.setenv("PSG_NEWTON_N", str(n))
    P.lib()
    lib = TimestepLibrary(P.dropin_path("ns3d_newton"), "ns3d_newton")
    xi, et, zt = random_vorticity3d(n, 17)
    a, b, c, t = lib.ns3d_newton(xi, et, zt, n, NU, DT, 6, ampfor=AMP, kf=KF, tstart=0.5)
    ra, rb, rc, rt = O.ns3d_newton_timestep(xi, et, zt, n, NU, DT, 6, ampfor=AMP, kfy=KF,
                                            tstart=0.5)
    for x, r in ((a, ra), (b, rb), (c, rc)):
        assert relerr(x, r) < TOL[precision]
    assert t == pytest.approx(rt, rel=1e-14)


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build not present")
def test_oracle_and_dropin_match_reference_build(precision, monkeypatch):
    n = 128
    monkeypatch.setenv("PSG_NEWTON_N", str(n))
    xi, et, zt = random_vorticity3d(n, 5)
    ref = TimestepLibrary(REF, "ns3d_newton")
    sa, sb, sc, st = ref.ns3d_newton(xi, et, zt, n, NU, DT, 2, ampfor=AMP, kf=KF)
    oa, ob, oc, ot = O.ns3d_newton_timestep(xi, et, zt, n, NU, DT, 2, ampfor=AMP, kfy=KF)
    for x, r in ((oa, sa), (ob, sb), (oc, sc)):
        assert relerr(x, r) < 1e-12
    P.lib()
    lib = TimestepLibrary(P.dropin_path("ns3d_newton"), "ns3d_newton")
    a, b, c, t = lib.ns3d_newton(xi, et, zt, n, NU, DT, 2, ampfor=AMP, kf=KF)
    for x, r in ((a, sa), (b, sb), (c, sc)):
        assert relerr(x, r) < TOL[precision]
    assert t == pytest.approx(st, rel=1e-14)
