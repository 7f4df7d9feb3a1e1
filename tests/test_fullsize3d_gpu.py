"""The 3D step at the benchmark's full size (256^3), checked through properties
that do not depend on the size, and against the reference's own FP64 step.

* energy budget of one RK4/CN step (FP64): the dealiased nonlinear term moves
  energy between modes without changing the total, so the change of
  E = sum |w|^2/k^2 over a step is the viscous loss -nu dt (Z0 + Z1) (the
  trapezoid of dE/dt = -2 nu Z), to 1e-3 of the change;
* the vorticity stays divergence-free (k . w = 0 to round-off, FP64);
* translation equivariance: stepping a state shifted by a grid translation
  equals shifting the stepped state (FP64 to 1e-12, FP32 to 2e-5, relative L2);
* FP32 engine against the FP64 engine over 10 steps of the benchmark workload
  (relative L2 <= 1e-5);
* the FP64 and FP32 Boussinesq drop-ins against the reference's FP64
  timestep_cuda_ (built from its sources for sm_100a) over 2 steps, with the
  parity tolerances of the small-grid fixtures (1e-10 and 2e-5, max-norm).
"""
import os

import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.abi import TimestepLibrary
from psgpu_b200.fields import Grid3D, taylor_green3d
from tests.golden_cases import relerr

pytestmark = pytest.mark.gpu

N, NU, DT = 256, 1 / 1600, 1e-3
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_bous3d.so")


def _run(comps, precision, nsteps, scheme=P.SCHEME_NS_RK4):
    e = P.NS3D(N, scheme, precision=precision, nu=NU)
    try:
        e.upload(*comps)
        before = e.energetics()
        e.step(DT, nsteps)
        after = e.energetics()
        return np.stack(e.download()), before, after
    finally:
        e.close()


def _rel2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_energy_budget_and_divergence_fp64():
    comps = taylor_green3d(N, 11, amp=0.3)
    w, (E0, Z0, _), (E1, Z1, _) = _run(comps, 64, 1)
    dE = E1 - E0
    assert dE < 0
    assert abs(dE + NU * DT * (Z0 + Z1)) <= 1e-3 * abs(dE)
    kx, ky, kz = Grid3D(N).wavenumbers()
    div = np.abs(kx * w[0] + ky * w[1] + kz * w[2])
    kmag = np.sqrt(kx * kx + ky * ky + kz * kz)
    assert div.max() <= 1e-12 * float(np.max(kmag * np.sqrt(np.sum(np.abs(w) ** 2, axis=0))))


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-5)])
def test_translation_equivariance(precision, tol):
    g = Grid3D(N)
    kx, ky, kz = g.wavenumbers()
    s = 2 * np.pi / N * np.array([5.0, 17.0, 101.0])
    ph = np.exp(-1j * (kx * s[0] + ky * s[1] + kz * s[2])) * g.mask()
    comps = taylor_green3d(N, 12, amp=0.3)
    shifted = [c * ph for c in comps]
    a, _, _ = _run(comps, precision, 3)
    b, _, _ = _run(shifted, precision, 3)
    assert _rel2(b, a * ph) <= tol


def test_fp32_against_fp64_on_the_benchmark_workload():
    comps = taylor_green3d(N, 1234, amp=1e-3)
    w64, _, _ = _run(comps, 64, 10)
    w32, _, _ = _run(comps, 32, 10)
    assert _rel2(w32, w64) <= 1e-5


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build not present")
@pytest.mark.parametrize("precision,tol", [(64, 1e-10), (32, 2e-5)])
def test_boussinesq_dropin_against_reference(precision, tol, monkeypatch):
    xi, et, zt = taylor_green3d(N, 1234, amp=1e-3)
    rho = 1e-2 * taylor_green3d(N, 77, amp=1.0)[2]
    ref = TimestepLibrary(REF, "bous3d").bous3d(xi, et, zt, rho, N, NU, DT, 2 * DT, ri=1.0,
                                                 sc=1.0, theta=np.pi / 2)
    monkeypatch.setenv("PSG_PRECISION", str(precision))
    P.lib()
    ours = TimestepLibrary(P.dropin_path("bous3d"), "bous3d").bous3d(
        xi, et, zt, rho, N, NU, DT, 2 * DT, ri=1.0, sc=1.0, theta=np.pi / 2)
    for a, b in zip(ours[:4], ref[:4]):
        assert relerr(a, b) < tol
    assert ours[4] == pytest.approx(ref[4], rel=1e-14)
