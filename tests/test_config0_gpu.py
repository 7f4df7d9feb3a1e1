"""The 2D Kolmogorov case as specified, and its energy budget.

Workload: [0, 2 pi]^2, 128^2, forcing sin(4y) (the reference's -2 at
(kx, ky) = (0, +-4), 2D_NavierStokes/src_RK4/kernels.h:264-266), nu = 1/40,
RK4 with the final Crank-Nicolson viscous factor, 2/3 dealias, dt = 0.005,
2000 steps, FP64; seeded initial vorticity on 1 <= |k| <= 8 with amplitude
~ 1/|k| and enstrophy 1.

* Parity: this package's 2D drop-in (libpsg_ns2d.so, no PSG_PRECISION set, so
  FP64) against the reference's own 2D timestep_cuda_ built from its sources
  (oracle/_ref/libref_ns2d.so), one 2000-step call each on the same initial
  state: max-norm relative error <= 1e-9 (FP64 round-off grown over 10 time
  units of chaotic flow).
* Energy budget in the reference's output conventions
  (2D_NavierStokes/src_RK4/src_gmres/out.F90:20-34): E = sum_LL |w|^2/k^2,
  enstrophy V = 2 sum_LL |w|^2, D = nu V, I = -Re w(0, kf)/kf.  The dealiased
  nonlinear term conserves E, so dE/dt = I - D; the central difference of E
  over two steps matches I - D to 1e-4 of D at dt = 0.005, and to second order
  in dt (the mismatch at dt/2 is a quarter of that at dt; the oracle gives
  5.4e-6 and 1.4e-6 at t = 2).
"""
import os

import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.abi import TimestepLibrary
from psgpu_b200.fields import Grid2D, kolmogorov_ic2d
from tests.golden_cases import relerr

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_ns2d.so")
N, NU, DT, STEPS, KF = 128, 1.0 / 40.0, 0.005, 2000, 4


def test_config0_2000_fp64_steps_against_the_reference(monkeypatch):
    if not os.path.exists(REF):
        pytest.skip("reference 2D step not built (oracle/build_ref.sh)")
    monkeypatch.delenv("PSG_PRECISION", raising=False)
    Z0 = kolmogorov_ic2d(N, 77)
    ours, t_ours = TimestepLibrary(P.dropin_path("ns2d"), "ns2d").ns2d(Z0, N, NU, DT, STEPS)
    ref, t_ref = TimestepLibrary(REF, "ns2d").ns2d(Z0, N, NU, DT, STEPS)
    assert np.isfinite(ours).all()
    assert relerr(ours, ref) < 1e-9
    assert t_ours == pytest.approx(t_ref, rel=1e-14)


def _budget(Z, n, nu, kf=KF):
    g = Grid2D(n)
    kx, ky = g.wavenumbers()
    keep = g.mask()
    wk = kx * kx + ky * ky
    vz = np.abs(Z) ** 2
    E = float(np.sum(vz[keep] / wk[keep]))
    V = 2.0 * float(np.sum(vz[keep]))
    D = V * nu
    iky = kf + g.kt  # row of ky = kf
    I = -float(np.real(Z[iky, 0])) / kf
    return E, D, I


def _mismatch(dt, t0=5.0):
    """|dE/dt - (I - D)| / D at t0, dE/dt from E at t0 -+ dt"""
    b = P.Batch2D([N], precision=64)
    b.upload(0, kolmogorov_ic2d(N, 78))
    m = int(round(t0 / dt))
    b.run(NU, dt, m - 1)
    Za = b.download(0)
    b.run(NU, dt, 1)
    Zm = b.download(0)
    b.run(NU, dt, 1)
    Zb = b.download(0)
    b.close()
    Ea, _, _ = _budget(Za, N, NU)
    Eb, _, _ = _budget(Zb, N, NU)
    _, D, I = _budget(Zm, N, NU)
    dEdt = (Eb - Ea) / (2 * dt)
    return abs(dEdt - (I - D)) / D, D, I


def test_forced_energy_budget_closes_to_second_order():
    e1, D, I = _mismatch(DT)
    e2, _, _ = _mismatch(DT / 2)
    assert D > 0 and abs(I) > 0
    assert e1 < 1e-4, e1
    # second order in dt: halving dt cuts the mismatch about fourfold
    assert e2 < 0.4 * e1 or e2 < 1e-9, (e1, e2)
