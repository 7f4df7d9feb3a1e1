"""Device energetics and device-pointer state transfer of the 3D engine.

The FP64 sums of the engine (energy = sum |w|^2/k^2, enstrophy = sum |w|^2 over
the kept modes, as the reference's computeStats forms them) against the
oracle's energy and a numpy enstrophy of the same downloaded state; tolerance
1e-12 relative for the FP64 engine and 1e-6 for FP32 (storage rounding only).
"""
import numpy as np
import pytest
import torch

import psgpu_b200 as P
from oracle import pyoracle as O
from psgpu_b200.fields import Grid3D, random_vorticity3d, taylor_green3d

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 1e-6)])
def test_energetics_matches_oracle(precision, tol):
    n = 32
    xi, et, zt = random_vorticity3d(n, 7)
    eng = P.NS3D(n, P.SCHEME_NS_RK4, precision=precision, nu=0.01)
    eng.upload(xi, et, zt)
    eng.step(1e-3, 3)
    a, b, c = eng.download()
    e, z, r = eng.energetics()
    g = Grid3D(n)
    z_np = float(sum(np.sum(np.abs(v[g.mask()]) ** 2) for v in (a, b, c)))
    assert e == pytest.approx(O.energy3d(a, b, c, n), rel=tol)
    assert z == pytest.approx(z_np, rel=tol)
    assert r == 0.0


def test_energetics_density_component():
    n = 16
    xi, et, zt = random_vorticity3d(n, 3)
    rho = random_vorticity3d(n, 4)[0]
    eng = P.NS3D(n, P.SCHEME_BOUS_RK4, precision=64, nu=0.01, ri=1.0, sc=1.0)
    eng.upload(xi, et, zt, rho)
    g = Grid3D(n)
    _, _, r = eng.energetics()
    assert r == pytest.approx(float(np.sum(np.abs(rho[g.mask()]) ** 2)), rel=1e-12)


@pytest.mark.parametrize("precision", [64, 32])
def test_device_upload_download_round_trip(precision):
    n = 32
    xi, et, zt = taylor_green3d(n, 11, amp=1e-2)
    g = Grid3D(n)
    src = [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in (xi, et, zt)]
    dst = [torch.zeros(g.shape, dtype=torch.complex128, device="cuda") for _ in range(3)]
    eng = P.NS3D(n, P.SCHEME_NS_RK4, precision=precision, nu=1e-3)
    eng.upload_device([t.data_ptr() for t in src])
    eng.step(1e-3, 2)
    eng.download_device([t.data_ptr() for t in dst])
    eng.sync()
    host = P.NS3D(n, P.SCHEME_NS_RK4, precision=precision, nu=1e-3)
    host.upload(xi, et, zt)
    host.step(1e-3, 2)
    ref = host.download()
    for d, r in zip(dst, ref):
        np.testing.assert_array_equal(d.cpu().numpy(), r)
