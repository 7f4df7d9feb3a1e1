"""Parity of the CUDA path with the reference.

Every golden fixture (made by the reference's own CUDA timestep_cuda_, FP64
cuFFT) is replayed through this package's drop-in library for the same
flavour, called through the reference's C ABI with the same arguments.

Tolerances (max-norm relative error over the state, against the reference):
  FP64 engine: 1e-10   (transform round-off only)
  FP32 engine: 2e-5    (FP32 storage and transforms, FP32 accumulation)
"""
import os

import numpy as np
import pytest

import psgpu_b200 as P
from oracle import pyoracle as O
from psgpu_b200.abi import TimestepLibrary
from psgpu_b200.fields import Grid2D, Grid3D, kolmogorov_ic2d, random_vorticity3d, taylor_green3d
from tests.golden_cases import cases, relerr

pytestmark = pytest.mark.gpu

CASES = cases()
TOL = {64: 1e-10, 32: 2e-5}


@pytest.fixture(params=[64, 32], ids=["fp64", "fp32"])
def precision(request, monkeypatch):
    monkeypatch.setenv("PSG_PRECISION", str(request.param))
    return request.param


def _lib(flavour):
    P.lib()
    return TimestepLibrary(P.dropin_path(flavour), flavour)


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_through_dropin(name, precision):
    d = CASES[name]
    fl, n = d["flavour"], int(d["n"])
    tol = TOL[precision]
    if fl == "ns2d":
        Z, t = _lib("ns2d").ns2d(d["Z_in"], n, d["nu"], d["dt"], int(d["nstop"]))
        assert relerr(Z, d["Z_out"]) < tol
        assert t == pytest.approx(d["time"], rel=1e-14)
    elif fl == "ns3d":
        a, b, c, t, ph = _lib("ns3d").ns3d(d["xii_in"], d["eta_in"], d["zet_in"], n, d["nu"],
                                           d["dt"], int(d["nstop"]), ampfor=d["ampfor"], kf=d["kf"])
        for x, k in ((a, "xii_out"), (b, "eta_out"), (c, "zet_out")):
            assert relerr(x, d[k]) < tol, k
        assert relerr(ph, d["phys_out"]) < tol
    elif fl == "euler3d":
        a, b, c, t, ph = _lib("euler3d").euler3d(d["xii_in"], d["eta_in"], d["zet_in"], n,
                                                 d["dt"], int(d["nstop"]))
        for x, k in ((a, "xii_out"), (b, "eta_out"), (c, "zet_out")):
            assert relerr(x, d[k]) < tol, k
        assert relerr(ph, d["phys_out"]) < tol
        assert t == pytest.approx(d["time"], rel=1e-14)
    elif fl == "bous3d":
        r = _lib("bous3d").bous3d(d["xii_in"], d["eta_in"], d["zet_in"], d["rho_in"], n, d["nu"],
                                  d["dt"], d["tend"], ri=d["ri"], sc=d["sc"], theta=d["theta"],
                                  ampfor=d["ampfor"], kf=d["kf"])
        for x, k in zip(r[:4], ("xii_out", "eta_out", "zet_out", "rho_out")):
            assert relerr(x, d[k]) < tol, k
        assert r[4] == pytest.approx(d["time"], rel=1e-14)
    elif fl == "bous3d_deriv":
        r = _lib("bous3d").bous3d_timederiv(d["xii_in"], d["eta_in"], d["zet_in"], d["rho_in"], n,
                                            d["nu"], ri=d["ri"], sc=d["sc"], theta=d["theta"],
                                            ampfor=d["ampfor"], kf=d["kf"])
        for x, k in zip(r, ("xii_out", "eta_out", "zet_out", "rho_out")):
            assert relerr(x, d[k]) < tol, k


def test_ns2d_long_run_against_oracle():
    """2D Kolmogorov flow, N=128, nu=1/40, dt=0.005, 400 steps: FP32 against FP64."""
    n, nu, dt, ns = 128, 1 / 40, 0.005, 400
    Z0 = kolmogorov_ic2d(n, 101)
    ref, _ = O.ns2d_timestep(Z0, n, nu, dt, ns)
    b = P.Batch2D([n], precision=32)
    b.upload(0, Z0)
    b.run(nu, dt, ns)
    Z = b.download(0)
    assert relerr(Z, ref) < 2e-5


def test_ns3d_rk4_against_oracle():
    """RK4/CN (Boussinesq scheme, Ri = 0) at N=64 on a Taylor-Green start, 20 steps;
    the vorticity does not see the density at Ri = 0."""
    n, nu, dt, ns = 64, 1 / 1600, 1e-3, 20
    xi, et, zt = taylor_green3d(n, 7, amp=1e-3)
    r = O.bous3d_timestep(xi, et, zt, np.zeros_like(xi), n, nu, dt, (ns + 0.5) * dt)
    for prec, tol in ((64, 1e-11), (32, 2e-5)):
        e = P.NS3D(n, P.SCHEME_NS_RK4, precision=prec, nu=nu)
        e.upload(xi, et, zt)
        e.step(dt, ns)
        e.step(0.5 * dt, 1)
        out = e.download()
        for x, y in zip(out, r[:3]):
            assert relerr(x, y) < tol


def test_masked_input_modes_are_cleared():
    """Garbage in masked modes of the input (outside the sphere and in the kx=0
    lower half) is treated as the reference does: the oracle is the checker."""
    n, nu, dt = 32, 1 / 20, 0.01
    g = Grid3D(n)
    rng = np.random.default_rng(3)
    xi, et, zt = random_vorticity3d(n, 9, kmin=0.5, kmax=9.5, solenoidal=True)
    junk = ~g.mask()
    xi = xi + junk * (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape))
    nuzn, nu1 = g.cn_coeffs(nu, dt)
    a = O.ns3d_timestep(xi, et, zt, n, nu, dt, 3, ampfor=-4.0, kfy=4.0)
    e = P.NS3D(n, P.SCHEME_NS_HEUN, precision=64, nu=nu, ampfor=-4.0, kf=4.0)
    e.upload(xi, et, zt)
    e.step(dt, 3)
    out = e.download()
    for x, y in zip(out, a[:3]):
        assert relerr(x, y) < 1e-10
    assert np.abs(out[0][junk]).max() == 0


def test_zero_steps_returns_input():
    n = 32
    Z = kolmogorov_ic2d(n, 5)
    b = P.Batch2D([n], precision=64)
    b.upload(0, Z)
    b.run(1 / 40, 0.005, 0)
    assert relerr(b.download(0), Z) == 0.0


def test_upload_download_roundtrip_fp64():
    n = 32
    xi, et, zt = random_vorticity3d(n, 2)
    e = P.NS3D(n, P.SCHEME_NS_RK4, precision=64)
    e.upload(xi, et, zt)
    out = e.download()
    for x, y in zip(out, (xi, et, zt)):
        assert (x == y).all()


def test_batch_of_mixed_sizes_matches_single_runs():
    sizes = [64, 16, 128, 32, 64]
    nus = [1 / 20, 1 / 40, 1 / 60, 1 / 30, 1 / 100]
    dt, ns = 0.005, 25
    b = P.Batch2D(sizes, precision=64)
    ics = [kolmogorov_ic2d(s, 40 + i) for i, s in enumerate(sizes)]
    for i, z in enumerate(ics):
        b.upload(i, z)
    b.run(nus, dt, ns)
    for i, s in enumerate(sizes):
        ref, _ = O.ns2d_timestep(ics[i], s, nus[i], dt, ns)
        assert relerr(b.download(i), ref) < 1e-10
