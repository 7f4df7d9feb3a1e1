"""The C DNS driver psg_dns3 (params.txt -> random start -> Heun/CN steps ->
stats.dat / engy.dat / Zk.out, raw vorticity volumes every NOUTV steps)
against the same integration through the Python binding of the engine,
FP64, 32^3."""
import os
import subprocess

import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200 import host as H
from psgpu_b200.fields import to_physical3d
from tests.test_host_cpu import _params_text

pytestmark = pytest.mark.gpu


def test_dns3_driver(tmp_path):
    job = tmp_path / "JOB0"
    job.mkdir()
    (job / "params.txt").write_text(_params_text(TSTEP="0.1", outfreq1="0.02", DELT="0.01"))
    r = subprocess.run([H.driver_path(), "-n", "32", "-d", str(job), "-p", "64"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    n, nu, dt = 32, 1 / 20.0, 0.01
    # statistics after steps 3, 5, 7, 9 (NT = 2, 4, 6, 8 counted from 0) and of
    # the final state (finalise.h:19-22)
    rows = np.loadtxt(job / "stats.dat", ndmin=2)
    assert rows.shape == (5, 6)
    np.testing.assert_allclose(rows[:, 0], [0.03, 0.05, 0.07, 0.09, 0.1], rtol=1e-6)
    assert np.loadtxt(job / "engy.dat", ndmin=2).shape == (5, 7)
    ic = H.ic_random3d(n, 837920, 1.0)
    eng = P.NS3D(n, P.SCHEME_NS_HEUN, precision=64, nu=nu, ampfor=-4.0, kf=4.0)
    eng.upload(*ic)
    eng.step(dt, 3)
    e, _, _ = eng.energetics()
    assert rows[0, 1] == pytest.approx(e, rel=1e-6)  # %e keeps 7 digits
    eng.step(dt, 7)
    ref = eng.download()
    meta, *st = H.read_state3d(str(job / "Zk.out"), "D", 1, n)
    assert meta[0] == pytest.approx(10 * dt) and meta[1] == pytest.approx(nu)
    for a, b in zip(st, ref):
        np.testing.assert_array_equal(a, b)


def test_dns3_driver_recurrence_files(tmp_path):
    job = tmp_path / "JOB0"
    job.mkdir()
    (job / "params.txt").write_text(_params_text(TSTEP="0.2", outfreq1="0.02", DELT="0.01",
                                                 STATSFLAG="0", RCFLAG="1"))
    r = subprocess.run([H.driver_path(), "-n", "32", "-d", str(job), "-p", "32"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    info = (job / "UPOinfo_ts.dat").read_text().splitlines()
    assert info[0].startswith("Guess No")
    size = (job / "UPO_ZK.out").stat().st_size
    nkt = 11 * 21 * 21
    assert size % (56 + 3 * 16 * nkt) == 0 and size // (56 + 3 * 16 * nkt) == len(info) - 1
    assert not (job / "stats.dat").exists()


def _velocity(z, g):
    """u = i k x w / k^2 on the kept modes (setVelocity, 3D_NavierStokes/src/kernels.h:168-205)"""
    kx, ky, kz = g.wavenumbers()
    wk = np.maximum(kx * kx + ky * ky + kz * kz, 0.001)
    m = g.mask()
    xi, et, zt = z
    return [1j * (ky * zt - kz * et) / wk * m, 1j * (kz * xi - kx * zt) / wk * m,
            1j * (kx * et - ky * xi) / wk * m]


def test_dns3_driver_raw_volumes(tmp_path):
    """Volumes before steps NT = 0, NOUTV, ... (3D_NavierStokes/src/cuda.cu:72-93):
    xii001.raw is the physical vorticity of the start, xii002.raw that after
    NOUTV steps (the inverse transform as the reference feeds cuFFT, in
    numpy), FP64 with x fastest."""
    job = tmp_path / "JOB0"
    job.mkdir()
    (job / "params.txt").write_text(_params_text(TSTEP="0.1", outfreq1="0.02", outfreq2="0.04",
                                                 DELT="0.01"))
    r = subprocess.run([H.driver_path(), "-n", "32", "-d", str(job), "-p", "64"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    n, nu, dt = 32, 1 / 20.0, 0.01
    names = sorted(p.name for p in job.glob("*.raw"))
    # NT = 0, 4, 8 of NSTOP = 10
    assert names == [f"{c}{i:03d}.raw" for c in ("eta", "xii", "zet") for i in (1, 2, 3)]
    ic = H.ic_random3d(n, 837920, 1.0)
    eng = P.NS3D(n, P.SCHEME_NS_HEUN, precision=64, nu=nu, ampfor=-4.0, kf=4.0)
    eng.upload(*ic)
    states = {0: ic}
    eng.step(dt, 4)
    states[4] = eng.download()
    for k, nt in ((1, 0), (2, 4)):
        for q, c in enumerate(("xii", "eta", "zet")):
            vol = np.fromfile(job / f"{c}{k:03d}.raw", dtype=np.float64).reshape(n, n, n)
            ref = to_physical3d(states[nt][q], n)
            assert np.max(np.abs(vol - ref)) <= 1e-12 * np.max(np.abs(ref)), (k, c)


def test_dns3_driver_end_of_run_statistics(tmp_path):
    """STATSFLAG = 1: avgs.dat, means.dat and pdfs.dat as the DNS's finalise
    writes them (3D_NavierStokes/src/finalise.h:19-166), restated here from the
    engine's own states: the time average of the states the statistics saw
    (after steps 3, 5, 7, 9 and the final 10), its physical velocity; the mean
    squares of the physical velocity before steps 2, 4, 6, 8 (the first, at
    NT = 0, is overwritten: avgVelocity runs with tavgCount still 0 at NT =
    NOUT); x averages per (z, y); pdfs of energy, dissipation and input over the
    five statistics.  FP64, 32^3; 1e-10 (max-norm relative)."""
    job = tmp_path / "JOB0"
    job.mkdir()
    (job / "params.txt").write_text(_params_text(TSTEP="0.1", outfreq1="0.02", DELT="0.01"))
    r = subprocess.run([H.driver_path(), "-n", "32", "-d", str(job), "-p", "64"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    n, nu, dt, kf, amp = 32, 1 / 20.0, 0.01, 4, -4.0
    g = P.Grid3D(n)
    ic = H.ic_random3d(n, 837920, 1.0)
    eng = P.NS3D(n, P.SCHEME_NS_HEUN, precision=64, nu=nu, ampfor=amp, kf=float(kf))
    eng.upload(*ic)
    S = {0: [np.asarray(a).reshape(g.shape) for a in ic]}
    for t in range(1, 11):
        eng.step(dt, 1)
        S[t] = [np.asarray(a).reshape(g.shape) for a in eng.download()]
    seen = [S[t] for t in (3, 5, 7, 9, 10)]
    tavg = [sum(s[q] for s in seen) / len(seen) for q in range(3)]
    U = [to_physical3d(u, n) for u in _velocity(tavg, g)]
    ms = [sum(to_physical3d(u, n) ** 2 for u in [_velocity(S[t], g)[q] for t in (2, 4, 6, 8)]) / 4
          for q in range(3)]
    nr = n ** 3
    raw = np.fromfile(job / "avgs.dat", dtype=np.float64)
    assert raw.size == 5 * (1 + nr)
    rec = raw.reshape(5, 1 + nr)
    np.testing.assert_allclose(rec[:, 0], 10 * dt)
    want = [U[0], U[1], U[2], ms[1], ms[0] - U[0] ** 2]
    for k in range(5):
        got = rec[k, 1:].reshape(n, n, n)
        assert np.max(np.abs(got - want[k])) <= 1e-10 * np.max(np.abs(want[k])), k
    means = np.loadtxt(job / "means.dat")
    assert means.shape == (n * n, 6)
    prof = [a.mean(axis=2) for a in (U[0], U[1], ms[0] - U[0] ** 2, ms[1])]  # [z][y]
    yy, zz = np.meshgrid(np.arange(n) * 2 * np.pi / n, np.arange(n) * 2 * np.pi / n)
    np.testing.assert_allclose(means[:, 0], yy.ravel(), atol=1e-14)
    np.testing.assert_allclose(means[:, 1], zz.ravel(), atol=1e-14)
    for q in range(4):
        assert np.max(np.abs(means[:, 2 + q] - prof[q].ravel())) <= 1e-10 * np.max(np.abs(prof[q]))
    # pdfs: the energy, dissipation and input of the five statistics
    kx, ky, kz = g.wavenumbers()
    m = g.mask()
    wk = np.maximum(kx * kx + ky * ky + kz * kz, 0.001)
    vals = []
    for s in seen:
        vz = sum(np.abs(s[q]) ** 2 for q in range(3))
        e = float(np.sum((vz / wk)[m]))
        d = float(np.sum(vz[m])) * nu * nu * 8.0 * kf * kf
        sel = m & (kx == 0) & (ky == kf)
        inp = (amp * float(np.sum(s[0].real[sel & (kz == kf)]))
               - amp * float(np.sum(s[0].real[sel & (kz == -kf)]))) * nu * kf * kf
        vals.append((e, d, inp))
    vals = np.array(vals)
    lo, hi = np.minimum(vals.min(0), 0.0), np.maximum(vals.max(0), 0.0)
    pdf = np.loadtxt(job / "pdfs.dat")
    if hi[1] - lo[1] > 0.001:
        assert pdf.shape == (100, 6)
        for q in range(3):
            dx = (hi[q] * 1.0000001 - lo[q]) / 100
            cnt = np.zeros(101)
            for v in vals[:, q]:
                j = int((v - lo[q]) / dx) + 1
                if j <= 100:
                    cnt[j] += 1
            np.testing.assert_allclose(pdf[:, 2 * q], lo[q] + (np.arange(100) - 0.5) * dx, rtol=1e-9,
                                       atol=1e-12 * abs(dx))
            np.testing.assert_allclose(pdf[:, 2 * q + 1], cnt[:100] / (5 * dx), rtol=1e-9)
    else:
        assert pdf.size == 0
