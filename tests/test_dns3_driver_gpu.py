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
    # statistics after steps 3, 5, 7, 9 (NT = 2, 4, 6, 8 counted from 0)
    rows = np.loadtxt(job / "stats.dat", ndmin=2)
    assert rows.shape == (4, 6)
    np.testing.assert_allclose(rows[:, 0], [0.03, 0.05, 0.07, 0.09], rtol=1e-6)
    assert np.loadtxt(job / "engy.dat", ndmin=2).shape == (4, 7)
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


def test_dns3_driver_raw_volumes(tmp_path):
    """Volumes before steps NT = 0, NOUTV, ... (3D_NavierStokes/src/cuda.cu:72-93):
    xii001.raw is the physical vorticity of the start, xii002.raw that after
    NOUTV steps, FP64 with x fastest."""
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
    for k, nt in ((1, 0), (2, 4)):
        eng.step(dt, (nt + 1) - (0 if k == 1 else 1), dump_last=True)
        ph = eng.physical()
        for q, c in enumerate(("xii", "eta", "zet")):
            vol = np.fromfile(job / f"{c}{k:03d}.raw", dtype=np.float64).reshape(n, n, n)
            np.testing.assert_array_equal(vol, ph[q])
