"""Host-side driver pieces of libpsgpu.so, on CPU: the params.txt reader, the
drivers' random-number generator and random starts, type "A"/"C"/"D" state
files and the statistics lines.

The generator is checked draw for draw against an independent Python
restatement of ranno / ran1 (3D_NavierStokes/src/init.F90:236-292); the
Fortran driver itself cannot run here (no Fortran compiler), so the random
start's parity with the reference is pinned by that restatement and by the
start's defining properties (modes, moduli, enstrophy), not by the
reference's output.
"""
import math
import os
import struct

import numpy as np
import pytest

from psgpu_b200 import PsgError
from psgpu_b200 import host as H
from psgpu_b200.fields import Grid2D, Grid3D


def _params_text(**over):
    vals = dict(ISEED="837920", IREST="0", infile="none", infile_type="D", KF="4", Re="20.0",
                TSTEP="50.0", ResidualThreshold="1.0", outfreq1="0.1", outfreq2="10.0",
                DELT="0.01", AMPV="1.0", STATSFLAG="1", RCFLAG="0", UPOflag="0", ISTOP="1")
    vals.update(over)
    order = ["ISEED", "IREST", "infile", "infile type", "KF", "Re", "TSTEP", "ResidualThreshold",
             "outfreq1", "outfreq2", "DELT", "AMPV", "STATSFLAG", "RCFLAG", "UPOflag", "ISTOP"]
    return "".join(f"{k} = {vals[k.replace(' ', '_')]}\n" for k in order)


def test_params_reader_and_derived_values(tmp_path):
    p = tmp_path / "params.txt"
    p.write_text(_params_text())
    d = H.read_params3d(str(p))
    assert d["iseed"] == 837920 and d["kf"] == 4 and d["infile_type"] == "D"
    assert d["re"] == 20.0 and d["delt"] == 0.01 and d["statsflag"] == 1
    assert d["v2"] == pytest.approx(1 / 20.0)
    assert d["ampfor"] == -0.25 * 16
    assert d["nstop"] == int(50.0 / 0.01)
    assert d["nout"] == int(0.1 / 0.01) and d["noutv"] == int(10.0 / 0.01)


def test_params_fortran_float_without_point(tmp_path):
    # F12.4 input: digits without a decimal point carry 4 implied decimals
    p = tmp_path / "params.txt"
    p.write_text(_params_text(Re="20"))
    assert H.read_params3d(str(p))["re"] == pytest.approx(0.002)


def test_params_bad_label(tmp_path):
    p = tmp_path / "params.txt"
    p.write_text(_params_text().replace("KF = ", "KX = "))
    with pytest.raises(PsgError, match="label"):
        H.read_params3d(str(p))


class _Ran:
    """independent restatement of ranno / ran1"""

    def __init__(self):
        self.junk, self.iy, self.iv = 0, 0, [0] * 32

    def ran1(self, idum):
        ia, im, iq, ir, ntab = 16807, 2147483647, 127773, 2836, 32
        ndiv = 1 + (im - 1) // ntab
        if idum <= 0 or self.iy == 0:
            idum = max(-idum, 1)
            for j in range(ntab + 8, 0, -1):
                k = int(idum / iq)
                idum = ia * (idum - k * iq) - ir * k
                if idum < 0:
                    idum += im
                if j <= ntab:
                    self.iv[j - 1] = idum
            self.iy = self.iv[0]
        k = int(idum / iq)
        idum = ia * (idum - k * iq) - ir * k
        if idum < 0:
            idum += im
        j = 1 + self.iy // ndiv
        self.iy = self.iv[j - 1]
        self.iv[j - 1] = idum
        return min(self.iy * (1.0 / im), 1.0 - 1.2e-7)

    def ranno(self, i):
        tp = 4.0 * math.asin(1.0)
        if i != 0:
            if i > 0:
                i = -i
            self.junk = i
            return (self.ran1(i) - 0.5) * tp
        self.junk -= 1
        return (self.ran1(self.junk) - 0.5) * tp


@pytest.mark.parametrize("seed", [837920, 1, 12345])
def test_ranno_matches_restatement(seed):
    r = _Ran()
    r.ranno(seed)
    ref = np.array([r.ranno(0) for _ in range(2000)])
    got = H.ranno_draws(seed, 2000)
    np.testing.assert_array_equal(got, ref)
    assert np.all(np.abs(got) < math.pi)


def test_random_start_3d():
    n, ampv = 32, 1.0
    xi, et, zt = H.ic_random3d(n, 837920, ampv)
    g = Grid3D(n)
    kx, ky, kz = g.wavenumbers()
    wk = np.sqrt(kx * kx + ky * ky + kz * kz)
    shell = g.mask() & (wk > 2.5) & (wk <= 9.5)
    for v in (xi, et, zt):
        assert np.all(v[~shell] == 0)
        mod = np.abs(v[shell])
        assert np.allclose(mod, mod[0], rtol=1e-13)
    ens = 2 * sum(np.sum(np.abs(v) ** 2) for v in (xi, et, zt))
    assert ens == pytest.approx(ampv, rel=1e-13)
    # the phases are the generator's draws, three per kept mode, kx outermost, kz innermost
    r = _Ran()
    r.ranno(837920)
    order = [(ikz, iky, ikx) for ikx in range(g.iktx) for iky in range(g.ikty) for ikz in range(g.iktz)
             if g.mask()[ikz, iky, ikx]]
    ph = np.array([[r.ranno(0) for _ in range(3)] for _ in order])
    for j, idx in enumerate(order[:50]):
        if shell[idx]:
            for q, v in enumerate((xi, et, zt)):
                assert np.angle(v[idx]) == pytest.approx(math.remainder(ph[j, q], 2 * math.pi), abs=1e-12)


def test_random_start_2d():
    n, ampv = 64, 1.0
    Z = H.ic_random2d(n, 4242, ampv)
    g = Grid2D(n)
    kx, ky = g.wavenumbers()
    wk = np.sqrt(kx * kx + ky * ky)
    shell = g.mask() & (wk > 2.5) & (wk <= 9.5) & (kx >= 1)
    assert np.all(Z[~shell] == 0)
    assert np.allclose(np.abs(Z[shell]), np.abs(Z[shell][0]), rtol=1e-13)
    assert 2 * np.sum(np.abs(Z) ** 2) == pytest.approx(ampv, rel=1e-13)


def _record(payload: bytes) -> bytes:
    return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))


def test_state_files(tmp_path):
    n = 16
    g = Grid3D(n)
    rng = np.random.default_rng(3)
    states = [[rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape) for _ in range(3)]
              for _ in range(2)]
    metas = [np.arange(7.0) + 10 * r for r in range(2)]
    body = lambda r: metas[r].tobytes() + b"".join(a.tobytes() for a in states[r])
    # type D: header record, then one record per state
    d = tmp_path / "Zk.in"
    d.write_bytes(_record(struct.pack("<4i", 2, g.iktx, g.ikty, g.iktz)) + _record(body(0)) +
                  _record(body(1)))
    # type A: the same content as a stream; type C: records of the fields only
    a = tmp_path / "A.in"
    a.write_bytes(body(0) + body(1))
    c = tmp_path / "C.in"
    c.write_bytes(b"".join(_record(b"".join(x.tobytes() for x in states[r])) for r in range(2)))
    for path, kind in ((d, "D"), (a, "A"), (c, "C")):
        for r in (1, 2):
            meta, *st = H.read_state3d(str(path), kind, r, n)
            for x, y in zip(st, states[r - 1]):
                np.testing.assert_array_equal(x, y)
            if kind != "C":
                np.testing.assert_array_equal(meta, metas[r - 1])
    with pytest.raises(PsgError):
        H.read_state3d(str(d), "D", 3, n)
    with pytest.raises(PsgError, match="resolution"):
        H.read_state3d(str(d), "D", 1, 32)
