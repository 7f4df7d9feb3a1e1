"""The GPU recurrence search against a Python restatement of the DNS's
recurrence check (3D_NavierStokes/src/functions.h:251-389 with the ring
bookkeeping of cuda.cu:116-138), on a synthetic sequence that is periodic up
to a grid translation for a while and then loses its period: the same
checks must emit the same guess (start time, period, shifts exactly; residual
to 1e-10) with the same stored state."""
import math

import numpy as np
import pytest
import torch

import psgpu_b200 as P
from psgpu_b200.fields import Grid3D

pytestmark = pytest.mark.gpu


class RecRef:
    """ri None: the 3D NS DNS's check; ri given: the Boussinesq DNS's
    (3D_Boussinesq/src/functions.h:189-205, 416-616) on four fields"""

    def __init__(self, n, store, nw, ns, thresh, nout, delt, tstart, v2, alpha=1.0, ri=None):
        self.ri = ri
        g = Grid3D(n)
        K = n // 3
        self.K, self.store, self.nw, self.ns = K, store, nw, ns
        self.thresh, self.nout, self.delt, self.tstart, self.v2 = thresh, nout, delt, tstart, v2
        self.freq2 = 2 * nout * delt
        idx = []
        for iz in range(2 * nw):
            for iy in range(2 * nw):
                for ix in range(nw):
                    idx.append((K - nw + iz, K - nw + iy, ix))
        self.idx = tuple(np.array(i) for i in zip(*idx))
        self.k = [self.idx[2] * alpha, self.idx[1] - K, self.idx[0] - K]
        self.ll = g.mask()[self.idx]
        tp = 4.0 * math.asin(1.0)
        self.sx = [tp * i / (ns[0] * alpha) for i in range(ns[0])]
        self.sy = [tp * i / ns[1] for i in range(ns[1])]
        self.sz = [tp * i / ns[2] for i in range(ns[2])]
        self.ring = [None] * store
        self.norms = [0.0] * store
        self.nStore = self.nCopy = self.iStart = self.recOut = 0
        self.minResOuter = 0.0
        self.guess = None

    def put(self, slot, st):
        self.ring[slot] = [a.copy() for a in st]
        sub = np.stack([a[self.idx] for a in st])
        if self.ri is None:
            self.norms[slot] = float(np.sum(np.abs(sub[:, self.ll]) ** 2))
        else:  # whole box; ri on the density's real part only, as written
            r = sub[3]
            self.norms[slot] = float(np.sum(np.abs(sub[:3]) ** 2)
                                     + np.sum(self.ri * r.real ** 2 + r.imag ** 2))

    def check(self, nt):
        tme = self.tstart + (nt - self.nout) * self.delt
        newest = np.stack([a[self.idx] for a in self.ring[self.nCopy]])
        minResInner, minPeriod, res = 10000.0, 10000.0, 0.0
        minPflag, minStoreInner, minCountInner = 1, 0, 0
        sxi = syi = szi = 0.0
        for icount in range(self.nStore - 1, 0, -1):
            period = ((self.nStore - icount) * self.nout) * self.delt
            slot = (icount + self.iStart) % self.store
            if self.ri is not None and period < 0.5:
                continue
            if period > 20.0 and abs(period - self.freq2 * math.floor(period / self.freq2 + 0.5)) > 1e-4:
                continue
            old = np.stack([a[self.idx] for a in self.ring[slot]])
            resPrev, res = res, 10000.0
            for sy in self.sy:
                for sz in self.sz:
                    for sx in self.sx:
                        ph = np.exp(-1j * (self.k[0] * sx + self.k[1] * sy + self.k[2] * sz))
                        d = newest * ph
                        w = np.ones(len(d))
                        if self.ri is not None:
                            w[3] = self.ri
                        cr = np.sum(d.real * old.real + d.imag * old.imag, axis=1)
                        r2 = -2 * np.sum(w * cr) + np.sum(w * np.sum(np.abs(d) ** 2, axis=1)) \
                            + self.norms[slot]
                        den = self.norms[self.nCopy] + (self.norms[slot] if self.ri is not None else 0.0)
                        x = r2 / den
                        r = math.sqrt(x) if x >= 0 else math.nan  # as C's sqrt
                        if r < res:
                            res, bs = r, (sx, sy, sz)
            if res > resPrev and minPflag == 1:
                minPeriod = period
            else:
                minPflag = 0
            if res < minResInner and period > minPeriod:
                minResInner, minStoreInner = res, slot
                minCountInner = self.nStore - icount
                sxi, syi, szi = bs
        emitted = False
        if minResInner < self.thresh and self.recOut == 0:
            self.minResOuter, self.recOut = self.thresh, 1
        if minResInner < self.minResOuter and self.recOut == 1:
            self.minResOuter = minResInner
            self.best = (tme + minCountInner * self.nout * self.delt, self.v2,
                         minCountInner * self.nout * self.delt, sxi, syi, szi, minResInner,
                         minStoreInner)
        if minResInner > self.thresh and self.recOut == 1:
            self.recOut = 0
            self.guess = self.best
            emitted = True
        return emitted

    def add(self, nt, st):
        emitted = self.check(nt) if self.nStore >= 1 else False
        self.nStore += 1
        if self.nStore >= self.store:
            self.nStore = self.store
            self.nCopy = (self.nCopy + 1) % self.store
            self.iStart = self.nCopy
        else:
            self.nCopy = self.nStore
        self.put(self.nCopy, st)
        return emitted


def _sequence(n, count, period, nsx, seed=5, nc=3):
    g = Grid3D(n)
    kx, _, _ = g.wavenumbers()
    rng = np.random.default_rng(seed)
    m = g.mask()
    z0 = [(rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * m for _ in range(nc)]
    a = 2 * math.pi * 7 / (nsx * period)  # after one period: a grid translation of 7 steps
    out = []
    for t in range(count):
        if t < 3 * period:
            # periodic up to the translation, plus a little noise so that no
            # residual sits at round-off (where its sign is arbitrary)
            amp = 1.0 + 0.3 * math.sin(2 * math.pi * t / period)
            out.append([(z * amp + 2e-3 * (rng.standard_normal(g.shape) +
                                           1j * rng.standard_normal(g.shape)) * m)
                        * np.exp(-1j * kx * a * t) for z in z0])
        else:
            out.append([(rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * m
                        for _ in range(nc)])
    return out


@pytest.mark.parametrize("store", [40, 12])
def test_recurrence_matches_restatement(store):
    n, nw, ns, nout, dt, thr = 16, 4, (30, 2, 2), 1, 0.1, 0.05
    seq = _sequence(n, 30, 8, ns[0])
    gpu = P.Recurrence3D(n, nout, dt, thr, store_size=store, norm_width=nw, nshift=ns, v2=0.02)
    ref = RecRef(n, store, nw, ns, thr, nout, dt, 0.0, 0.02)
    dev = lambda st: torch.from_numpy(np.stack(st)).cuda()
    gpu.start(dev(seq[0]))
    ref.put(0, seq[0])
    emitted = []
    for t in range(1, len(seq)):
        e_gpu = gpu.add(t * nout, dev(seq[t]))
        e_ref = ref.add(t * nout, seq[t])
        assert e_gpu == e_ref, t
        if e_gpu:
            meta, st = gpu.guess()
            tm, v2, per, sx, sy, sz, res, slot = ref.guess
            assert meta["time"] == pytest.approx(tm, abs=1e-12)
            assert meta["period"] == pytest.approx(per, abs=1e-12)
            assert (meta["shift_x"], meta["shift_y"], meta["shift_z"]) == pytest.approx((sx, sy, sz))
            assert meta["residual"] == pytest.approx(res, rel=1e-10, abs=1e-13)
            for a, b in zip(st, ref.ring[slot]):
                np.testing.assert_array_equal(a, b)
            emitted.append(meta)
    if store >= 16:
        # the periodic stretch is found: period 8 outputs; the state moved by
        # +7 grid steps in x, so the shift that maps it back is -7 = 23 (mod 30)
        assert emitted and emitted[0]["period"] == pytest.approx(0.8)
        assert emitted[0]["shift_x"] == pytest.approx(2 * math.pi * 23 / 30)


def test_boussinesq_recurrence_matches_restatement():
    """The Boussinesq DNS's variant on four fields (density weighted by Ri).
    Its norm of a stored state weights only the density's real part by Ri
    (3D_Boussinesq/src/functions.h:199) while the residual weights both parts,
    so an exact recurrence leaves a floor of sqrt((1 - Ri) sum Im(rho)^2 /
    (|Z_old|^2 + |Z_new|^2)); the density here is a tenth of the vorticity
    (floor ~ 0.015, below the threshold 0.05).  The selection reports twice the
    period (1.6) with the matching shift 16 (= -2 x 7 mod 30) grid steps."""
    n, nw, ns, nout, dt, thr, ri = 16, 4, (30, 2, 2), 1, 0.1, 0.05, 0.7
    seq = [[a, b, c, 0.1 * d] for a, b, c, d in _sequence(n, 30, 8, ns[0], seed=9, nc=4)]
    gpu = P.Recurrence3D(n, nout, dt, thr, store_size=40, norm_width=nw, nshift=ns, v2=0.02, ri=ri)
    ref = RecRef(n, 40, nw, ns, thr, nout, dt, 0.0, 0.02, ri=ri)
    dev = lambda st: torch.from_numpy(np.stack(st)).cuda()
    gpu.start(dev(seq[0]))
    ref.put(0, seq[0])
    n_emit = 0
    for t in range(1, len(seq)):
        e_gpu = gpu.add(t * nout, dev(seq[t]))
        e_ref = ref.add(t * nout, seq[t])
        assert e_gpu == e_ref, t
        if e_gpu:
            n_emit += 1
            meta, st = gpu.guess()
            tm, v2, per, sx, sy, sz, res, slot = ref.guess
            assert meta["period"] == pytest.approx(per, abs=1e-12)
            assert (meta["shift_x"], meta["shift_y"], meta["shift_z"]) == pytest.approx((sx, sy, sz))
            assert meta["residual"] == pytest.approx(res, rel=1e-10, abs=1e-13)
            assert len(st) == 4
            for a, b in zip(st, ref.ring[slot]):
                np.testing.assert_array_equal(a, b)
            assert meta["period"] == pytest.approx(1.6)
            assert meta["shift_x"] == pytest.approx(2 * math.pi * 16 / 30)
    assert n_emit >= 1
