"""The batched 2D GPU recurrence search against a Python restatement of the 2D
DNS's recurrence check (2D_NavierStokes/src_RK4/functions.h:105-309 with the
ring bookkeeping the 3D DNS loop shares, 3D_NavierStokes/src/cuda.cu:116-138).

Three runs are searched at once, each on a synthetic sequence that is periodic
up to a grid translation for a while (a different period per run) and then
loses its period; every check must emit the same guesses as the restatement
(run, start time, period and shifts exactly; residual to 1e-10) with the same
stored state.  A second case feeds real 2D Kolmogorov states from the batch
engine in FP32 and FP64."""
import math

import numpy as np
import pytest
import torch

import psgpu_b200 as P
from psgpu_b200.fields import Grid2D, kolmogorov_ic2d

pytestmark = pytest.mark.gpu


class RecRef2D:
    def __init__(self, n, store, nw, ns, thresh, nout, delt, tstart, v2, alpha=1.0):
        g = Grid2D(n)
        K = n // 3
        self.store, self.ns = store, ns
        self.thresh, self.nout, self.delt, self.tstart, self.v2 = thresh, nout, delt, tstart, v2
        self.freq2 = 2 * nout * delt
        idx = [(K - nw + iy, ix) for iy in range(2 * nw) for ix in range(nw)]
        self.idx = tuple(np.array(i) for i in zip(*idx))
        self.k = [self.idx[1] * alpha, self.idx[0] - K]
        self.ll = g.mask()[self.idx]
        tp = 4.0 * math.asin(1.0)
        self.sx = [tp * i / (ns[0] * alpha) for i in range(ns[0])]
        self.sy = [tp * i / ns[1] for i in range(ns[1])]
        self.ring = [None] * store
        self.norms = [0.0] * store
        self.nStore = self.nCopy = self.iStart = self.recOut = 0
        self.minResOuter = 0.0
        self.guess = None

    def put(self, slot, st):
        self.ring[slot] = st.copy()
        self.norms[slot] = float(np.sum(np.abs(st[self.idx][self.ll]) ** 2))

    def check(self, nt):
        tme = self.tstart + (nt - self.nout) * self.delt
        newest = self.ring[self.nCopy][self.idx]
        minResInner, minPeriod, res = 10000.0, 10000.0, 0.0
        minPflag, minStoreInner, minCountInner = 1, 0, 0
        sxi = syi = 0.0
        for icount in range(self.nStore - 1, 0, -1):
            period = ((self.nStore - icount) * self.nout) * self.delt
            slot = (icount + self.iStart) % self.store
            if period > 20.0 and abs(period - self.freq2 * math.floor(period / self.freq2 + 0.5)) > 1e-4:
                continue
            old = self.ring[slot][self.idx]
            resPrev, res = res, 10000.0
            for sy in self.sy:
                for sx in self.sx:
                    d = newest * np.exp(-1j * (self.k[0] * sx + self.k[1] * sy))
                    r2 = (-2 * np.sum(d.real * old.real + d.imag * old.imag)
                          + np.sum(np.abs(d) ** 2) + self.norms[slot])
                    x = r2 / self.norms[self.nCopy]
                    r = math.sqrt(x) if x >= 0 else math.nan
                    if r < res:
                        res, bs = r, (sx, sy)
            if res > resPrev and minPflag == 1:
                minPeriod = period
            else:
                minPflag = 0
            if res < minResInner and period > minPeriod:
                minResInner, minStoreInner = res, slot
                minCountInner = self.nStore - icount
                sxi, syi = bs
        emitted = False
        if minResInner < self.thresh and self.recOut == 0:
            self.minResOuter, self.recOut = self.thresh, 1
        if minResInner < self.minResOuter and self.recOut == 1:
            self.minResOuter = minResInner
            self.best = (tme + minCountInner * self.nout * self.delt, self.v2,
                         minCountInner * self.nout * self.delt, sxi, syi, minResInner,
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


def _sequence(n, count, period, nsx, seed):
    g = Grid2D(n)
    kx, _ = g.wavenumbers()
    rng = np.random.default_rng(seed)
    m = g.mask()
    z0 = (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * m
    a = 2 * math.pi * 5 / (nsx * period)  # one period moves the state 5 grid shifts in x
    out = []
    for t in range(count):
        if t < 3 * period:
            amp = 1.0 + 0.3 * math.sin(2 * math.pi * t / period)
            out.append((z0 * amp + 2e-3 * (rng.standard_normal(g.shape)
                                           + 1j * rng.standard_normal(g.shape)) * m)
                       * np.exp(-1j * kx * a * t))
        else:
            out.append((rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * m)
    return out


@pytest.mark.parametrize("store", [40, 12])
def test_recurrence2d_matches_restatement(store):
    n, nw, ns, nout, dt, thr = 32, 6, (24, 4), 1, 0.1, 0.05
    periods = (8, 6, 9)
    v2 = (0.02, 0.03, 0.04)
    seqs = [_sequence(n, 32, p, ns[0], 10 + r) for r, p in enumerate(periods)]
    R = len(periods)
    gpu = P.Recurrence2D(R, n, nout, dt, thr, v2, store_size=store, norm_width=nw, nshift=ns)
    refs = [RecRef2D(n, store, nw, ns, thr, nout, dt, 0.0, v2[r]) for r in range(R)]
    dev = lambda t: [torch.from_numpy(np.ascontiguousarray(seqs[r][t])).cuda() for r in range(R)]
    gpu.start(dev(0))
    for r in range(R):
        refs[r].put(0, seqs[r][0])
    seen = 0
    found = []
    for t in range(1, 32):
        e_gpu = gpu.add(t * nout, dev(t))
        e_ref = [refs[r].add(t * nout, seqs[r][t]) for r in range(R)]
        assert e_gpu == sum(e_ref), t
        emitted_runs = [r for r in range(R) if e_ref[r]]
        for k, r in zip(range(seen, seen + e_gpu), emitted_runs):
            meta, Z = gpu.guess(k)
            tm, vv, per, sx, sy, res, slot = refs[r].guess
            assert meta["run"] == r
            assert meta["time"] == pytest.approx(tm, abs=1e-12)
            assert meta["v2"] == vv
            assert meta["period"] == pytest.approx(per, abs=1e-12)
            assert (meta["shift_x"], meta["shift_y"]) == pytest.approx((sx, sy))
            assert meta["residual"] == pytest.approx(res, rel=1e-10, abs=1e-13)
            np.testing.assert_array_equal(Z, refs[r].ring[slot])
            found.append(meta)
        seen += e_gpu
    if store >= 16:
        # every run's periodic stretch is found at a multiple m of its period
        # (the reference's first-turning-point rule can skip the first one); the
        # state moved +5 grid shifts in x per period, so the shift that maps it
        # back is 24 - 5 m (mod 24)
        for r, p in enumerate(periods):
            hits = [m for m in found if m["run"] == r]
            assert hits
            mult = hits[0]["period"] / (0.1 * p)
            assert abs(mult - round(mult)) < 1e-9 and 1 <= round(mult) <= 3
            assert hits[0]["shift_x"] == pytest.approx(2 * math.pi * ((24 - 5 * round(mult)) % 24) / 24)


@pytest.mark.parametrize("precision", [64, 32])
def test_recurrence2d_on_batch_states(precision):
    """Kolmogorov runs from the batch engine: the search reads the engine's own
    device states (FP32 or FP64) and its guesses equal the restatement's on the
    same (downloaded) states."""
    n, nu, dt, nout = 32, 1 / 30, 0.005, 20
    R = 2
    b = P.Batch2D([n] * R, precision=precision)
    for r in range(R):
        b.upload(r, kolmogorov_ic2d(n, 300 + r))
    b.run(nu, dt, 4000)  # past the transient
    b.sync()
    gpu = P.Recurrence2D(R, n, nout, dt, 0.3, 1 / 30, store_size=60, norm_width=6,
                         nshift=(32, 4))
    refs = [RecRef2D(n, 60, 6, (32, 4), 0.3, nout, dt, 0.0, 1 / 30) for _ in range(R)]
    rnd = (lambda z: z.astype(np.complex64).astype(np.complex128)) if precision == 32 else (lambda z: z)
    gpu.start(b)
    for r in range(R):
        refs[r].put(0, rnd(_device_z(b, r, n, precision)))
    total = 0
    for t in range(1, 120):
        b.run(nu, dt, nout)
        b.sync()
        e = gpu.add(t * nout, b)
        er = [refs[r].add(t * nout, rnd(_device_z(b, r, n, precision))) for r in range(R)]
        assert e == sum(er), t
        total += e
    assert gpu.count == total


class _DevBytes:
    """a device address as a byte array torch can wrap (__cuda_array_interface__)"""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1",
                                         "data": (ptr, False), "version": 3}


def _device_z(b, r, n, precision):
    """instance r's state exactly as the device holds it (without the FP32 carried error)"""
    g = Grid2D(n)
    nbytes = g.nkt * (16 if precision == 64 else 8)
    torch.cuda.synchronize()
    raw = torch.as_tensor(_DevBytes(b.device_state(r), nbytes), device="cuda").cpu().numpy()
    z = raw.view(np.complex128 if precision == 64 else np.complex64).reshape(g.shape)
    return z.astype(np.complex128)
