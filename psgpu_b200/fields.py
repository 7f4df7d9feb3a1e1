"""Spectral layout, index maps and seeded initial conditions (host side, numpy).

The truncated spectral box follows psgpu's storage exactly:

* 2D: ``Z(IKTX, IKTY)`` Fortran order, i.e. numpy shape ``(IKTY, IKTX)``,
  ``kx = ikx * alpha``, ``ky = iky - KTY``
  (2D_NavierStokes/src_RK4/src_gmres/main.F90:328-335).
* 3D: ``XII(NKT)`` with ``ik = (ikz*IKTY + iky)*IKTX + ikx``, numpy shape
  ``(IKTZ, IKTY, IKTX)`` (3D_NavierStokes/src/init.F90:25-36).

``KT = N//3``, ``IKTX = KT+1``, ``IKTY = IKTZ = 2*KT+1``.  The mask keeps
``kx > 0`` or the upper half of the ``kx = 0`` plane, and ``|k| <= KT - 1/2``
(3D_NavierStokes/src/init.F90:38-57, 2D .../src_gmres/init.F90:25-39).

Physical fields relate to spectral coefficients as cuFFT's C2R does:
``f(x) = sum_k F_k exp(+i k.x)`` over the Hermitian-completed spectrum.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Grid2D:
    n: int
    alpha: float = 1.0

    @property
    def kt(self):
        return self.n // 3

    @property
    def iktx(self):
        return self.kt + 1

    @property
    def ikty(self):
        return 2 * self.kt + 1

    @property
    def nkt(self):
        return self.iktx * self.ikty

    @property
    def shape(self):
        return (self.ikty, self.iktx)

    def wavenumbers(self):
        kx = np.arange(self.iktx, dtype=np.float64)[None, :] * self.alpha
        ky = (np.arange(self.ikty, dtype=np.float64) - self.kt)[:, None]
        return np.broadcast_to(kx, self.shape).copy(), np.broadcast_to(ky, self.shape).copy()

    def mask(self):
        kx, ky = self.wavenumbers()
        wk = np.sqrt(kx * kx + ky * ky)
        keep = np.ones(self.shape, dtype=bool)
        keep &= ~(kx < 0)
        keep &= ~((kx == 0) & (ky <= 0))
        keep &= ~(wk > self.kt - 0.5)
        return keep

    def ikf(self):
        """padding map (2D .../src_gmres/main.F90:292-310), length (N/2+1)*N"""
        n, K, X = self.n, self.kt, self.iktx
        nx2 = n // 2 + 1
        out = -np.ones((n, nx2), np.int32)
        for iy in range(n):
            if iy <= K:
                src = iy + K
            elif iy >= n - K:
                src = iy + K - n
            else:
                continue
            out[iy, :X] = np.arange(X) + X * src
        return out.ravel()

    def ikn(self):
        """gather map (2D .../src_gmres/main.F90:312-325); sized (N/2+1)*N because
        the reference copies that many ints (src_gmres/init.h:164)."""
        n, K, X, Y = self.n, self.kt, self.iktx, self.ikty
        nx2 = n // 2 + 1
        out = np.zeros(nx2 * n, np.int32)
        for iy in range(Y):
            row = (n + iy - K) if iy < K else (iy - K)
            out[iy * X:(iy + 1) * X] = row * nx2 + np.arange(X)
        return out


@dataclass(frozen=True)
class Grid3D:
    n: int
    alpha: float = 1.0

    @property
    def kt(self):
        return self.n // 3

    @property
    def iktx(self):
        return self.kt + 1

    @property
    def ikty(self):
        return 2 * self.kt + 1

    @property
    def iktz(self):
        return 2 * self.kt + 1

    @property
    def nkt(self):
        return self.iktx * self.ikty * self.iktz

    @property
    def shape(self):
        return (self.iktz, self.ikty, self.iktx)

    def wavenumbers(self):
        kx = np.arange(self.iktx, dtype=np.float64)[None, None, :] * self.alpha
        ky = (np.arange(self.ikty, dtype=np.float64) - self.kt)[None, :, None]
        kz = (np.arange(self.iktz, dtype=np.float64) - self.kt)[:, None, None]
        b = lambda a: np.broadcast_to(a, self.shape).copy()
        return b(kx), b(ky), b(kz)

    def mask(self):
        kx, ky, kz = self.wavenumbers()
        wk = np.sqrt(kx * kx + ky * ky + kz * kz)
        keep = np.ones(self.shape, dtype=bool)
        keep &= ~(kx < 0)
        keep &= ~((kx == 0) & (ky < 0))
        keep &= ~((kx == 0) & (ky == 0) & (kz <= 0))
        keep &= ~(wk > self.kt - 0.5)
        return keep

    def ikf(self):
        """padding map (3D_NavierStokes/src/main.F90:100-156), length (N/2+1)*N*N"""
        n, K, X, Y = self.n, self.kt, self.iktx, self.ikty
        nx2 = n // 2 + 1
        idx = np.arange(n)
        src = np.where(idx <= K, idx + K, np.where(idx >= n - K, idx + K - n, -1))
        out = -np.ones((n, n, nx2), np.int64)
        zz = src[:, None, None]
        yy = src[None, :, None]
        xx = np.arange(nx2)[None, None, :]
        ok = (zz >= 0) & (yy >= 0) & (xx < X)
        val = xx + X * (yy + Y * zz)
        out = np.where(ok, val, -1)
        return out.astype(np.int32).ravel()

    def ikn(self):
        """gather map (3D_NavierStokes/src/main.F90:158-199), length NKT"""
        n, K, X, Y = self.n, self.kt, self.iktx, self.ikty
        nx2 = n // 2 + 1
        i = np.arange(Y)
        row = np.where(i < K, n + i - K, i - K)
        zz = row[:, None, None]
        yy = row[None, :, None]
        xx = np.arange(X)[None, None, :]
        return ((zz * n + yy) * nx2 + xx).astype(np.int32).ravel()

    def cn_coeffs(self, nu, dt):
        """NUZN, NU1 arrays of the 3D NS driver (3D_NavierStokes/src/init.F90:194-198)."""
        kx, ky, kz = self.wavenumbers()
        keep = self.mask()
        wk = np.sqrt(kx * kx + ky * ky + kz * kz)
        with np.errstate(divide="ignore"):
            NU = 10.0 ** (np.log10(nu) + 2.0 * np.log10(np.where(wk > 0, wk, 1.0)))
        nuzn = np.where(keep, (1.0 - 0.5 * NU * dt) / dt, 0.0)
        nu1 = np.where(keep, dt / (1.0 + 0.5 * NU * dt), 0.0)
        return nuzn.ravel(), nu1.ravel()


# --------------------------------------------------------------------------
# initial conditions
# --------------------------------------------------------------------------

def kolmogorov_ic2d(n: int, seed: int, kmin: float = 1.0, kmax: float = 8.0,
                    enstrophy: float = 1.0, alpha: float = 1.0) -> np.ndarray:
    """Seeded random vorticity on kmin <= |k| <= kmax, amplitude ~ |k|^-1, uniform
    random phases, rescaled so that 2*sum_LL |w_k|^2 = enstrophy (the reference's
    enstrophy convention, 2D .../src_gmres/init.F90:186-205)."""
    g = Grid2D(n, alpha)
    kx, ky = g.wavenumbers()
    keep = g.mask()
    wk = np.sqrt(kx * kx + ky * ky)
    rng = np.random.default_rng(seed)
    phase = rng.uniform(-np.pi, np.pi, size=g.shape)
    sel = keep & (wk >= kmin) & (wk <= kmax)
    amp = np.where(sel, 1.0 / np.where(wk > 0, wk, 1.0), 0.0)
    Z = amp * np.exp(1j * phase)
    ens = 2.0 * np.sum(np.abs(Z[keep]) ** 2)
    Z *= math.sqrt(enstrophy / ens)
    return Z.astype(np.complex128)


def taylor_green3d(n: int, seed: int, amp: float = 1e-3, kmax: float = 4.0,
                   alpha: float = 1.0) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Taylor-Green vorticity of u = (sin x cos y cos z, -cos x sin y cos z, 0),
    i.e. w = (-cos x sin y sin z, -sin x cos y sin z, 2 sin x sin y cos z), plus a
    seeded divergence-free perturbation i k x a(k) on 1 <= |k| <= kmax whose
    coefficient norm is ``amp`` times the Taylor-Green coefficient norm."""
    g = Grid3D(n, alpha)
    K = g.kt
    xi = np.zeros(g.shape, np.complex128)
    et = np.zeros(g.shape, np.complex128)
    zt = np.zeros(g.shape, np.complex128)
    for sy in (-1, 1):
        for sz in (-1, 1):
            iy, iz = sy + K, sz + K
            xi[iz, iy, 1] = sy * sz / 8.0
            et[iz, iy, 1] = sz / 8.0
            zt[iz, iy, 1] = -sy / 4.0
    tg_norm = math.sqrt(sum(np.sum(np.abs(a) ** 2) for a in (xi, et, zt)))
    if amp:
        kx, ky, kz = g.wavenumbers()
        keep = g.mask()
        wk = np.sqrt(kx * kx + ky * ky + kz * kz)
        sel = keep & (wk >= 1.0) & (wk <= kmax)
        rng = np.random.default_rng(seed)
        a = [(rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * sel
             for _ in range(3)]
        px = 1j * (ky * a[2] - kz * a[1])
        py = 1j * (kz * a[0] - kx * a[2])
        pz = 1j * (kx * a[1] - ky * a[0])
        pn = math.sqrt(sum(np.sum(np.abs(p) ** 2) for p in (px, py, pz)))
        s = amp * tg_norm / pn
        xi += s * px
        et += s * py
        zt += s * pz
    return xi, et, zt


def random_vorticity3d(n: int, seed: int, kmin: float = 2.5, kmax: float = 9.5,
                       enstrophy: float = 1.0, solenoidal: bool = False,
                       alpha: float = 1.0):
    """Unit-amplitude random-phase vorticity on a shell (the 3D DNS driver's IC form,
    3D_NavierStokes/src/init.F90:169-182), optionally projected to be
    divergence-free, rescaled to 2*sum|w|^2 = enstrophy over the kept modes."""
    g = Grid3D(n, alpha)
    kx, ky, kz = g.wavenumbers()
    keep = g.mask()
    wk = np.sqrt(kx * kx + ky * ky + kz * kz)
    sel = keep & (wk > kmin) & (wk <= kmax)
    rng = np.random.default_rng(seed)
    f = [np.where(sel, np.exp(1j * rng.uniform(-np.pi, np.pi, g.shape)), 0) for _ in range(3)]
    if solenoidal:
        k2 = np.where(wk > 0, wk * wk, 1.0)
        dot = (kx * f[0] + ky * f[1] + kz * f[2]) / k2
        f = [f[0] - kx * dot, f[1] - ky * dot, f[2] - kz * dot]
    ens = 2.0 * sum(np.sum(np.abs(a[keep]) ** 2) for a in f)
    s = math.sqrt(enstrophy / ens)
    return tuple((s * a).astype(np.complex128) for a in f)


def to_physical3d(F: np.ndarray, n: int) -> np.ndarray:
    """Inverse transform of one spectral box the way the reference feeds cuFFT:
    Hermitian completion of the kx=0 plane, zero padding, unnormalised C2R."""
    g = Grid3D(n)
    K, X = g.kt, g.iktx
    F = F.reshape(g.shape).copy()
    # fill the lower half of the kx=0 plane from the upper half (conj kernel)
    for iz in range(g.iktz):
        for iy in range(g.ikty):
            if iy < K or (iy == K and iz < K):
                F[iz, iy, 0] = np.conj(F[2 * K - iz, 2 * K - iy, 0])
    F[K, K, 0] = 0
    P = np.zeros((n, n, n // 2 + 1), np.complex128)
    idx = np.concatenate([np.arange(K, 2 * K + 1), np.arange(0, K)])
    pos = np.concatenate([np.arange(0, K + 1), np.arange(n - K, n)])
    P[np.ix_(pos, pos, np.arange(X))] = F[np.ix_(idx, idx, np.arange(X))]
    return np.fft.irfftn(P, s=(n, n, n), axes=(0, 1, 2), norm="forward")
