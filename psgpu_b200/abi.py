"""Python binding of the reference-compatible ``timestep_cuda_`` entry points.

psgpu's Fortran drivers call one C-ABI entry point per flavour, every argument
by pointer.  This module declares those signatures once and fills the argument
lists the way the drivers do (wavenumbers, masks, index maps, CN arrays), so the
same call drives either a library built from the reference's own sources or
this package's drop-in libraries (``libpsg_ns2d.so`` ...).

Signatures (all pointers, no hidden lengths):

* 2D:  2D_NavierStokes/src_RK4/src_gmres/cuda.cu:16-34, called at
  src_gmres/main.F90:708-710.
* 3D NS (DNS build): 3D_NavierStokes/src/cuda.cu:18-54, main.F90:203-204.
* 3D Euler: 3D_Euler/src/cuda.cu:17-44.
* 3D Boussinesq (GMRES build): 3D_Boussinesq/src/src_gmres/cuda.cu:12-49,
  ``timederiv_cuda_`` at :319-356.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

from .fields import Grid2D, Grid3D

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(x):
    return C.byref(C.c_double(float(x)))


def _i(x):
    return C.byref(C.c_int(int(x)))


def _pd(a):
    return a.ctypes.data_as(_dp)


def _pi(a):
    return a.ctypes.data_as(_ip)


def _cplx(a, shape):
    a = np.array(a, dtype=np.complex128, order="C", copy=True)
    return a.reshape(shape)


class TimestepLibrary:
    """One flavour's shared object exporting ``timestep_cuda_`` (and for the
    Boussinesq flavour ``timederiv_cuda_``)."""

    FLAVOURS = ("ns2d", "ns3d", "ns3d_newton", "euler3d", "bous3d", "bous3d_dns")

    def __init__(self, path: str, flavour: str):
        if flavour not in self.FLAVOURS:
            raise ValueError(f"unknown flavour {flavour!r}")
        self.path = os.path.abspath(path)
        self.flavour = flavour
        self.lib = C.CDLL(self.path, mode=C.RTLD_LOCAL)
        self.fn = self.lib.timestep_cuda_
        self.fn.restype = None
        self.fn.argtypes = None  # variadic-by-pointer; built per call

    # ------------------------------------------------------------------ 2D
    def ns2d(self, Z, n, nu, dt, nstop, alpha=1.0, tstart=0.0):
        """Integrate NSTOP RK4/CN steps of 2D Kolmogorov flow. Returns (Z, time)."""
        g = Grid2D(n, alpha)
        Z = _cplx(Z, g.shape)
        kx, ky = g.wavenumbers()
        kx = np.ascontiguousarray(kx.ravel()); ky = np.ascontiguousarray(ky.ravel())
        LC = g.mask().astype(np.int32).ravel()
        ikF = g.ikf(); ikN = g.ikn()
        ZR = np.zeros(n * n)
        t = np.zeros(1)
        self.fn(_pd(Z.view(np.float64)), _pd(ZR), _pd(kx), _pd(ky), _pd(t), _d(tstart),
                _d(nstop * dt), _d(dt), _d(alpha), _d(nu), _pi(ikF), _pi(ikN),
                _i(g.iktx), _i(g.ikty), _i(g.kt), _i(n), _i(n), _i(nstop), _pi(LC))
        return Z, float(t[0])

    # ------------------------------------------------------------------ 3D
    def _grid3(self, n, alpha):
        g = Grid3D(n, alpha)
        kx, ky, kz = (np.ascontiguousarray(a.ravel()) for a in g.wavenumbers())
        LC = g.mask().astype(np.int32).ravel()
        return g, kx, ky, kz, LC, g.ikf(), g.ikn()

    def ns3d(self, xii, eta, zet, n, nu, dt, nstop, ampfor=0.0, kf=4, tstart=0.0,
             alpha=1.0, workdir=None, steps_per_call=None):
        """3D NS Heun/CN (DNS build).  Returns (xii, eta, zet, time, phys[3,n,n,n]).
        The DNS build writes raw volumes to JOB<rank>/ at NT=0, so the call runs in
        a scratch working directory holding JOB0/.  ``steps_per_call`` splits the
        integration into several calls (each call restarts from the returned state
        with TSTART advanced, which for this scheme is the same trajectory)."""
        if steps_per_call and steps_per_call < nstop:
            t = tstart
            done = 0
            while done < nstop:
                k = min(steps_per_call, nstop - done)
                xii, eta, zet, tt, phys = self.ns3d(xii, eta, zet, n, nu, dt, k, ampfor, kf,
                                                    t, alpha, workdir)
                done += k
                t = tstart + done * dt
            return xii, eta, zet, tt, phys
        g, kx, ky, kz, LC, ikF, ikN = self._grid3(n, alpha)
        xii, eta, zet = (_cplx(a, g.shape) for a in (xii, eta, zet))
        nuzn, nu1 = g.cn_coeffs(nu, dt)
        phys = np.zeros((3, n * n * n))
        t = np.zeros(1)
        with _scratch_cwd(workdir, ("JOB0",)):
            self.fn(_pd(xii.view(np.float64)), _pd(eta.view(np.float64)),
                    _pd(zet.view(np.float64)), _pd(phys[0]), _pd(phys[1]), _pd(phys[2]),
                    _pd(nuzn), _pd(nu1), _pd(kx), _pd(ky), _pd(kz), _pd(t), _d(tstart),
                    _d(ampfor), _d(dt), _d(1.0), _d(float(kf)), _d(nu), _d(alpha),
                    _pi(ikF), _pi(ikN), _pi(LC), _i(g.iktx), _i(g.ikty), _i(g.iktz),
                    _i(g.kt), _i(g.nkt), _i(n), _i(n), _i(n), _i(nstop), _i(1),
                    _i(nstop + 1), _i(0), _i(0), _i(0))
        return xii, eta, zet, float(t[0]), phys.reshape(3, n, n, n)

    def ns3d_newton(self, xii, eta, zet, n, nu, dt, nstop, ampfor=0.0, kf=4, tstart=0.0,
                    alpha=1.0):
        """3D NS Heun/CN as the Newton-solver build steps it (18 arguments; the grid
        is the library's: 128 for the reference build, PSG_NEWTON_N for ours).
        Returns (xii, eta, zet, time)."""
        g, kx, ky, kz, LC, ikF, ikN = self._grid3(n, alpha)
        xii, eta, zet = (_cplx(a, g.shape) for a in (xii, eta, zet))
        nuzn, nu1 = g.cn_coeffs(nu, dt)
        t = np.zeros(1)
        self.fn(_pd(xii.view(np.float64)), _pd(eta.view(np.float64)), _pd(zet.view(np.float64)),
                _pd(nuzn), _pd(nu1), _pd(kx), _pd(ky), _pd(kz), _pd(t), _d(tstart), _d(ampfor),
                _d(dt), _i(int(kf)), _d(nu), _pi(ikF), _pi(ikN), _pi(LC), _i(nstop))
        return xii, eta, zet, float(t[0])

    def euler3d(self, xii, eta, zet, n, dt, nstop, tstart=0.0, alpha=1.0, workdir=None):
        g, kx, ky, kz, LC, ikF, ikN = self._grid3(n, alpha)
        xii, eta, zet = (_cplx(a, g.shape) for a in (xii, eta, zet))
        phys = np.zeros((3, n * n * n))
        t = np.zeros(1)
        with _scratch_cwd(workdir, ()):
            self.fn(_pd(xii.view(np.float64)), _pd(eta.view(np.float64)),
                    _pd(zet.view(np.float64)), _pd(phys[0]), _pd(phys[1]), _pd(phys[2]),
                    _pd(kx), _pd(ky), _pd(kz), _pd(t), _d(tstart), _d(dt), _d(alpha),
                    _pi(ikF), _pi(ikN), _pi(LC), _i(g.iktx), _i(g.ikty), _i(g.iktz),
                    _i(g.kt), _i(g.nkt), _i(n), _i(n), _i(n), _i(nstop), _i(1),
                    _i(nstop + 1), _i(0))
        return xii, eta, zet, float(t[0]), phys.reshape(3, n, n, n)

    def bous3d(self, xii, eta, zet, rho, n, nu, dt, tend, ri=0.0, sc=1.0, theta=0.0,
               ampfor=0.0, kf=4, tstart=0.0, time0=0.0, alpha=1.0):
        """3D Boussinesq RK4/CN (GMRES build, no file output): integrate from tstart
        to tend.  Returns (xii, eta, zet, rho, time)."""
        g, kx, ky, kz, LC, ikF, ikN = self._grid3(n, alpha)
        xii, eta, zet, rho = (_cplx(a, g.shape) for a in (xii, eta, zet, rho))
        t = np.array([time0], dtype=np.float64)
        self.fn(_pd(xii.view(np.float64)), _pd(eta.view(np.float64)),
                _pd(zet.view(np.float64)), _pd(rho.view(np.float64)),
                _pd(kx), _pd(ky), _pd(kz), _pd(t), _d(tstart), _d(tend), _d(ampfor),
                _d(dt), _d(1.0), _d(float(kf)), _d(nu), _d(ri), _d(sc), _d(theta),
                _d(alpha), _d(0.0), _pi(ikF), _pi(ikN), _pi(LC), _i(g.iktx), _i(g.ikty),
                _i(g.iktz), _i(g.kt), _i(g.nkt), _i(n), _i(n), _i(n), _i(1), _i(1),
                _i(0), _i(0), _i(0), _i(0))
        return xii, eta, zet, rho, float(t[0])

    def bous3d_dns(self, xii, eta, zet, rho, n, nu, dt, tend, ri=0.0, sc=1.0, theta=0.0,
                   ampfor=0.0, kf=4, dtarget=0.0, adapt=0, stats=0, nout=1, noutv=10 ** 6,
                   tstart=0.0, time0=0.0, alpha=1.0, workdir=None, rec=0, resthresh=1.0):
        """3D Boussinesq RK4/CN as the DNS build steps it (3D_Boussinesq/src/
        cuda.cu:21-58): integrate while t <= tend, with the adaptive step
        (adapt = 1) and the forcing throttle (dtarget != 0) at output times
        (every nout steps, stats != 0), and with rec = 1 the recurrence search
        (guesses to JOB0/UPO_ZK.out).  The reference build writes its
        diagnostics under JOB0/ of the working directory, so the call runs in a
        scratch directory holding JOB0/ (or in `workdir`).  Returns
        (xii, eta, zet, rho, time)."""
        g, kx, ky, kz, LC, ikF, ikN = self._grid3(n, alpha)
        xii, eta, zet, rho = (_cplx(a, g.shape) for a in (xii, eta, zet, rho))
        t = np.array([time0], dtype=np.float64)
        with _scratch_cwd(workdir, ("JOB0",)):
            self.fn(_pd(xii.view(np.float64)), _pd(eta.view(np.float64)),
                    _pd(zet.view(np.float64)), _pd(rho.view(np.float64)),
                    _pd(kx), _pd(ky), _pd(kz), _pd(t), _d(tstart), _d(tend), _d(ampfor),
                    _d(dt), _d(resthresh), _d(float(kf)), _d(nu), _d(ri), _d(sc), _d(theta),
                    _d(alpha), _d(dtarget), _pi(ikF), _pi(ikN), _pi(LC), _i(g.iktx),
                    _i(g.ikty), _i(g.iktz), _i(g.kt), _i(g.nkt), _i(n), _i(n), _i(n),
                    _i(nout), _i(noutv), _i(stats), _i(rec), _i(adapt), _i(0))
        return xii, eta, zet, rho, float(t[0])

    def bous3d_inplace(self, comps, n, nu, dt, tend, ri=0.0, sc=1.0, theta=0.0, ampfor=0.0,
                       kf=4, tstart=0.0, alpha=1.0):
        """The Boussinesq call on caller-owned arrays (complex128 boxes, e.g. in
        pinned memory), overwritten in place; the driver-side argument arrays are
        built once per grid and cached.  Returns the advanced time."""
        key = (n, alpha)
        cache = getattr(self, "_args3", {})
        if key not in cache:
            cache[key] = self._grid3(n, alpha)
            self._args3 = cache
        g, kx, ky, kz, LC, ikF, ikN = cache[key]
        for a in comps:
            if a.dtype != np.complex128 or a.size != g.nkt or not a.flags.c_contiguous:
                raise ValueError("state arrays must be contiguous complex128 boxes")
        t = np.zeros(1)
        self.fn(*[_pd(a.view(np.float64)) for a in comps],
                _pd(kx), _pd(ky), _pd(kz), _pd(t), _d(tstart), _d(tend), _d(ampfor),
                _d(dt), _d(1.0), _d(float(kf)), _d(nu), _d(ri), _d(sc), _d(theta),
                _d(alpha), _d(0.0), _pi(ikF), _pi(ikN), _pi(LC), _i(g.iktx), _i(g.ikty),
                _i(g.iktz), _i(g.kt), _i(g.nkt), _i(n), _i(n), _i(n), _i(1), _i(1),
                _i(0), _i(0), _i(0), _i(0))
        return float(t[0])

    def bous3d_timederiv(self, xii, eta, zet, rho, n, nu, ri=0.0, sc=1.0, theta=0.0,
                         ampfor=0.0, kf=4, alpha=1.0):
        """dz/dt of the Boussinesq system.  Signature as timestep_cuda_ of the same
        build (3D_Boussinesq/src/src_gmres/cuda.cu:319-356); the state arrays are
        overwritten with the time derivative."""
        fn = self.lib.timederiv_cuda_
        fn.restype = None
        g, kx, ky, kz, LC, ikF, ikN = self._grid3(n, alpha)
        xii, eta, zet, rho = (_cplx(a, g.shape) for a in (xii, eta, zet, rho))
        t = np.zeros(1)
        fn(_pd(xii.view(np.float64)), _pd(eta.view(np.float64)),
           _pd(zet.view(np.float64)), _pd(rho.view(np.float64)),
           _pd(kx), _pd(ky), _pd(kz), _pd(t), _d(0.0), _d(0.0), _d(ampfor),
           _d(1.0), _d(1.0), _d(float(kf)), _d(nu), _d(ri), _d(sc), _d(theta),
           _d(alpha), _d(0.0), _pi(ikF), _pi(ikN), _pi(LC), _i(g.iktx), _i(g.ikty),
           _i(g.iktz), _i(g.kt), _i(g.nkt), _i(n), _i(n), _i(n), _i(1), _i(1),
           _i(0), _i(0), _i(0), _i(0))
        return xii, eta, zet, rho


class _scratch_cwd:
    """Run a call inside a scratch directory (the DNS builds write files)."""

    def __init__(self, workdir, subdirs):
        self.workdir = workdir
        self.subdirs = subdirs
        self._tmp = None
        self._old = None

    def __enter__(self):
        self._old = os.getcwd()
        if self.workdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="psg_ref_")
            wd = self._tmp.name
        else:
            wd = self.workdir
            os.makedirs(wd, exist_ok=True)
        for s in self.subdirs:
            os.makedirs(os.path.join(wd, s), exist_ok=True)
        os.chdir(wd)
        return wd

    def __exit__(self, *exc):
        os.chdir(self._old)
        if self._tmp is not None:
            self._tmp.cleanup()
        return False
