"""ctypes front end of the FP64 CPU oracle (oracle/_build/libpsg_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg import this module.

Arrays follow the reference layout: complex128 spectral boxes with kx fastest,
shape (IKTZ, IKTY, IKTX) in 3D and (IKTY, IKTX) in 2D.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "libpsg_oracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        d, i = C.c_double, C.c_int
        L.orc_nkt2d.argtypes = [i]; L.orc_nkt2d.restype = i
        L.orc_nkt3d.argtypes = [i]; L.orc_nkt3d.restype = i
        L.orc_layout2d.argtypes = [i, d, _dp, _dp, _ip]
        L.orc_layout3d.argtypes = [i, d, _dp, _dp, _dp, _ip]
        L.orc_ikf2d.argtypes = [i, _ip]; L.orc_ikn2d.argtypes = [i, _ip]
        L.orc_ikf3d.argtypes = [i, _ip]; L.orc_ikn3d.argtypes = [i, _ip]
        L.orc_ns2d_timestep.argtypes = [_dp, i, d, d, d, i, _dp]
        L.orc_ns2d_timestep.restype = i
        L.orc_ns2d_timederiv.argtypes = [_dp, _dp, i, d, d]
        L.orc_ns2d_timederiv.restype = i
        L.orc_ns3d_timestep.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, i, d, d, d, d, i, d, _dp]
        L.orc_ns3d_timestep.restype = i
        L.orc_ns3d_newton_timestep.argtypes = [_dp, _dp, _dp, _dp, _dp, i, d, d, d, d, i, d, _dp]
        L.orc_ns3d_newton_timestep.restype = i
        L.orc_euler3d_timestep.argtypes = [_dp, _dp, _dp, _dp, i, d, d, i, d, _dp]
        L.orc_euler3d_timestep.restype = i
        L.orc_bous3d_timestep.argtypes = [_dp, _dp, _dp, _dp, i, d, d, d, d, d, d, d, d, d, d, _dp]
        L.orc_bous3d_timestep.restype = i
        L.orc_bous3d_timederiv.argtypes = [_dp] * 8 + [i, d, d, d, d, d, d, d]
        L.orc_bous3d_timederiv.restype = i
        L.orc_energy3d.argtypes = [_dp, _dp, _dp, i, d]; L.orc_energy3d.restype = d
        L.orc_num_threads.restype = i
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _ip_(a):
    return a.ctypes.data_as(_ip)


def _c(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.copy()


def layout2d(n, alpha=1.0):
    nkt = lib().orc_nkt2d(n)
    kx = np.zeros(nkt); ky = np.zeros(nkt); LL = np.zeros(nkt, np.int32)
    lib().orc_layout2d(n, alpha, _p(kx), _p(ky), _ip_(LL))
    return kx, ky, LL


def layout3d(n, alpha=1.0):
    nkt = lib().orc_nkt3d(n)
    kx = np.zeros(nkt); ky = np.zeros(nkt); kz = np.zeros(nkt); LL = np.zeros(nkt, np.int32)
    lib().orc_layout3d(n, alpha, _p(kx), _p(ky), _p(kz), _ip_(LL))
    return kx, ky, kz, LL


def ikf2d(n):
    a = np.zeros((n // 2 + 1) * n, np.int32); lib().orc_ikf2d(n, _ip_(a)); return a


def ikn2d(n):
    # the reference copies n2 ints from this host array (src_gmres/init.h:164)
    a = np.zeros((n // 2 + 1) * n, np.int32); lib().orc_ikn2d(n, _ip_(a)); return a


def ikf3d(n):
    a = np.zeros((n // 2 + 1) * n * n, np.int32); lib().orc_ikf3d(n, _ip_(a)); return a


def ikn3d(n):
    a = np.zeros(lib().orc_nkt3d(n), np.int32); lib().orc_ikn3d(n, _ip_(a)); return a


def ns2d_timestep(Z, n, nu, dt, nstop, alpha=1.0):
    Z = _c(Z); t = np.zeros(1)
    rc = lib().orc_ns2d_timestep(_p(Z.view(np.float64)), n, alpha, nu, dt, nstop, _p(t))
    assert rc == 0
    return Z, float(t[0])


def ns2d_timederiv(Z, n, nu, alpha=1.0):
    Z = _c(Z); dZ = np.zeros_like(Z)
    rc = lib().orc_ns2d_timederiv(_p(Z.view(np.float64)), _p(dZ.view(np.float64)), n, alpha, nu)
    assert rc == 0
    return dZ


def cn_coeffs3d(n, nu, dt, alpha=1.0):
    """NUZN/NU1 as 3D_NavierStokes/src/init.F90:194-198 builds them."""
    kx, ky, kz, LL = layout3d(n, alpha)
    wk = np.sqrt(kx * kx + ky * ky + kz * kz)
    with np.errstate(divide="ignore"):
        NU = 10.0 ** (np.log10(nu) + 2.0 * np.log10(np.where(wk > 0, wk, 1.0)))
    nuzn = np.where(LL == 1, (1.0 - 0.5 * NU * dt) / dt, 0.0)
    nu1 = np.where(LL == 1, dt / (1.0 + 0.5 * NU * dt), 0.0)
    return nuzn, nu1


def ns3d_timestep(xii, eta, zet, n, nu, dt, nstop, ampfor=0.0, kfy=4.0, tstart=0.0,
                  alpha=1.0, want_phys=False):
    xii, eta, zet = _c(xii), _c(eta), _c(zet)
    nuzn, nu1 = cn_coeffs3d(n, nu, dt, alpha)
    phys = np.zeros(3 * n ** 3) if want_phys else None
    t = np.zeros(1)
    rc = lib().orc_ns3d_timestep(_p(xii.view(np.float64)), _p(eta.view(np.float64)),
                                 _p(zet.view(np.float64)),
                                 _p(phys) if phys is not None else None,
                                 _p(nuzn), _p(nu1), n, alpha, ampfor, kfy, dt, nstop,
                                 tstart, _p(t))
    assert rc == 0
    out = (xii, eta, zet, float(t[0]))
    if want_phys:
        out = out + (phys.reshape(3, n, n, n),)
    return out


def ns3d_newton_timestep(xii, eta, zet, n, nu, dt, nstop, ampfor=0.0, kfy=4.0, tstart=0.0,
                         alpha=1.0):
    """the Newton-solver build's Heun/CN step (its own forcing form)"""
    xii, eta, zet = _c(xii), _c(eta), _c(zet)
    nuzn, nu1 = cn_coeffs3d(n, nu, dt, alpha)
    t = np.zeros(1)
    rc = lib().orc_ns3d_newton_timestep(_p(xii.view(np.float64)), _p(eta.view(np.float64)),
                                        _p(zet.view(np.float64)), _p(nuzn), _p(nu1), n, alpha,
                                        ampfor, kfy, dt, nstop, tstart, _p(t))
    assert rc == 0
    return xii, eta, zet, float(t[0])


def euler3d_timestep(xii, eta, zet, n, dt, nstop, tstart=0.0, alpha=1.0, want_phys=False):
    xii, eta, zet = _c(xii), _c(eta), _c(zet)
    phys = np.zeros(3 * n ** 3) if want_phys else None
    t = np.zeros(1)
    rc = lib().orc_euler3d_timestep(_p(xii.view(np.float64)), _p(eta.view(np.float64)),
                                    _p(zet.view(np.float64)),
                                    _p(phys) if phys is not None else None,
                                    n, alpha, dt, nstop, tstart, _p(t))
    assert rc == 0
    out = (xii, eta, zet, float(t[0]))
    if want_phys:
        out = out + (phys.reshape(3, n, n, n),)
    return out


def bous3d_timestep(xii, eta, zet, rho, n, nu, dt, tend, ri=0.0, sc=1.0, theta=0.0,
                    ampfor=0.0, kfy=4.0, tstart=0.0, time0=0.0, alpha=1.0):
    xii, eta, zet, rho = _c(xii), _c(eta), _c(zet), _c(rho)
    t = np.array([time0])
    steps = lib().orc_bous3d_timestep(_p(xii.view(np.float64)), _p(eta.view(np.float64)),
                                      _p(zet.view(np.float64)), _p(rho.view(np.float64)),
                                      n, alpha, ampfor, kfy, nu, ri, sc, theta, dt, tstart,
                                      tend, _p(t))
    assert steps >= 0
    return xii, eta, zet, rho, float(t[0]), steps


def bous3d_timederiv(xii, eta, zet, rho, n, nu, ri=0.0, sc=1.0, theta=0.0, ampfor=0.0,
                     kfy=4.0, alpha=1.0):
    ins = [_c(a) for a in (xii, eta, zet, rho)]
    outs = [np.zeros_like(a) for a in ins]
    rc = lib().orc_bous3d_timederiv(*[_p(a.view(np.float64)) for a in ins],
                                    *[_p(a.view(np.float64)) for a in outs],
                                    n, alpha, ampfor, kfy, nu, ri, sc, theta)
    assert rc == 0
    return outs


def energy3d(xii, eta, zet, n, alpha=1.0):
    return lib().orc_energy3d(_p(_c(xii).view(np.float64)), _p(_c(eta).view(np.float64)),
                              _p(_c(zet).view(np.float64)), n, alpha)


def num_threads():
    return lib().orc_num_threads()
