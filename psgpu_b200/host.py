"""Python access to the host-side driver pieces of libpsgpu.so
(include/psgpu_host.h): parameter files, the drivers' random starts and their
generator, and the type "D" state files."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import LIBDIR, PsgError, lib
from .fields import Grid2D, Grid3D


class Params3D(C.Structure):
    _fields_ = [("iseed", C.c_int), ("irest", C.c_int), ("infile", C.c_char * 256),
                ("infile_type", C.c_char * 256), ("kf", C.c_int), ("re", C.c_double),
                ("tstep", C.c_double), ("residual_threshold", C.c_double),
                ("outfreq1", C.c_double), ("outfreq2", C.c_double), ("delt", C.c_double),
                ("ampv", C.c_double), ("statsflag", C.c_int), ("rcflag", C.c_int),
                ("upoflag", C.c_int), ("istop", C.c_int), ("v2", C.c_double),
                ("ampfor", C.c_double), ("nstop", C.c_int), ("nout", C.c_int), ("noutv", C.c_int)]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = v.decode() if isinstance(v, bytes) else v
        return d


class RannoState(C.Structure):
    _fields_ = [("junk", C.c_int), ("iy", C.c_int), ("iv", C.c_int * 32)]


def _L():
    L = lib()
    if not getattr(L, "_host_declared", False):
        dp = C.POINTER(C.c_double)
        L.psg_read_params3d.argtypes = [C.c_char_p, C.POINTER(Params3D)]
        L.psg_ranno_init.argtypes = [C.POINTER(RannoState)]
        L.psg_ranno_init.restype = None
        L.psg_ranno.argtypes = [C.POINTER(RannoState), C.c_int]
        L.psg_ranno.restype = C.c_double
        L.psg_ic_random3d.argtypes = [C.c_int, C.c_int, C.c_double, dp, dp, dp]
        L.psg_ic_random2d.argtypes = [C.c_int, C.c_int, C.c_double, dp]
        L.psg_read_state3d.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, dp, dp, dp, dp]
        L._host_declared = True
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def read_params3d(path: str) -> dict:
    p = Params3D()
    if _L().psg_read_params3d(path.encode(), C.byref(p)) != 0:
        raise PsgError(lib().psg_last_error().decode())
    return p.as_dict()


def ranno_draws(seed: int, count: int) -> np.ndarray:
    """ranno(seed) then `count` draws of ranno(0)"""
    L = _L()
    s = RannoState()
    L.psg_ranno_init(C.byref(s))
    L.psg_ranno(C.byref(s), seed)
    return np.array([L.psg_ranno(C.byref(s), 0) for _ in range(count)])


def ic_random3d(n: int, iseed: int, ampv: float = 1.0):
    g = Grid3D(n)
    out = [np.zeros(g.shape, np.complex128) for _ in range(3)]
    if _L().psg_ic_random3d(n, iseed, ampv, *[_dp(o) for o in out]) != 0:
        raise PsgError(lib().psg_last_error().decode())
    return tuple(out)


def ic_random2d(n: int, iseed: int, ampv: float = 1.0):
    g = Grid2D(n)
    Z = np.zeros(g.shape, np.complex128)
    if _L().psg_ic_random2d(n, iseed, ampv, _dp(Z)) != 0:
        raise PsgError(lib().psg_last_error().decode())
    return Z


def read_state3d(path: str, kind: str, record: int, n: int):
    """(meta[7], xii, eta, zet) of record `record` (1-based) of a restart file"""
    g = Grid3D(n)
    meta = np.zeros(7)
    out = [np.zeros(g.shape, np.complex128) for _ in range(3)]
    rc = _L().psg_read_state3d(path.encode(), kind.encode(), record, n, _dp(meta),
                               *[_dp(o) for o in out])
    if rc != 0:
        raise PsgError(lib().psg_last_error().decode())
    return (meta,) + tuple(out)


def driver_path(name: str = "psg_dns3") -> str:
    p = os.path.join(os.path.dirname(LIBDIR), "bin", name)
    if not os.path.exists(p):
        raise PsgError(f"driver {p} is not built (run python -m psgpu_b200.build)")
    return p
