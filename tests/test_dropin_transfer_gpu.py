"""Host transfer of the Boussinesq drop-in (libpsg_bous3d.so).

An in-place call on page-locked state arrays whose entries outside the kept
modes are zero moves only the kept modes (the conversion kernels read and write
the host arrays directly); any other call copies the whole boxes.  Both paths
must return the same state bit for bit:

* page-locked, clean input (kept path) against pageable copies of it (whole-box
  path), FP64 and FP32 engines, two calls in a row;
* page-locked input with one non-kept entry set (the call falls back to the
  whole box after its host check) against the pageable call on the same input;
* PSG_DROPIN_FULL_COPY=1 on page-locked input against the kept path;
* the non-kept entries of every output are zero.
"""
import os

import numpy as np
import pytest
import torch

import psgpu_b200 as P
from psgpu_b200.abi import TimestepLibrary
from psgpu_b200.fields import Grid3D, taylor_green3d

pytestmark = pytest.mark.gpu

N, NU, DT = 32, 1.0 / 400.0, 2e-3


def _pinned(a):
    t = torch.empty(a.size * 2, dtype=torch.float64, pin_memory=True)
    v = t.numpy().view(np.complex128).reshape(a.shape)
    v[...] = a
    return v, t


def _state(dirty):
    xi, et, zt = taylor_green3d(N, 5, amp=1e-2)
    comps = [xi, et, zt, 0.1 * xi]
    if dirty:
        g = Grid3D(N)
        m = g.mask()
        idx = np.argwhere(~m)[7]
        comps[1] = comps[1].copy()
        comps[1][tuple(idx)] = 0.25 + 0.5j
    return comps


def _call(lib, comps):
    lib.bous3d_inplace(comps, N, NU, DT, 5 * DT + 0.5 * DT, ri=1.0)


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("dirty", [False, True])
def test_kept_transfer_matches_whole_box(prec, dirty):
    os.environ["PSG_PRECISION"] = str(prec)
    try:
        lib = TimestepLibrary(P.dropin_path("bous3d"), "bous3d")
        src = _state(dirty)
        pinned = [_pinned(a) for a in src]
        pin = [p[0] for p in pinned]
        page = [a.copy() for a in src]
        for _ in range(2):
            _call(lib, pin)
            _call(lib, page)
            for a, b in zip(pin, page):
                assert np.array_equal(a, b)
        m = Grid3D(N).mask()
        for a in pin:
            assert np.isfinite(a).all()
            assert not np.any(a[~m])
        if not dirty:
            os.environ["PSG_DROPIN_FULL_COPY"] = "1"
            try:
                again = [_pinned(a) for a in src]
                full = [p[0] for p in again]
                _call(lib, full)
                _call(lib, full)
            finally:
                os.environ.pop("PSG_DROPIN_FULL_COPY", None)
            for a, b in zip(full, pin):
                assert np.array_equal(a, b)
    finally:
        os.environ.pop("PSG_PRECISION", None)
