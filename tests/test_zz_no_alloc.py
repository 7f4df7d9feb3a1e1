"""psg_ns2d_step_noalloc: the 2D step for callers that cannot allocate device
memory (a plugin inside a runtime that owns the GPU's memory, code running
during stream capture, a fixed-budget embedded driver).  Its scratch is an
array compiled into the library; the caller only hands over device pointers
to the state.  Checked against the batched entry point on the same inputs,
two calls in a row, through the C ABI.  This file is collected last."""
import ctypes as C

import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.fields import Grid2D, kolmogorov_ic2d

pytestmark = pytest.mark.gpu

TOL = {64: 1e-10, 32: 2e-5}


def _to_device(Z, prec):
    import torch
    dt = torch.float64 if prec == 64 else torch.float32
    a = np.ascontiguousarray(Z, np.complex128).view(np.float64).ravel()
    return torch.tensor(a, dtype=dt, device="cuda")


def _to_host(t, shape):
    a = t.detach().to("cpu").double().numpy()
    return a.view(np.complex128).reshape(shape)


def _batch(Z, n, prec, nu, dt, ns):
    b = P.Batch2D([n], precision=prec)
    b.upload(0, Z)
    b.run(nu, dt, ns)
    out = b.download(0)
    b.close()
    return out


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("n", [32, 128])
def test_noalloc_matches_batched_entry_point(n, prec):
    import torch
    L = P.lib()
    g = Grid2D(n)
    nu, dt = 1 / 40, 0.005
    # call 1: out-of-place, 12 steps
    Za = kolmogorov_ic2d(n, 71)
    din = _to_device(Za, prec)
    dout = torch.zeros_like(din)
    rc = L.psg_ns2d_step_noalloc(n, prec, nu, dt, 12, C.c_void_p(din.data_ptr()),
                                 C.c_void_p(dout.data_ptr()), None)
    assert rc == 0, L.psg_last_error()
    torch.cuda.synchronize()
    ref = _batch(Za, n, prec, nu, dt, 12)
    err = np.abs(_to_host(dout, g.shape) - ref).max() / np.abs(ref).max()
    assert err < TOL[prec]
    # call 2: another state, in place, 7 steps; the scratch keeps call 1's contents
    Zb = kolmogorov_ic2d(n, 72)
    dz = _to_device(Zb, prec)
    rc = L.psg_ns2d_step_noalloc(n, prec, nu, dt, 7, C.c_void_p(dz.data_ptr()),
                                 C.c_void_p(dz.data_ptr()), None)
    assert rc == 0, L.psg_last_error()
    torch.cuda.synchronize()
    ref = _batch(Zb, n, prec, nu, dt, 7)
    err = np.abs(_to_host(dz, g.shape) - ref).max() / np.abs(ref).max()
    assert err < TOL[prec]


def test_noalloc_rejects_grids_beyond_the_array():
    L = P.lib()
    rc = L.psg_ns2d_step_noalloc(256, 32, 1 / 40, 0.005, 1, C.c_void_p(1), C.c_void_p(1), None)
    assert rc != 0
    assert b"128" in L.psg_last_error()
