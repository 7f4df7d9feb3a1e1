"""psg_ns2d_step_noalloc: the 2D step for callers that cannot allocate device
memory when they step -- a plugin inside a runtime that owns the GPU's memory,
code running during stream capture, a fixed-budget embedded driver.  Its
scratch is an array compiled into the library; the caller only hands over
device pointers to the state.  Checked against the batched entry point on the
same inputs, two calls in a row, through the C ABI, at every grid the array
holds; a long FP32 run checks that the carried rounding error matches the
batched FP32 engine's; and a call is shown to allocate no device memory.
This file is collected last."""
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


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("n", [16, 32, 64, 128])
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
    assert _rel(_to_host(dout, g.shape), _batch(Za, n, prec, nu, dt, 12)) < TOL[prec]
    # call 2: another state, in place, 7 steps; the scratch keeps call 1's contents
    Zb = kolmogorov_ic2d(n, 72)
    dz = _to_device(Zb, prec)
    rc = L.psg_ns2d_step_noalloc(n, prec, nu, dt, 7, C.c_void_p(dz.data_ptr()),
                                 C.c_void_p(dz.data_ptr()), None)
    assert rc == 0, L.psg_last_error()
    torch.cuda.synchronize()
    assert _rel(_to_host(dz, g.shape), _batch(Zb, n, prec, nu, dt, 7)) < TOL[prec]


def test_noalloc_fp32_long_run_carries_the_rounding_error():
    """500 FP32 steps: the batched FP32 engine carries each update's rounding
    error; so does this entry point.  Both start from the same FP32 values."""
    import torch
    L = P.lib()
    n, nu, dt, ns = 64, 1 / 40, 0.005, 500
    g = Grid2D(n)
    Z = kolmogorov_ic2d(n, 73)
    Z32 = Z.astype(np.complex64).astype(np.complex128)  # exactly representable in FP32
    dz = _to_device(Z32, 32)
    rc = L.psg_ns2d_step_noalloc(n, 32, nu, dt, ns, C.c_void_p(dz.data_ptr()),
                                 C.c_void_p(dz.data_ptr()), None)
    assert rc == 0, L.psg_last_error()
    torch.cuda.synchronize()
    ours = _to_host(dz, g.shape)
    ref32 = _batch(Z32, n, 32, nu, dt, ns)
    ref64 = _batch(Z32, n, 64, nu, dt, ns)
    # same arithmetic as the batched FP32 engine up to its final hi+lo sum
    assert _rel(ours, ref32) < 1e-6
    # and as close to FP64 as the batched FP32 engine is
    assert _rel(ours, ref64) < 3 * max(_rel(ref32, ref64), 1e-7)


def test_noalloc_allocates_no_device_memory():
    import torch
    L = P.lib()
    n = 128
    Z = kolmogorov_ic2d(n, 74)
    dz = _to_device(Z, 64)
    for _ in range(2):  # the first call sets up the array; later calls only launch
        assert L.psg_ns2d_step_noalloc(n, 64, 1 / 40, 0.005, 3, C.c_void_p(dz.data_ptr()),
                                       C.c_void_p(dz.data_ptr()), None) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for prec in (64, 32):
        d = dz if prec == 64 else _to_device(Z, 32)
        if prec == 32:
            torch.cuda.synchronize()
            free0, _ = torch.cuda.mem_get_info()
        assert L.psg_ns2d_step_noalloc(n, prec, 1 / 40, 0.005, 3, C.c_void_p(d.data_ptr()),
                                       C.c_void_p(d.data_ptr()), None) == 0
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (prec, free0 - free1)


def test_noalloc_rejects_grids_beyond_the_array():
    L = P.lib()
    rc = L.psg_ns2d_step_noalloc(256, 32, 1 / 40, 0.005, 1, C.c_void_p(1), C.c_void_p(1), None)
    assert rc != 0
    assert b"128" in L.psg_last_error()
