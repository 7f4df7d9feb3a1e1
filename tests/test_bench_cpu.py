"""bench.py's host-side arithmetic, checked without a GPU: the algorithmic bytes
of the 256^3 passes (the roofline's numerators), the RK4 step count of a
Boussinesq call, the nominal FFT flops of the 2D ensemble, and the kept-mode
count that the drop-in's end-to-end byte report uses."""
import math

import numpy as np
import pytest

import bench
from psgpu_b200.fields import Grid3D


def test_pass_bytes_256_fp32():
    mb = [round(x / 1e6, 1) for x in bench.algorithmic_bytes(256, 8)]
    # z-inverse, y-inverse, x-pass, y-forward: one read and one write of the
    # kept modes; the last entry is the z-forward's transform input
    assert mb[:4] == [241.1, 451.2, 405.8, 225.6]
    X, Y, N = 86, 171, 256
    assert bench.algorithmic_bytes(256, 8)[0] == 8 * (3 * X * Y * Y + 6 * X * Y * N)


def test_rk4_evaluations_follow_the_reference_loop():
    # full steps while tend - t > dt, then one step of the remainder
    assert bench.rk4_evaluations(0.0, 0.01, 1e-3) == 10
    assert bench.rk4_evaluations(0.0, 0.0105, 1e-3) == 11
    assert bench.rk4_evaluations(0.0, 0.0, 1e-3) == 0


def test_ensemble_flops():
    f = bench.ensemble_flops([64, 128, 256], 3)
    want = 3 * sum(4 * 5 * 2.5 * n * n * math.log2(n * n) for n in (64, 128, 256))
    assert f == pytest.approx(want, rel=1e-15)
    assert bench.ensemble_flops([], 5) == 0


def test_kept_mode_count_256():
    m = Grid3D(256).mask()
    assert int(m.sum()) == 1263714
    # four FP64 complex fields each way per 10-step call, per step (the bench's
    # h2d_bytes_per_step / d2h_bytes_per_step on the kept path)
    assert int(4 * int(m.sum()) * 16 / 10) == 8087769
    assert np.count_nonzero(~m) == Grid3D(256).nkt - 1263714
