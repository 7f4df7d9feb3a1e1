"""The batched 2D engine's graph launch and autotuner.

* set_params + launch (a captured CUDA graph, replayed) gives bit-identical
  states to run();
* the autotuner (block size, then each grid size's transform schedule) leaves
  every instance's state as it found it, and every block size gives
  bit-identical results for the same schedule (the line transforms do not
  depend on how lines are assigned to thread groups);
* the packed f32x2 schedule of every size agrees with the scalar one to 1e-5
  (max-norm relative) after 20 steps: the same transforms, rounded in another
  order; an FP64 batch refuses packed sizes;
* a mixed FP32 ensemble after many steps stays within 1e-4 of the FP64 engine.
"""
import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.fields import kolmogorov_ic2d

pytestmark = pytest.mark.gpu

SIZES = [64, 128, 256, 32, 128, 64, 16, 256]


def _batch(prec=32):
    b = P.Batch2D(SIZES, precision=prec)
    for i, n in enumerate(SIZES):
        b.upload(i, kolmogorov_ic2d(n, 30 + i))
    return b


def _params():
    rng = np.random.default_rng(8)
    nu = 1.0 / rng.uniform(20, 100, len(SIZES))
    return nu, np.full(len(SIZES), 0.005), np.full(len(SIZES), 20, np.int32)


def test_graph_launch_matches_run():
    nu, dt, ns = _params()
    a, b = _batch(), _batch()
    for _ in range(2):
        a.run(nu, dt, ns)
    b.set_params(nu, dt, ns)
    b.launch()
    b.launch()
    a.sync(); b.sync()
    for i in range(len(SIZES)):
        np.testing.assert_array_equal(a.download(i), b.download(i))


def test_autotune_restores_state_and_variants_agree():
    nu, dt, ns = _params()
    b = _batch()
    before = [b.download(i) for i in range(len(SIZES))]
    b.set_params(nu, dt, ns)
    v, ms = b.autotune()
    assert 0 <= v < 3 and ms[v] > 0
    for i in range(len(SIZES)):
        np.testing.assert_array_equal(b.download(i), before[i])
    sched = b.schedule()
    assert set(sched) == {16, 32, 64, 128, 256}
    for n in set(SIZES):
        assert sched[n][1][0] > 0 and sched[n][1][1] > 0  # both schedules timed
    b.launch(); b.sync()
    ref = _batch()
    ref.set_schedule({n: sched[n][0] for n in sched})
    ref.run(nu, dt, ns); ref.sync()
    for i in range(len(SIZES)):
        np.testing.assert_array_equal(b.download(i), ref.download(i))


def test_packed_schedule_matches_scalar():
    nu, dt, ns = _params()
    out = {}
    for packed in (False, True):
        b = _batch()
        b.set_schedule(set(SIZES) if packed else set())
        b.run(nu, dt, ns); b.sync()
        out[packed] = [b.download(i) for i in range(len(SIZES))]
    for i in range(len(SIZES)):
        a, c = out[True][i], out[False][i]
        assert np.isfinite(a).all()
        assert np.max(np.abs(a - c)) / np.max(np.abs(c)) < 1e-5, (i, SIZES[i])
    b64 = _batch(64)
    with pytest.raises(P.PsgError):
        b64.set_schedule({128})


def test_fp32_ensemble_tracks_fp64():
    nu, dt, _ = _params()
    ns = np.full(len(SIZES), 400, np.int32)
    r = {}
    for prec in (64, 32):
        b = _batch(prec)
        b.run(nu, dt, ns); b.sync()
        r[prec] = [b.download(i) for i in range(len(SIZES))]
    for i in range(len(SIZES)):
        err = np.max(np.abs(r[32][i] - r[64][i])) / np.max(np.abs(r[64][i]))
        assert err < 1e-4, (i, SIZES[i], err)
