"""The restatement of the reference's Newton-GMRES-hookstep (oracle/newton2d.py)
pinned on the host, without a GPU.

* It converges a perturbed laminar Kolmogorov state at Re = 5 to the laminar
  fixed point (omega = -2/(nu kf^2) at (0, kf); the Newton solve for a
  "periodic orbit" of a steady state must give NER <= 1e-12), with the
  reference's forward-difference Jv on the oracle step.
* The committed orbits of tests/golden/upo2d_n32_re30.npz are fixed points of
  the oracle's period map: shift(Phi_T(z)) = z to 1e-11 relative.
* The first Newton step from the first committed guess reproduces the
  recorded one: the same GMRES iteration and hookstep trial counts, the same
  trust radius, the same residual to 1e-9.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from oracle.newton2d import Newton2D, grid2d

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIX = os.path.join(ROOT, "tests", "golden", "upo2d_n32_re30.npz")


def _blocks(n, nu):
    def phi(z, t, dt):
        ns = int(t / dt)
        return O.ns2d_timestep(z, n, nu, t / ns, ns)[0]

    def rhs(z):
        return O.ns2d_timederiv(z, n, nu)

    return phi, rhs


def test_laminar_state_converges():
    n, nu, kf = 16, 1 / 5.0, 4
    kx, ky, LL = grid2d(n)
    rng = np.random.default_rng(1)
    Z = 0.01 * (rng.standard_normal(LL.shape) + 1j * rng.standard_normal(LL.shape)) * LL
    Z[n // 3 + kf, 0] += -2.0 / (nu * kf * kf)
    phi, rhs = _blocks(n, nu)
    r = Newton2D(n, phi, rhs, gmresmax=40).solve(Z, T=2.0, dt=0.01, max_newton=10)
    assert r.status == "CONVERGED" and r.ner <= 1e-12
    # quadratic convergence near the solution
    ners = [s.ner for s in r.steps]
    assert ners[-1] < 1e-3 * ners[-2]


def _fix():
    d = dict(np.load(FIX))
    return {k: (v.item() if v.ndim == 0 else v) for k, v in d.items()}


def test_committed_orbits_are_fixed_points_of_the_oracle():
    d = _fix()
    n, nu = int(d["n"]), 1.0 / float(d["re"])
    kx, ky, LL = grid2d(n)
    phi, _ = _blocks(n, nu)
    for k in range(int(d["nguess"])):
        Z, T, sx = d[f"o{k}_Z"], float(d[f"o{k}_T"]), float(d[f"o{k}_sx"])
        sy, rs = float(d[f"g{k}_sy"]), int(d[f"g{k}_rsym"])
        ZT = phi(Z, T, float(d["dt"]))
        src = np.conj(ZT[::-1, :]) if rs else ZT
        S = np.exp(-1j * kx * sx) * np.exp(-1j * ky * sy) * src * LL
        ner = np.sqrt(np.sum(np.abs(S - Z) ** 2)) / np.sqrt(np.sum(np.abs(ZT) ** 2))
        assert ner < 1e-11, (k, ner)
    if int(d["nguess"]) > 1:
        assert abs(float(d["o0_T"]) - float(d["o1_T"])) > 1e-4  # two distinct orbits


def test_first_newton_step_reproduces_the_fixture():
    d = _fix()
    n, nu, dt = int(d["n"]), 1.0 / float(d["re"]), float(d["dt"])
    phi, rhs = _blocks(n, nu)
    r = Newton2D(n, phi, rhs, gmresmax=60, netol=1e-12).solve(
        d["g0_Z"], float(d["g0_T"]), float(d["g0_sx"]), float(d["g0_sy"]), int(d["g0_rsym"]),
        dt, max_newton=1)
    s = r.steps[0]
    assert s.gmres == int(d["o0_trace_gmres"][0])
    assert s.hook == int(d["o0_trace_hook"][0])
    assert s.delta == float(d["o0_trace_delta"][0])
    assert s.ner == pytest.approx(float(d["o0_trace_ner"][0]), rel=1e-9)
    assert s.T == pytest.approx(float(d["o0_trace_T"][0]), rel=1e-12)
