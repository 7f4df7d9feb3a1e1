"""The batched GPU Newton-GMRES-hookstep against the reference's algorithm, and
convergence onto unstable relative periodic orbits of turbulent Kolmogorov flow.

Fixture: tests/golden/upo2d_n32_re30.npz (made by tests/golden/make_upo2d.py):
two guesses found by a recurrence search of a 32^2, Re = 30 run, and the
orbits the restatement of the reference's solver (oracle/newton2d.py, FD Jv,
DGESDD) converged them to with the oracle step, NETOL = 1e-12.

* The GPU solver (exact tangent Jv in FP64 and in FP32, and the forward
  difference) converges both guesses to |F|/|Phi_T(z)| <= 1e-10 (the residual
  is FP64 in every form) and lands on the fixture's orbits:
  period and shift to 1e-7, state to 1e-5 (max-norm relative).  The orbits are
  unstable: a Floquet multiplier of modulus > 1.
* Decisions, step by step, exact Jv: the restatement driven by the GPU solver's
  own building blocks (Phi_T, tangent, dz/dt of psg_upo2d_apply) against the
  GPU solver's trace over three Newton steps: the same GMRES iteration counts,
  hookstep trial counts and trust radii; period, shift and residual to 1e-8.
* Decisions, step by step, FD Jv: the restatement driven by the reference's
  own CUDA step (oracle/_ref/libref_ns2d.so, one timestep_cuda_ call per
  integration, exactly as the reference's driver calls it) against the GPU
  solver in its FD mode over two Newton steps: the same counts and radii;
  period and shift to 1e-5, residual to 1e-3 relative (the 1/eps = 1e7
  difference quotient magnifies the two FP64 integrators' round-off).
"""
import os

import numpy as np
import pytest

import psgpu_b200 as P
from oracle import pyoracle as O
from oracle.newton2d import Newton2D
from psgpu_b200.floquet import floquet
from tests.golden_cases import relerr

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIX = os.path.join(ROOT, "tests", "golden", "upo2d_n32_re30.npz")
REF2D = os.path.join(ROOT, "oracle", "_ref", "libref_ns2d.so")


def _fix():
    d = dict(np.load(FIX))
    return {k: (v.item() if v.ndim == 0 else v) for k, v in d.items()}


def _guess(d, k):
    return (d[f"g{k}_Z"], float(d[f"g{k}_T"]), float(d[f"g{k}_sx"]), float(d[f"g{k}_sy"]),
            int(d[f"g{k}_rsym"]))


@pytest.mark.parametrize("form", ["exact64", "exact32", "fd"])
def test_converges_onto_the_fixture_orbits(form):
    d = _fix()
    n, nu, dt, G = int(d["n"]), 1.0 / float(d["re"]), float(d["dt"]), int(d["nguess"])
    exact = form != "fd"
    u = P.UPO2D(G, n, kmax=60, exact_jv=exact, jv_precision=32 if form == "exact32" else 64)
    for k in range(G):
        Z, T, sx, sy, rs = _guess(d, k)
        u.set_guess(k, Z, T=T, sx=sx, sy=sy, rsym=rs, nu=nu, dt=dt)
    u.solve(max_newton=40, tol=1e-10, gmres_tol=1e-3)
    for k in range(G):
        r = u.get(k)
        assert r["status"] == "CONVERGED", (k, r["status"], r["residual"])
        assert r["residual"] <= 1e-10
        assert abs(r["T"] - d[f"o{k}_T"]) < 1e-7
        dsx = (r["sx"] - d[f"o{k}_sx"] + np.pi) % (2 * np.pi) - np.pi
        assert abs(dsx) < 1e-7
        assert relerr(r["Z"], d[f"o{k}_Z"]) < 1e-5
    if form == "exact64":
        ev, _ = floquet(u, 0, k=24)
        assert np.abs(ev).max() > 1.0 + 1e-3  # unstable
    u.close()


def _gpu_blocks(n, nu):
    """Phi_T, tangent and dz/dt from the GPU solver's own integrator."""
    b = P.UPO2D(1, n, kmax=2, exact_jv=True)

    def phi(Z, T, dt):
        b.set_guess(0, Z, T=T, nu=nu, dt=dt)
        return b.apply(0, 1)[0]

    def tangent(Z, q, T, dt):
        b.set_guess(0, Z, T=T, nu=nu, dt=dt)
        return b.apply(0, 0, q)[1]

    def rhs(Z):
        b.set_guess(0, Z, T=1.0, nu=nu, dt=0.005)
        return b.apply(0, 2)[0]

    return b, phi, tangent, rhs


def _compare(steps, trace, nsteps, tol_T, tol_ner):
    assert len(trace) >= nsteps and len(steps) >= nsteps
    for s, t in zip(steps[:nsteps], trace[:nsteps]):
        assert t["gmres"] == s.gmres, (s.ine, t["gmres"], s.gmres)
        assert t["hook"] == s.hook, (s.ine, t["hook"], s.hook)
        assert t["delta"] == pytest.approx(s.delta, rel=1e-12), s.ine
        assert abs(t["T"] - s.T) < tol_T, (s.ine, t["T"], s.T)
        assert abs(t["sx"] - s.sx) < tol_T, (s.ine, t["sx"], s.sx)
        assert t["ner"] == pytest.approx(s.ner, rel=tol_ner), (s.ine, t["ner"], s.ner)


def test_decisions_match_the_restatement_exact_jv():
    d = _fix()
    n, nu, dt = int(d["n"]), 1.0 / float(d["re"]), float(d["dt"])
    Z, T, sx, sy, rs = _guess(d, 0)
    b, phi, tangent, rhs = _gpu_blocks(n, nu)
    ref = Newton2D(n, phi, rhs, tangent=tangent, gmresmax=60).solve(Z, T, sx, sy, rs, dt, 3)
    b.close()
    u = P.UPO2D(1, n, kmax=60, exact_jv=True)
    u.set_guess(0, Z, T=T, sx=sx, sy=sy, rsym=rs, nu=nu, dt=dt)
    u.solve(max_newton=3, tol=1e-12, gmres_tol=1e-3)
    _compare(ref.steps, u.trace(0), 3, 1e-8, 1e-8)
    u.close()


def test_decisions_match_the_reference_step_fd_jv():
    if not os.path.exists(REF2D):
        pytest.skip("reference 2D step not built (oracle/build_ref.sh)")
    from psgpu_b200.abi import TimestepLibrary
    d = _fix()
    n, nu, dt = int(d["n"]), 1.0 / float(d["re"]), float(d["dt"])
    Z, T, sx, sy, rs = _guess(d, 0)
    ref_lib = TimestepLibrary(REF2D, "ns2d")

    def phi(z, t, truedelt):
        ns = int(t / truedelt)
        return ref_lib.ns2d(z, n, nu, t / ns, ns)[0]

    def rhs(z):
        return O.ns2d_timederiv(z, n, nu)

    ref = Newton2D(n, phi, rhs, gmresmax=60).solve(Z, T, sx, sy, rs, dt, 2)
    u = P.UPO2D(1, n, kmax=60, exact_jv=False)
    u.set_guess(0, Z, T=T, sx=sx, sy=sy, rsym=rs, nu=nu, dt=dt)
    u.solve(max_newton=2, tol=1e-12, gmres_tol=1e-3)
    _compare(ref.steps, u.trace(0), 2, 1e-5, 1e-3)
    u.close()


def test_fp32_tangent_matches_fp64():
    """The FP32 exact tangent (jv_precision 32) against the FP64 one over a
    period (T = 20, 4000 steps) of the unstable fixture orbit: relative L2
    difference below 2e-3 (measured 6.1e-4 on a B200), inside the GMRES
    tolerance of 1e-3 that the Krylov products serve."""
    d = _fix()
    n, nu, dt = int(d["n"]), 1.0 / float(d["re"]), float(d["dt"])
    Z, T = d["o0_Z"], float(d["o0_T"])
    rng = np.random.default_rng(4)
    m = P.Grid2D(n).mask()
    q = (rng.standard_normal(m.shape) + 1j * rng.standard_normal(m.shape)) * m
    out = {}
    for prec in (64, 32):
        u = P.UPO2D(1, n, kmax=2, exact_jv=True, jv_precision=prec)
        u.set_guess(0, Z, T=T, nu=nu, dt=dt)
        out[prec] = u.apply(0, 0, q)[1]
        u.close()
    rel = np.linalg.norm(out[32] - out[64]) / np.linalg.norm(out[64])
    assert rel < 2e-3, rel
