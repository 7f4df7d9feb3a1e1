"""The UPO solver's building blocks and a converging Newton-GMRES-hookstep run.

* dz/dt against the oracle's restatement of TIMEDERIV (FP64; the reference
  driver builds nu k^2 as 10**(log10 nu + 2 log10 |k|), identical to round-off);
* Phi_T(z) of the FP64 integrator against the oracle step;
* the exact tangent dPhi_T(z) q against central differences of the oracle step
  (truncation O(eps^2) = 1e-10 with eps = 1e-5), and its linearity;
* Newton-GMRES-hookstep from a perturbed laminar state at Re = 5 (stable laminar
  flow) reaching |F|/|Phi_T(z)| <= 1e-10 with exact and finite-difference Jv.
"""
import numpy as np
import pytest

import psgpu_b200 as P
from oracle import pyoracle as O
from psgpu_b200.fields import Grid2D, kolmogorov_ic2d
from tests.golden_cases import relerr

pytestmark = pytest.mark.gpu


def _masked_random(n, seed, amp=1.0):
    g = Grid2D(n)
    rng = np.random.default_rng(seed)
    q = (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * g.mask()
    return amp * q / np.sqrt(np.sum(np.abs(q) ** 2))


def test_timederiv_matches_oracle():
    n, nu = 32, 1 / 40
    Z = kolmogorov_ic2d(n, 3)
    u = P.UPO2D(1, n, kmax=4)
    u.set_guess(0, Z, T=0.1, nu=nu, dt=0.005)
    d, _ = u.apply(0, 2)
    ref = O.ns2d_timederiv(Z, n, nu)
    assert relerr(d, ref) < 1e-12


def test_phi_matches_oracle():
    n, nu, dt, T = 32, 1 / 40, 0.005, 0.2
    Z = kolmogorov_ic2d(n, 4)
    u = P.UPO2D(1, n, kmax=4)
    u.set_guess(0, Z, T=T, nu=nu, dt=dt)
    phi, _ = u.apply(0, 1)
    ref, _ = O.ns2d_timestep(Z, n, nu, dt, int(round(T / dt)))
    assert relerr(phi, ref) < 1e-12


def test_tangent_matches_central_differences():
    n, nu, dt, T = 32, 1 / 40, 0.005, 0.2
    ns = int(round(T / dt))
    Z = kolmogorov_ic2d(n, 5) * 3.0
    q = _masked_random(n, 6)
    u = P.UPO2D(1, n, kmax=4)
    u.set_guess(0, Z, T=T, nu=nu, dt=dt)
    _, jq = u.apply(0, 0, q)
    eps = 1e-5
    zp, _ = O.ns2d_timestep(Z + eps * q, n, nu, dt, ns)
    zm, _ = O.ns2d_timestep(Z - eps * q, n, nu, dt, ns)
    fd = (zp - zm) / (2 * eps)
    assert relerr(jq, fd) < 1e-7
    _, j2 = u.apply(0, 0, 2.0 * q)
    assert relerr(j2, 2.0 * jq) < 1e-14


@pytest.mark.parametrize("exact", [True, False], ids=["exact-jv", "fd-jv"])
def test_newton_converges_to_laminar_state(exact):
    n, nu, dt = 32, 1 / 5, 0.005
    g = Grid2D(n)
    K = g.kt
    lam = np.zeros(g.shape, np.complex128)
    lam[K + 4, 0] = -0.125 / nu
    Z = lam + _masked_random(n, 7, amp=0.05)
    u = P.UPO2D(2, n, kmax=30, exact_jv=exact)
    u.set_guess(0, Z, T=1.0, nu=nu, dt=dt)
    u.set_guess(1, lam + _masked_random(n, 8, amp=0.02), T=0.75, nu=nu, dt=dt)
    u.solve(max_newton=20, tol=1e-10)
    for i in range(2):
        r = u.get(i)
        assert r["status"] == "CONVERGED", r
        assert r["residual"] <= 1e-10
        assert relerr(r["Z"], lam) < 1e-8


@pytest.mark.parametrize("n", [64, 128])
def test_cluster_sizes_give_the_same_integration(n, monkeypatch):
    """One, two or four blocks per guess (PSG_UPO_CLUSTER) split the same
    per-column and per-row work differently: Phi_T(z) and the exact tangent
    must come out bit for bit the same."""
    nu, dt, T = 1 / 40, 0.005, 0.1
    Z = kolmogorov_ic2d(n, 7) * 2.0
    q = _masked_random(n, 8)
    out = {}
    for cs in ("1", "2", "4"):
        monkeypatch.setenv("PSG_UPO_CLUSTER", cs)
        u = P.UPO2D(2, n, kmax=4)
        u.set_guess(0, Z, T=T, nu=nu, dt=dt)
        u.set_guess(1, Z, T=T, nu=nu, dt=dt)
        out[cs] = u.apply(1, 0, q)
    for cs in ("2", "4"):
        np.testing.assert_array_equal(out[cs][0], out["1"][0])
        np.testing.assert_array_equal(out[cs][1], out["1"][1])


def test_mixed_cluster_sizes_in_one_batch(monkeypatch):
    """64 guesses with periods spread over a factor of six: with clusters
    allowed, the longest guesses get four blocks, the middle two and the
    shortest one, in three concurrent launches; one Newton iteration of the
    whole batch must give bit for bit what one block per guess gives."""
    n, nu, dt, ng = 32, 1 / 40, 0.005, 64
    rng = np.random.default_rng(21)
    periods = rng.uniform(0.05, 0.3, ng)
    starts = [kolmogorov_ic2d(n, 100 + i) * 2.0 for i in range(ng)]
    res = {}
    for cs in ("1", "4"):
        monkeypatch.setenv("PSG_UPO_CLUSTER", cs)
        u = P.UPO2D(ng, n, kmax=6)
        for i in range(ng):
            u.set_guess(i, starts[i], T=float(periods[i]), nu=nu, dt=dt)
        u.solve(max_newton=1, tol=1e-10)
        res[cs] = [u.get(i) for i in range(ng)]
        u.close()
    for a, b in zip(res["4"], res["1"]):
        np.testing.assert_array_equal(a["Z"], b["Z"])
        assert (a["T"], a["sx"], a["residual"], a["gmres"]) == (b["T"], b["sx"], b["residual"], b["gmres"])
