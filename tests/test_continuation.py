"""Arc-length continuation in nu, on the host (no GPU).

* The restatement's pseudo-arclength corrector (oracle/newton2d.py with
  `arc`, the reference's arclcFLAG2 branches of 2D_NavierStokes/src_RK4/
  src_gmres/main.F90) on the oracle step follows the laminar branch of
  Kolmogorov flow, omega(0, kf) = -2/(nu kf^2): from a perturbed first-order
  prediction it converges to the point of the branch that the arc equation
  picks, state and nu to 1e-9, and the arc equation holds.
* The continuation driver (psgpu_b200/continuation.py) around a stand-in
  solver whose converged points lie on a known smooth branch: the natural
  first step lands at nu - delta_v2; every later point satisfies its arc
  equation; the step control doubles the last secant on the second step,
  grows by 10 % up to the largest step taken and halves after a failed
  corrector, keeping the history; a failed first step halves delta_v2.
"""
import math

import numpy as np
import pytest

import psgpu_b200.continuation as CT
from oracle import pyoracle as O
from oracle.newton2d import Newton2D, grid2d
from psgpu_b200.fields import Grid2D


def _blocks(n):
    def phi(z, t, dt, nu):
        ns = int(t / dt)
        return O.ns2d_timestep(z, n, nu, t / ns, ns)[0]

    def rhs(z, nu):
        return O.ns2d_timederiv(z, n, nu)

    return phi, rhs


def test_oracle_arc_corrector_follows_the_laminar_branch():
    n, kf = 16, 4
    K = n // 3
    kx, ky, LL = grid2d(n)

    def lam(nu):
        z = np.zeros(LL.shape, np.complex128)
        z[K + kf, 0] = -2.0 / (nu * kf * kf)
        return z

    nu1, nu2, T = 0.2, 0.19, 0.5
    Z1, Z2 = lam(nu1), lam(nu2)
    dZ = Z2 - Z1
    dr2 = math.sqrt(float(np.sum(np.abs(dZ[LL]) ** 2)) + (nu2 - nu1) ** 2)
    dzr, dvr = dZ / dr2, (nu2 - nu1) / dr2
    ndelta = 2.0 * dr2
    rng = np.random.default_rng(7)
    Zp = Z2 + dzr * ndelta + 1e-3 * (rng.standard_normal(LL.shape) + 1j * rng.standard_normal(
        LL.shape)) * LL
    vp = nu2 + dvr * ndelta
    arc = dict(dZrdr=dzr, Zr2=Z2, dTrdr=0.0, dSrdr=0.0, dv2rdr=dvr, Tr2=T, Sr2=0.0, v2r2=nu2,
               ndelta=ndelta)
    phi, rhs = _blocks(n)
    r = Newton2D(n, phi, rhs, gmresmax=40).solve(Zp, T=T, dt=0.01, max_newton=12, nu=vp, arc=arc)
    assert r.status == "CONVERGED", (r.status, r.ner)

    # the point of the branch on the arc: <dzr, lam(v) - Z2> + dvr (v - nu2) = ndelta
    def g(v):
        return float(np.sum((np.conj(dzr) * (lam(v) - Z2)).real[LL])) + dvr * (v - nu2) - ndelta

    lo, hi = nu2 - 0.1, nu2
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if g(mid) > 0:
            lo = mid
        else:
            hi = mid
    v_star = 0.5 * (lo + hi)
    assert abs(r.nu - v_star) < 1e-9 * v_star
    assert np.abs(r.Z - lam(v_star)).max() < 1e-9 * np.abs(lam(v_star)).max()
    assert abs(g(r.nu)) < 1e-9
    assert [s.nu for s in r.steps][-1] == r.nu


# ------------------------------------------------------------- the driver
class _Branch:
    """z(s), T(s), shift(s), nu(s) along a smooth curve"""

    def __init__(self, n):
        g = Grid2D(n)
        self.mask = g.mask()
        rng = np.random.default_rng(3)
        self.a, self.b, self.c = [
            (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * self.mask * w
            for w in (1.0, 0.05, 0.01)]

    def at(self, s):
        return (self.a + s * self.b + s * s * self.c, 5.0 + 0.1 * s + 0.02 * s * s, 0.05 * s,
                0.04 - 0.002 * s - 0.0002 * s * s)

    def project(self, Z):
        m = self.mask
        return float(np.sum((np.conj(self.b) * (Z - self.a)).real[m]) /
                     np.sum(np.abs(self.b[m]) ** 2))


class _FakeUPO:
    """Stands in for UPO2D: 'converges' each guess to the branch point its
    equations pick (fixed nu without an arc, the arc equation with one)."""
    branch = None
    fail_calls = ()

    def __init__(self, nguess, n, **kw):
        self.grid = Grid2D(n)
        self.G = [dict() for _ in range(nguess)]
        self.calls = 0
        self.log = []

    def close(self):
        pass

    def set_guess(self, i, Z, T, sx=0.0, sy=0.0, rsym=0, nu=0.0, dt=0.005):
        self.G[i] = {"Z": np.array(Z), "T": T, "sx": sx, "nu": nu, "arc": None}

    def set_arc(self, i, dZrdr, Zr2, dTrdr, dSrdr, dv2rdr, Tr2, Sr2, v2r2, ndelta):
        self.G[i]["arc"] = (np.array(dZrdr), np.array(Zr2), dTrdr, dSrdr, dv2rdr, Tr2, Sr2,
                            v2r2, ndelta)

    @staticmethod
    def _solve_s(f, s0):
        # scalar Newton from the guess's projection onto the branch: the root nearest the guess
        s = s0
        for _ in range(60):
            h = 1e-6
            d = (f(s + h) - f(s - h)) / (2 * h)
            s -= f(s) / d
        assert abs(f(s)) < 1e-11
        return s

    def solve(self, max_newton=30, tol=1e-10, gmres_tol=1e-3):
        B, m = self.branch, self.grid.mask()
        self.calls += 1
        for g in self.G:
            g["ok"] = self.calls not in self.fail_calls
            self.log.append((self.calls, g["nu"], g["arc"] is not None and g["arc"][8]))
            s0 = B.project(g["Z"])
            if g["arc"] is None:
                s = self._solve_s(lambda s: B.at(s)[3] - g["nu"], s0)
            else:
                dz, z2, dT, dS, dv, T2, S2, v2, nd = g["arc"]

                def f(s):
                    Z, T, S, v = B.at(s)
                    return (float(np.sum((np.conj(dz) * (Z - z2)).real[m])) + dT * (T - T2)
                            + dS * (S - S2) + dv * (v - v2) - nd)

                s = self._solve_s(f, s0)
            g["s"] = s
            g["Z"], g["T"], g["sx"], g["nu"] = B.at(s)

    def get(self, i):
        g = self.G[i]
        return {"Z": g["Z"], "T": g["T"], "sx": g["sx"], "residual": 0.0, "newton": 1,
                "status": "CONVERGED" if g["ok"] else "NEWTON FAILED"}

    def nu(self, i):
        return self.G[i]["nu"]


def _driver(monkeypatch, fail_calls=(), delta_v2=0.001, **kw):
    n = 16
    B = _Branch(n)
    _FakeUPO.branch, _FakeUPO.fail_calls = B, fail_calls
    monkeypatch.setattr(CT, "UPO2D", _FakeUPO)
    Z0, T0, S0, v0 = B.at(0.0)
    c = CT.Continuation2D(n, [{"Z": Z0, "T": T0, "sx": S0, "nu": v0}], dt=0.01, delta_v2=delta_v2,
                          **kw)
    return c, B


def _arc_residual(c, b, pt, B):
    # the arc equation at the point the corrector returned
    (Z1, T1, S1, v1), (Z2, T2, S2, v2) = b["hist"][0], b["hist"][1]
    m = c.mask
    d = Z2 - Z1
    dr = math.sqrt(float(np.sum(np.abs(d[m]) ** 2)) + (S2 - S1) ** 2 + (v2 - v1) ** 2 +
                   (T2 - T1) ** 2)
    return (float(np.sum((np.conj(d / dr) * (pt["Z"] - Z2)).real[m])) + (T2 - T1) / dr *
            (pt["T"] - T2) + (S2 - S1) / dr * (pt["sx"] - S2) + (v2 - v1) / dr * (pt["nu"] - v2)
            - b["delta_r2"])


def test_driver_follows_a_smooth_branch(monkeypatch):
    c, B = _driver(monkeypatch, first_order=True)
    b = c.B[0]
    p1 = c.step()[0]
    assert p1["nu"] == pytest.approx(0.04 - 0.001, abs=1e-12)  # natural first step
    assert b["second"] and not b["first"]
    secants = []
    for k in range(5):
        pt = c.step()[0]
        assert pt is not None
        # first-order corrector: the arc equation along the secant tangent
        assert abs(_arc_residual(c, b, pt, B)) < 1e-9
        secants.append(b["delta_r2"])
        if k == 0:
            # second run: Ndelta_r = 2 x the secant of the natural step
            assert b["ndelta_max"] == pytest.approx(b["delta_r2"])
    nus = [p["nu"] for p in b["points"]]
    assert all(x > y for x, y in zip(nus, nus[1:]))  # moving down in nu along the branch
    # step sizes never exceed the largest one taken
    assert max(secants) <= b["ndelta_max"] * (1 + 1e-12)
    c.close()


def test_second_order_prediction_is_closer(monkeypatch):
    errs = {}
    for first in (True, False):
        # short steps: the quadratic extrapolation's gain grows as the step shrinks
        c, B = _driver(monkeypatch, first_order=first, delta_v2=0.0001)
        for _ in range(4):
            c.step()
        b = c.B[0]
        c._prepare(0, b)  # the next prediction
        g = c.upo.G[0]
        pred = np.concatenate([g["Z"][c.mask], [g["T"], g["sx"], g["nu"]]])
        c.upo.solve()
        r = c.upo.get(0)
        corr = np.concatenate([r["Z"][c.mask], [r["T"], r["sx"], c.upo.nu(0)]])
        errs[first] = np.linalg.norm(pred - corr)
        c.close()
    assert errs[False] < 0.2 * errs[True], errs


def test_driver_step_control_after_failures(monkeypatch):
    # solve calls: 1 natural step, 2 second run, 3 fails, 4 retried, 5 fails, 6 retried
    c, B = _driver(monkeypatch, fail_calls=(3, 5))
    b = c.B[0]
    c.step()
    c.step()
    hist = [h[3] for h in b["hist"][1:]]
    nd_max = b["ndelta_max"]
    assert c.step()[0] is None  # failed corrector: history kept
    assert [h[3] for h in b["hist"][1:]] == hist
    nd_fail = b["ndelta"]
    assert c.step()[0] is not None
    assert b["ndelta"] == pytest.approx(nd_fail / 2.0)  # halved after the failure
    assert b["ndelta_max"] == nd_max
    assert c.step()[0] is None
    nd_fail = b["ndelta"]
    assert c.step()[0] is not None
    assert b["ndelta"] == pytest.approx(nd_fail / 2.0)
    c.close()


def test_failed_natural_step_halves_delta_v2(monkeypatch):
    c, B = _driver(monkeypatch, fail_calls=(1,))
    b = c.B[0]
    assert c.step()[0] is None
    assert b["first"]
    p = c.step()[0]
    # v2 = v0 - delta_v2, then after the failure v2 + delta_v2 - delta_v2 / 2
    assert p["nu"] == pytest.approx(0.04 - 0.0005, abs=1e-12)
    assert b["delta_v2"] == 0.0005
    c.close()
