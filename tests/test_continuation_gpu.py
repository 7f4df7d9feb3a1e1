"""Arc-length continuation in nu on the batched GPU solver, from the unstable
periodic orbits of tests/golden/upo2d_n32_re30.npz (32^2, Re = 30).

* One pseudo-arclength corrector (the reference's arclcFLAG2 path of
  2D_NavierStokes/src_RK4/src_gmres/main.F90), step by step against the
  restatement (oracle/newton2d.py with `arc`):
  - exact Jv: the restatement driven by the GPU solver's own Phi_T, tangent
    and dz/dt at the viscosity each call asks for, over three Newton steps:
    the same GMRES and hookstep counts and trust radii, period, shift and
    residual to 1e-7, nu to 1e-10 (dPhi_T/dnu is a central difference over
    nu (1 +- 1e-5): the two sides round its cancellation differently, about
    1e-11 relative, which the residual carries at 2e-8 on a B200);
  - FD Jv: the restatement driven by the reference's own CUDA step
    (oracle/_ref/libref_ns2d.so, v2 passed per call as the reference's
    driver does) over two Newton steps: the same counts and radii, period,
    shift to 1e-5, residual to 1e-3 relative, nu to 1e-7 relative (the
    1/eps = 1e7 difference quotient magnifies the two integrators'
    round-off; 6e-9 measured).
* Continuation of both fixture orbits at once (one batched solve per step)
  over a natural step and two pseudo-arclength steps: every point converges
  to |F|/|Phi_T(z)| <= 1e-10, is a periodic orbit at its own nu
  (shift(Phi_T(z)) = z to 1e-9 by a separate integration), the arc equation
  holds to 1e-8, and nu moves the way the natural step started it.
"""
import math
import os

import numpy as np
import pytest

import psgpu_b200 as P
from oracle import pyoracle as O
from oracle.newton2d import Newton2D, grid2d
from psgpu_b200.continuation import Continuation2D

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIX = os.path.join(ROOT, "tests", "golden", "upo2d_n32_re30.npz")
REF2D = os.path.join(ROOT, "oracle", "_ref", "libref_ns2d.so")


def _fix():
    d = dict(np.load(FIX))
    return {k: (v.item() if v.ndim == 0 else v) for k, v in d.items()}


def _dot(a, b, m):
    return float(np.sum((np.conj(a) * b).real[m]))


def _arc_case(form):
    """A corrector from orbit 0: r1 = the fixture orbit at Re = 30, r2 = the
    orbit at nu - 1 % (a natural step, solved here), first-order prediction with
    Ndelta_r = 2 |r2 - r1| (the reference's second run)."""
    d = _fix()
    n, dt = int(d["n"]), float(d["dt"])
    nu1 = 1.0 / float(d["re"])
    nu2 = nu1 * 0.99
    Z1, T1, S1 = d["o0_Z"], float(d["o0_T"]), float(d["o0_sx"])
    u = P.UPO2D(1, n, kmax=60, exact_jv=True)
    u.set_guess(0, Z1, T=T1, sx=S1, nu=nu2, dt=dt)
    u.solve(max_newton=30, tol=1e-12, gmres_tol=1e-3)
    r = u.get(0)
    u.close()
    assert r["status"] == "CONVERGED", r["status"]
    Z2, T2, S2 = r["Z"], r["T"], r["sx"]
    m = P.Grid2D(n).mask()
    dZ = Z2 - Z1
    dr2 = math.sqrt(_dot(dZ, dZ, m) + (S2 - S1) ** 2 + (nu2 - nu1) ** 2 + (T2 - T1) ** 2)
    arc = dict(dZrdr=dZ / dr2, Zr2=Z2, dTrdr=(T2 - T1) / dr2, dSrdr=(S2 - S1) / dr2,
               dv2rdr=(nu2 - nu1) / dr2, Tr2=T2, Sr2=S2, v2r2=nu2, ndelta=2.0 * dr2)
    N = arc["ndelta"]
    pred = dict(Z=Z2 + arc["dZrdr"] * N, T=T2 + arc["dTrdr"] * N, sx=S2 + arc["dSrdr"] * N,
                nu=nu2 + arc["dv2rdr"] * N)
    return d, n, dt, arc, pred


def _gpu(n, dt, arc, pred, exact, steps):
    u = P.UPO2D(1, n, kmax=60, exact_jv=exact)
    u.set_guess(0, pred["Z"], T=pred["T"], sx=pred["sx"], nu=pred["nu"], dt=dt)
    u.set_arc(0, arc["dZrdr"], arc["Zr2"], arc["dTrdr"], arc["dSrdr"], arc["dv2rdr"], arc["Tr2"],
              arc["Sr2"], arc["v2r2"], arc["ndelta"])
    u.solve(max_newton=steps, tol=1e-12, gmres_tol=1e-3)
    tr = u.trace(0)
    u.close()
    return tr


def _compare(steps, trace, nsteps, tol_T, tol_ner, tol_nu):
    assert len(trace) >= nsteps and len(steps) >= nsteps
    for s, t in zip(steps[:nsteps], trace[:nsteps]):
        assert t["gmres"] == s.gmres, (s.ine, t["gmres"], s.gmres)
        assert t["hook"] == s.hook, (s.ine, t["hook"], s.hook)
        assert t["delta"] == pytest.approx(s.delta, rel=1e-12), s.ine
        assert abs(t["T"] - s.T) < tol_T, (s.ine, t["T"], s.T)
        assert abs(t["sx"] - s.sx) < tol_T, (s.ine, t["sx"], s.sx)
        assert t["ner"] == pytest.approx(s.ner, rel=tol_ner), (s.ine, t["ner"], s.ner)
        assert t["nu"] == pytest.approx(s.nu, rel=tol_nu), (s.ine, t["nu"], s.nu)


def test_corrector_decisions_match_the_restatement_exact_jv():
    d, n, dt, arc, pred = _arc_case("exact")
    b = P.UPO2D(1, n, kmax=2, exact_jv=True)

    def phi(Z, T, dt_, nu):
        b.set_guess(0, Z, T=T, nu=nu, dt=dt_)
        return b.apply(0, 1)[0]

    def tangent(Z, q, T, dt_, nu):
        b.set_guess(0, Z, T=T, nu=nu, dt=dt_)
        return b.apply(0, 0, q)[1]

    def rhs(Z, nu):
        b.set_guess(0, Z, T=1.0, nu=nu, dt=0.005)
        return b.apply(0, 2)[0]

    ref = Newton2D(n, phi, rhs, tangent=tangent, gmresmax=60).solve(
        pred["Z"], pred["T"], pred["sx"], 0.0, 0, dt, 3, nu=pred["nu"], arc=arc)
    b.close()
    tr = _gpu(n, dt, arc, pred, True, 3)
    _compare(ref.steps, tr, 3, 1e-7, 1e-7, 1e-10)


def test_corrector_decisions_match_the_reference_step_fd_jv():
    if not os.path.exists(REF2D):
        pytest.skip("reference 2D step not built (oracle/build_ref.sh)")
    from psgpu_b200.abi import TimestepLibrary
    d, n, dt, arc, pred = _arc_case("fd")
    ref_lib = TimestepLibrary(REF2D, "ns2d")

    def phi(z, t, truedelt, nu):
        ns = int(t / truedelt)
        return ref_lib.ns2d(z, n, nu, t / ns, ns)[0]

    def rhs(z, nu):
        return O.ns2d_timederiv(z, n, nu)

    ref = Newton2D(n, phi, rhs, gmresmax=60).solve(pred["Z"], pred["T"], pred["sx"], 0.0, 0, dt,
                                                  2, nu=pred["nu"], arc=arc)
    tr = _gpu(n, dt, arc, pred, False, 2)
    _compare(ref.steps, tr, 2, 1e-5, 1e-3, 1e-7)


def test_batched_continuation_of_both_orbits():
    d = _fix()
    n, dt = int(d["n"]), float(d["dt"])
    nu0 = 1.0 / float(d["re"])
    branches = [{"Z": d[f"o{k}_Z"], "T": float(d[f"o{k}_T"]), "sx": float(d[f"o{k}_sx"]),
                 "nu": nu0} for k in range(int(d["nguess"]))]
    c = Continuation2D(n, branches, dt=dt, delta_v2=0.005 * nu0, kmax=60, netol=1e-10,
                       max_newton=30)
    kx, ky, LL = grid2d(n)
    chk = P.UPO2D(1, n, kmax=2, exact_jv=True)
    for step in range(3):
        hist_before = [list(b["hist"]) for b in c.B]
        pts = c.step()
        for k, (b, pt) in enumerate(zip(c.B, pts)):
            assert pt is not None, (step, k)
            assert pt["residual"] <= 1e-10
            # a periodic orbit at its own nu, by a separate integration
            chk.set_guess(0, pt["Z"], T=pt["T"], nu=pt["nu"], dt=dt)
            ZT = chk.apply(0, 1)[0]
            S = np.exp(-1j * kx * pt["sx"]) * ZT * LL
            ner = np.linalg.norm((S - pt["Z"])[LL]) / np.linalg.norm(ZT[LL])
            assert ner < 1e-9, (step, k, ner)
            if step == 0:
                assert pt["nu"] == pytest.approx(nu0 * 0.995, rel=1e-14)
            else:
                (Z1, T1, S1, v1), (Z2, T2, S2, v2) = hist_before[k][1], hist_before[k][2]
                dZ = Z2 - Z1
                dr = math.sqrt(_dot(dZ, dZ, LL) + (S2 - S1) ** 2 + (v2 - v1) ** 2 +
                               (T2 - T1) ** 2)
                res = (_dot(dZ / dr, pt["Z"] - Z2, LL) + (T2 - T1) / dr * (pt["T"] - T2)
                       + (S2 - S1) / dr * (pt["sx"] - S2) + (v2 - v1) / dr * (pt["nu"] - v2)
                       - b["delta_r2"])
                assert abs(res) < 1e-8, (step, k, res)
    for b in c.B:
        nus = [nu0] + [p["nu"] for p in b["points"]]
        assert all(x > y for x, y in zip(nus, nus[1:])), nus
    chk.close()
    c.close()
