"""FP64 restatement of the reference's Newton-GMRES-hookstep search for
unstable periodic orbits of 2D Kolmogorov flow.

TEST INFRASTRUCTURE ONLY: the checker for the batched GPU solver
(psgpu_b200/csrc/psg_newton2d.cu) and the "plain form" the UPO benchmark is
timed against.  Only tests/ and bench.py import this module.

It follows 2D_NavierStokes/src_RK4/src_gmres/main.F90 line by line, for one
guess at a time, as the reference does:

* period snapping of a guess taken from a DNS (main.F90:688-692);
* Phi_T with NSTOP = INT(T/TRUEDELT), DELT = T/NSTOP (main.F90:697-699);
* the shift / shift-reflect of the final state (main.F90:718-731);
* F = shift(Phi_T(z)) - z, NER = |F|/|Phi_T(z)| (main.F90:756-762);
* per Newton step: TIMEDERIV at the shifted final state and at z, dZ/dS
  (main.F90:812-832); GMRES with the two extra rows <dz/dt, q>, <dz/dS, q>,
  modified Gram-Schmidt, DGESDD of the Hessenberg matrix and the residual
  |H y - |b| e1|/|b| (main.F90:853-1228); the forward-difference Jv with
  eps = 1e-7 (main.F90:1048-1116);
* the hookstep: mu-bisection to Delta/sqrt2 < |x| < sqrt2 Delta, the trial
  integration, NaN handling and the trust-region halve / double / revert
  logic (main.F90:1264-1623); dt halving after a blow-up (main.F90:1636-1665);
* the update, stall detection, convergence, PERIOD TOO SMALL and NEWTON
  FAILED statuses (main.F90:1667-1823);
* with `arc` (arclcFLAG2, the pseudo-arclength corrector of continuation in
  nu): the initial Narc (main.F90:633-640), |b| with Narc (806-812), the
  extra unknown nu and row vN3 in GMRES (1049-1061, 1121-1155), DIFFv2 and
  the trial's v2plus, Narcplus and |b{N+1}| against |b| (1350-1530,
  1538), v2plus in the save / revert (1550-1614), the update and the new
  Narc (1678, 1720-1727).  TIMEDERIV reads the one NU array the reference
  keeps, which the last hookstep trial set (v2plus), also after a revert.

The SVD is LAPACK's DGESDD through scipy.linalg.svd(lapack_driver='gesdd'),
the routine the reference calls (main.F90:1164).  The period map, the time
derivative and an optional exact tangent are callables supplied by the
caller (the reference's own CUDA step, this package's GPU building blocks or
the CPU oracle), so the same control flow can be driven by either.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np
import scipy.linalg as sla

ROOT2 = math.sqrt(2.0)


def grid2d(n: int, alpha: float = 1.0):
    """kx, ky (IKTY, IKTX) and the storage mask LL (2D_NavierStokes/src_RK4/init.F90:25-39)."""
    K = n // 3
    X, Y = K + 1, 2 * K + 1
    kx = (np.arange(X, dtype=np.float64) * alpha)[None, :].repeat(Y, 0)
    ky = (np.arange(Y, dtype=np.float64) - K)[:, None].repeat(X, 1)
    wk = kx * kx + ky * ky
    LL = (wk <= (K - 0.5) ** 2) & ~((kx == 0) & (ky <= 0))
    return kx, ky, LL


@dataclass
class Trial:
    delta: float      # trust radius the trial was taken with
    mu: float         # MUmid
    normx: float      # |x(mu)|
    nfpred: float     # NORMFNpred
    nfplus: float     # NORMFNplus
    action: str       # nan / halve / accept / double / revert


@dataclass
class NewtonStep:
    ine: int
    gmres: int        # IGM at exit (GMRES iterations of this step)
    gmr: float        # GMRES residual at exit
    hook: int         # IHOOK
    trials: list
    delta: float      # DELTA after the step
    T: float
    sx: float
    ner: float
    normfn: float
    nu: Optional[float] = None


@dataclass
class Result:
    status: str
    T: float
    sx: float
    sy: float
    ner: float
    Z: np.ndarray
    newton: int
    gmres: int
    hook: int
    steps: list = field(default_factory=list)
    integrations: int = 0
    nu: Optional[float] = None


class Newton2D:
    """phi(Z, T, dt) -> Phi_T(Z) taking NSTOP = INT(T/dt) steps of T/NSTOP;
    rhs(Z) -> dZ/dt (TIMEDERIV: N(Z) + forcing - nu k^2 Z on the kept modes);
    tangent(Z, q, T, dt) -> dPhi_T(Z) q, or None for the reference's forward
    difference.  With solve(..., arc=...) each is called with a further
    keyword nu= (the viscosity of that integration).  The exact-tangent form
    of the corrector takes dPhi_T/dnu by the central difference
    (Phi(nu (1 + 1e-5)) - Phi(nu (1 - 1e-5))) / (2e-5 nu)."""

    def __init__(self, n: int, phi: Callable, rhs: Callable, tangent: Optional[Callable] = None,
                 gmresmax: int = 60, netol: float = 1e-12, gmtol: float = 1e-3,
                 eps: float = 1e-7, delta0: float = 0.1, ihookmax: int = 50,
                 newtonmax: int = 100):
        self.n = n
        self.kx, self.ky, self.LL = grid2d(n)
        self.phi, self.rhs, self.tangent = phi, rhs, tangent
        self.gmresmax, self.netol, self.gmtol, self.eps = gmresmax, netol, gmtol, eps
        self.delta0, self.ihookmax, self.newtonmax = delta0, ihookmax, newtonmax
        self.integrations = 0

    # ---------------------------------------------------------------- helpers
    def _mask(self, a):
        return np.where(self.LL, a, 0.0 + 0.0j)

    def _dot(self, a, b):
        """SUM(REAL(CONJG(a)*b), LL)"""
        return float(np.sum((np.conj(a) * b).real[self.LL]))

    def _shift(self, Z, sx, sy, rsym):
        """main.F90:718-731: exp(-i kx sx) exp(-i ky sy) * (rsym ? conj(Z(kx,-ky)) : Z)"""
        src = np.conj(Z[::-1, :]) if rsym else Z
        return self._mask(np.exp(-1j * self.kx * sx) * np.exp(-1j * self.ky * sy) * src)

    def _step(self, Z, T, truedelt, nu=None):
        self.integrations += 1
        kw = {} if nu is None else {"nu": nu}
        return self._mask(np.asarray(self.phi(self._mask(Z), T, truedelt, **kw), np.complex128))

    def _rhs(self, Z, nu=None):
        kw = {} if nu is None else {"nu": nu}
        return self._mask(np.asarray(self.rhs(Z, **kw), np.complex128))

    # ------------------------------------------------------------------ solve
    def solve(self, Z, T, sx=0.0, sy=0.0, rsym=0, dt=0.005, max_newton=None, nu=None,
              arc=None) -> Result:
        """arc: None, or the corrector of a continuation step, a dict with dZrdr,
        Zr2, dTrdr, dSrdr, dv2rdr, Tr2, Sr2, v2r2, ndelta (then nu, the predicted
        viscosity, is an unknown too)."""
        LL = self.LL
        if arc is not None and nu is None:
            raise ValueError("an arc-length corrector needs the predicted nu")
        v2n = nu_rhs = nu
        if arc is not None:
            dzrdr = self._mask(np.asarray(arc["dZrdr"], np.complex128))
            zr2 = self._mask(np.asarray(arc["Zr2"], np.complex128))

            def narc_of(z, t, s, v):
                return (self._dot(dzrdr, z - zr2) + arc["dSrdr"] * (s - arc["Sr2"])
                        + arc["dv2rdr"] * (v - arc["v2r2"]) - arc["ndelta"]
                        + arc["dTrdr"] * (t - arc["Tr2"]))
        newtonmax = self.newtonmax if max_newton is None else max_newton
        truedelt0 = truedelt = dt
        delta = self.delta0
        # a period from a DNS is snapped to whole steps (main.F90:688-692)
        if abs(T - round(T / truedelt) * truedelt) < 1e-10:
            T = round(T / truedelt) * truedelt
        znewt = self._mask(np.asarray(Z, np.complex128))
        tnewt, snewtx, snewty = float(T), float(sx), float(sy)
        znn = self._step(znewt, tnewt, truedelt, v2n)
        znshift = self._shift(znn, snewtx, snewty, rsym)
        normz = math.sqrt(float(np.sum(np.abs(znn) ** 2)))
        fn = self._mask(znshift - znewt)
        normfn = math.sqrt(self._dot(fn, fn))
        ner = normfn / normz
        narc = narc_of(znewt, tnewt, snewtx, v2n) if arc is not None else 0.0
        res = Result("NEWTON FAILED", tnewt, snewtx, snewty, ner, znewt, 0, 0, 0, nu=v2n)
        if ner <= self.netol:
            res.status = "CONVERGED"
            res.integrations = self.integrations
            return res
        gmrescount = hookcount = 0
        nerold, nercount = 0.0, 0
        kmax = self.gmresmax
        ine = 0
        for ine in range(1, newtonmax + 1):
            normb = math.sqrt(normfn * normfn + narc * narc) if arc is not None else normfn
            q = [None] * (kmax + 1)
            qn1 = np.zeros(kmax + 1)
            qn2 = np.zeros(kmax + 1)
            qn3 = np.zeros(kmax + 1)
            q[0] = self._mask(-fn / normb)
            qn3[0] = -narc / normb
            dphidnu = None
            if arc is not None and self.tangent is not None:
                zp = self._step(znewt, tnewt, truedelt, v2n * (1.0 + 1e-5))
                zm = self._step(znewt, tnewt, truedelt, v2n * (1.0 - 1e-5))
                dphidnu = self._shift((zp - zm) * (0.5e5 / v2n), snewtx, snewty, rsym)
            dzndt = self._rhs(znshift, nu_rhs)
            dzdt = self._rhs(znewt, nu_rhs)
            dznds = self._mask(-1j * self.kx * znshift)
            dzds = self._mask(-1j * self.kx * znewt)
            H = np.zeros((kmax + 1, kmax))

            def jv(vec, vn_t, vn_s, vn_v=0.0):
                """J (vec, dT, dS, dnu) rows 1..N (main.F90:1047-1116 / 1360-1404)"""
                if self.tangent is None:
                    zo = self._mask(znewt + self.eps * vec)
                    nu_j = v2n + self.eps * vn_v if arc is not None else v2n
                    zn = self._step(zo, tnewt, truedelt, nu_j)
                    d = (zn - znn) / self.eps
                else:
                    self.integrations += 1
                    kw = {} if v2n is None else {"nu": v2n}
                    d = self._mask(np.asarray(self.tangent(znewt, self._mask(vec), tnewt,
                                                           truedelt, **kw), np.complex128))
                out = self._shift(d, snewtx, snewty, rsym) - vec + dznds * vn_s + dzndt * vn_t
                if dphidnu is not None:
                    out = out + dphidnu * vn_v
                return self._mask(out)

            # ------------------------------------------------------------ GMRES
            igm_done = 0
            gmr = float("inf")
            P = S = VH = None
            for igm in range(1, kmax + 1):
                v = jv(q[igm - 1], qn1[igm - 1], qn2[igm - 1], qn3[igm - 1])
                vn1 = self._dot(dzdt, q[igm - 1])
                vn2 = self._dot(dzds, q[igm - 1])
                vn3 = 0.0
                if arc is not None:
                    vn3 = (self._dot(dzrdr, q[igm - 1]) + arc["dTrdr"] * qn1[igm - 1]
                           + arc["dSrdr"] * qn2[igm - 1] + arc["dv2rdr"] * qn3[igm - 1])
                for j in range(igm):
                    h = self._dot(q[j], v) + qn1[j] * vn1 + qn2[j] * vn2 + qn3[j] * vn3
                    H[j, igm - 1] = h
                    v = self._mask(v - h * q[j])
                    vn1 -= h * qn1[j]
                    vn2 -= h * qn2[j]
                    vn3 -= h * qn3[j]
                hn = math.sqrt(self._dot(v, v) + vn1 * vn1 + vn2 * vn2 + vn3 * vn3)
                H[igm, igm - 1] = hn
                q[igm] = self._mask(v / hn)
                qn1[igm] = vn1 / hn
                qn2[igm] = vn2 / hn
                qn3[igm] = vn3 / hn
                Hm = H[:igm + 1, :igm]
                U, S, VH = sla.svd(Hm, full_matrices=True, lapack_driver="gesdd")
                P = normb * U[0, :]
                xh = P[:igm] / S
                yh = VH.T @ xh
                r = Hm @ yh
                r[0] -= normb
                gmr = float(np.sqrt(np.sum(r * r)) / normb)
                if gmr <= self.gmtol:
                    igm_done = igm
                    break
            if igm_done == 0:
                gmrescount += kmax + 1
                res.status = "GMRES FAILED"
                break
            igm = igm_done
            gmrescount += igm
            # --------------------------------------------------------- hookstep
            ihook = 0
            halve = dbl = False
            trials = []
            zplus2 = zn2 = fnplus2 = None
            tplus2 = splus2 = nfplus2 = v2plus2 = 0.0
            nfpred = nfplus = float("nan")
            zplus = zn = fnplus = None
            tplus = splus = v2plus = 0.0
            while True:
                ihook += 1
                if ihook > self.ihookmax:
                    break
                delta_now = delta
                xh = P[:igm] / S[:igm]
                normx = float(np.sqrt(np.sum(xh * xh)))
                mumid = 0.0
                if normx > ROOT2 * delta:
                    mu1, mu2 = 0.0, float(np.max(S[:igm]))
                    xh = P[:igm] * S[:igm] / (mu2 + S[:igm] * S[:igm])
                    normx = float(np.sqrt(np.sum(xh * xh)))
                    while not (normx < delta):
                        mu1, mu2 = mu2, 2.0 * mu2
                        xh = P[:igm] * S[:igm] / (mu2 + S[:igm] * S[:igm])
                        normx = float(np.sqrt(np.sum(xh * xh)))
                    mumid = mu2
                    while not (normx < ROOT2 * delta and normx > delta / ROOT2):
                        mumid = 0.5 * (mu2 + mu1)
                        xh = P[:igm] * S[:igm] / (mumid + S[:igm] * S[:igm])
                        normx = float(np.sqrt(np.sum(xh * xh)))
                        if normx > delta:
                            mu1 = mumid
                        else:
                            mu2 = mumid
                yh = VH[:igm, :igm].T @ xh
                diffz = self._mask(sum(q[j] * yh[j] for j in range(igm)))
                difft = float(np.dot(qn1[:igm], yh))
                diffs = float(np.dot(qn2[:igm], yh))
                diffv = float(np.dot(qn3[:igm], yh))
                jfdiff = jv(diffz, difft, diffs, diffv)
                fnpred = self._mask(fn + jfdiff)
                nfpred = math.sqrt(self._dot(fnpred, fnpred))
                nbpredc = math.sqrt(self._dot(fn, fn))  # |FN + const*J DIFF|, const = 0
                if arc is not None:
                    nbpredc = math.sqrt(nbpredc * nbpredc + narc * narc)
                zplus = self._mask(znewt + diffz)
                tplus = tnewt + difft
                splus = snewtx + diffs
                if arc is not None:
                    v2plus = v2n + diffv
                    nu_rhs = v2plus
                else:
                    v2plus = v2n
                zn = self._step(zplus, tplus, truedelt, v2plus)
                fnplus = self._mask(self._shift(zn, splus, snewty, rsym) - zplus)
                nfplus = math.sqrt(self._dot(fnplus, fnplus))
                nbplus = nfplus
                if arc is not None:
                    narcplus = narc_of(zplus, tplus, splus, v2plus)
                    nbplus = math.sqrt(nfplus * nfplus + narcplus * narcplus)
                if nfplus != nfplus or nfpred != nfpred:
                    delta /= 2.0
                    halve = True
                    trials.append(Trial(delta_now, mumid, normx, nfpred, nfplus, "nan"))
                    continue
                if nbplus >= nbpredc:
                    if dbl:
                        zplus, tplus, splus, zn, fnplus, nfplus = (zplus2, tplus2, splus2, zn2,
                                                                   fnplus2, nfplus2)
                        v2plus = v2plus2
                        delta /= 2.0
                        trials.append(Trial(delta_now, mumid, normx, nfpred, nfplus, "revert"))
                        break
                    delta /= 2.0
                    halve = True
                    trials.append(Trial(delta_now, mumid, normx, nfpred, nfplus, "halve"))
                else:
                    if halve:
                        trials.append(Trial(delta_now, mumid, normx, nfpred, nfplus, "accept"))
                        break
                    if dbl and nfplus > nfplus2:
                        zplus, tplus, splus, zn, fnplus, nfplus = (zplus2, tplus2, splus2, zn2,
                                                                   fnplus2, nfplus2)
                        v2plus = v2plus2
                        delta /= 2.0
                        trials.append(Trial(delta_now, mumid, normx, nfpred, nfplus, "revert"))
                        break
                    if mumid == 0.0:
                        trials.append(Trial(delta_now, mumid, normx, nfpred, nfplus, "accept"))
                        break
                    elif (abs(nfpred - nfplus) < 0.1 * abs(nfplus - normfn)
                          or nfplus < nfpred):
                        delta *= 2.0
                        dbl = True
                        zplus2, tplus2, splus2, zn2, fnplus2, nfplus2 = (zplus, tplus, splus, zn,
                                                                         fnplus, nfplus)
                        v2plus2 = v2plus
                        trials.append(Trial(delta_now, mumid, normx, nfpred, nfplus, "double"))
                    else:
                        trials.append(Trial(delta_now, mumid, normx, nfpred, nfplus, "accept"))
                        break
            hookcount += ihook
            # a blown-up integration: halve dt and retry (main.F90:1636-1665)
            if nfpred != nfpred or nfplus != nfplus:
                if truedelt < 0.1 * truedelt0:
                    res.status = "T-STEP FAILED"
                    break
                truedelt /= 2.0
                znshift = self._shift(znn, snewtx, snewty, rsym)
                res.steps.append(NewtonStep(ine, igm, gmr, ihook, trials, delta, tnewt, snewtx,
                                            ner, normfn, v2n))
                continue
            if ihook > self.ihookmax:
                res.status = "H-STEP FAILED"
                res.steps.append(NewtonStep(ine, igm, gmr, ihook, trials, delta, tnewt, snewtx,
                                            ner, normfn, v2n))
                break
            # ----------------------------------------------------------- update
            znn = zn
            znewt = zplus
            tnewt, snewtx = tplus, splus
            if arc is not None:
                v2n = v2plus
            znshift = self._shift(znn, snewtx, snewty, rsym)
            normz = math.sqrt(self._dot(znn, znn))
            fn = fnplus
            normfn = nfplus
            if arc is not None:
                narc = narc_of(znewt, tnewt, snewtx, v2n)
            ner = normfn / normz
            res.steps.append(NewtonStep(ine, igm, gmr, ihook, trials, delta, tnewt, snewtx, ner,
                                        normfn, v2n))
            rel = abs((ner - nerold) / ner)
            stalled = False
            if rel < 0.001:
                nercount += 1
                stalled = nercount > 3
            else:
                nercount = 0
            nerold = ner
            if stalled:
                res.status = "NEWTON STALLED"
                break
            if ner <= self.netol:
                res.status = "CONVERGED"
                break
            if tnewt < 0.1:
                res.status = "PERIOD TOO SMALL"
                break
        res.T, res.sx, res.sy, res.ner, res.Z, res.nu = tnewt, snewtx, snewty, ner, znewt, v2n
        res.newton = ine
        res.gmres, res.hook = gmrescount, hookcount
        res.integrations = self.integrations
        return res
