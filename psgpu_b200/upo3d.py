"""Newton-GMRES-hookstep search for unstable periodic orbits of the 3D flows.

The reference's 3D Newton drivers (3D_Boussinesq/src/src_gmres/main.F90 and
3D_NavierStokes/src_gmres/main.F90) are Fortran programs around one
timestep_cuda_ call per Krylov vector.  This module is that driver for one
guess at a time, on the GPU engine of this package:

* the state is the truncated spectral box of every component (xii, eta, zet,
  and rho for the Boussinesq scheme), held on the device as a torch complex128
  tensor; inner products, Gram-Schmidt and the Newton updates run there in
  FP64; the small Hessenberg SVD runs on the host (numpy);
* Phi_T steps the engine as the reference's Newton-solver step does: full
  steps of dt while T - t > dt, then one step of the remaining length
  (3D_Boussinesq/src/src_gmres/cuda.cu:187-250);
* Jv is the exact discrete tangent of that integration (psg_ns3d_linear, one
  tangent step per time step; RK4/CN schemes) or the reference's forward
  difference [Phi_T(z + eps q) - Phi_T(z)]/eps with eps = 1e-7
  (main.F90:1041-1125);
* the unknowns are the state, the period T and the shifts along the listed
  directions (the Boussinesq driver: x and z, main.F90:1120-1140), with one
  orthogonality row per extra unknown (<dz/dt, q>, <dz/ds, q>); dz/dt is the
  engine's time derivative (timederiv_cuda_, src_gmres/cuda.cu:319-533);
* GMRES with modified Gram-Schmidt, the GMRES residual from the SVD, the
  hookstep mu-bisection to Delta/sqrt2 < |x| < sqrt2 Delta, the trial
  integration and the trust-region halve / double / revert logic, NaN
  handling and dt halving, and the NEWTON STALLED (more than five steps under
  0.1 % change), CONVERGED, PERIOD TOO SMALL and NEWTON FAILED statuses follow
  the Boussinesq driver (main.F90:816-1810); the residual is
  |F| / sqrt(|Phi_T(z)|^2 + |z|^2) (main.F90:775) and the tolerances are its
  NETOL = 1e-10, GMTOL = 1e-7, Delta_0 = 0.1, 50 hookstep trials
  (main.F90:136-141).
"""
from __future__ import annotations

import math

import numpy as np

from . import NS3D, SCHEME_BOUS_RK4, SCHEME_NS_RK4, PsgError

ROOT2 = math.sqrt(2.0)


class UPO3D:
    def __init__(self, engine: NS3D, dt: float, shifts=("x", "z"), jv: str = "exact",
                 kmax: int = 60, netol: float = 1e-10, gmtol: float = 1e-7, eps: float = 1e-7,
                 delta0: float = 0.1, ihookmax: int = 50, stall: int = 5):
        import torch
        if engine.precision != 64:
            raise PsgError("the 3D UPO search integrates in FP64")
        if jv == "exact" and engine.scheme not in (SCHEME_BOUS_RK4, SCHEME_NS_RK4):
            raise PsgError("the exact tangent is provided for the RK4/CN schemes; use jv='fd'")
        self.eng, self.dt, self.jv = engine, float(dt), jv
        self.kmax, self.netol, self.gmtol, self.eps = kmax, netol, gmtol, eps
        self.delta0, self.ihookmax, self.stall = delta0, ihookmax, stall
        g = engine.grid
        kx, ky, kz = g.wavenumbers()
        dev = torch.device("cuda")
        self.k = {a: torch.from_numpy(np.ascontiguousarray(np.broadcast_to(v, g.shape))).to(dev)
                  for a, v in (("x", kx), ("y", ky), ("z", kz))}
        self.mask = torch.from_numpy(g.mask()).to(dev)
        self.shift_dirs = tuple(shifts)
        self.nc = engine.ncomp
        self.integrations = 0
        self.torch = torch

    # ------------------------------------------------------------ building blocks
    def _m(self, a):
        return a * self.mask

    def _dot(self, a, b):
        return float((a.conj() * b).real.mul(self.mask).sum())

    def _shift(self, z, s):
        """exp(-i (kx sx + ky sy + kz sz)) z on every component (main.F90:763-771)"""
        ph = 0
        for a, v in s.items():
            ph = ph + self.k[a] * v
        return self._m(z * self.torch.exp(-1j * ph))

    def _steps(self, T, dt):
        t, n = 0.0, 0
        while T - t > dt:
            n += 1
            t += dt
        return n, (T - t if t != T else 0.0)

    def phi(self, z, T, dt):
        torch = self.torch
        self.integrations += 1
        z = z.contiguous()
        self.eng.upload_device([z[q].data_ptr() for q in range(self.nc)])
        n, last = self._steps(T, dt)
        if n:
            self.eng.step(dt, n)
        if last:
            self.eng.step(last, 1)
        out = torch.empty_like(z)
        self.eng.download_device([out[q].data_ptr() for q in range(self.nc)])
        self.eng.sync()
        return self._m(out)

    def tangent(self, z, q, T, dt):
        self.integrations += 1
        z = z.contiguous()
        self.eng.upload_device([z[c].data_ptr() for c in range(self.nc)])
        n, last = self._steps(T, dt)
        x = self._m(q).contiguous()
        for _ in range(n):
            x = self.eng.linear(self.eng.LIN_TANGENT_STEP, x, dt=dt)
        if last:
            x = self.eng.linear(self.eng.LIN_TANGENT_STEP, x, dt=last)
        self.eng.sync()
        return self._m(x)

    def rhs(self, z):
        torch = self.torch
        z = z.contiguous()
        self.eng.upload_device([z[q].data_ptr() for q in range(self.nc)])
        d = self.eng.timederiv()
        return self._m(torch.from_numpy(np.stack(d)).to(z.device))

    # ------------------------------------------------------------------- solve
    def solve(self, Z, T, shifts=None, max_newton=100):
        """Z: array (ncomp, IKTZ, IKTY, IKTX) complex128; shifts: dict of the shift
        unknowns (and fixed shifts).  Returns a dict with the orbit, the status,
        a per-step trace and, per Newton step, the GMRES residual after each
        Krylov iteration (gmres_residuals)."""
        torch = self.torch
        dev = self.mask.device
        s = {a: 0.0 for a in ("x", "y", "z")}
        s.update(shifts or {})
        truedelt0 = truedelt = self.dt
        if abs(T - round(T / truedelt) * truedelt) < 1e-10:
            T = round(T / truedelt) * truedelt
        znewt = self._m(torch.as_tensor(np.asarray(Z, np.complex128)).to(dev))
        tnewt = float(T)
        delta = self.delta0
        znn = self.phi(znewt, tnewt, truedelt)
        fn = self._m(self._shift(znn, s) - znewt)
        normfn = math.sqrt(self._dot(fn, fn))
        normz = math.sqrt(self._dot(znn, znn) + self._dot(znewt, znewt))
        ner = normfn / normz
        out = {"status": "NEWTON FAILED", "steps": [], "gmres": 0, "hook": 0,
               "gmres_residuals": []}
        if ner <= self.netol:
            out.update(status="CONVERGED", Z=znewt.cpu().numpy(), T=tnewt, shifts=dict(s), ner=ner,
                       newton=0, integrations=self.integrations)
            return out
        dirs = self.shift_dirs
        nx = 1 + len(dirs)  # extra unknowns: T and the shifts
        kmax = self.kmax
        nerold, nercount = 0.0, 0
        ine = 0
        for ine in range(1, max_newton + 1):
            normb = normfn
            q = [None] * (kmax + 1)
            qn = np.zeros((kmax + 1, nx))
            q[0] = self._m(-fn / normb)
            znshift = self._shift(znn, s)
            dzndt = self.rhs(znshift)
            dzdt = self.rhs(znewt)
            dznds = [self._m(-1j * self.k[a] * znshift) for a in dirs]
            dzds = [self._m(-1j * self.k[a] * znewt) for a in dirs]
            H = np.zeros((kmax + 1, kmax))

            def jv(vec, vn):
                if self.jv == "fd":
                    zn = self.phi(self._m(znewt + self.eps * vec), tnewt, truedelt)
                    d = (zn - znn) / self.eps
                else:
                    d = self.tangent(znewt, vec, tnewt, truedelt)
                r = self._shift(d, s) - vec + dzndt * vn[0]
                for j in range(len(dirs)):
                    r = r + dznds[j] * vn[1 + j]
                return self._m(r)

            # -------------------------------------------------------------- GMRES
            igm_done, gmr = 0, float("inf")
            P = S = VH = None
            gmr_hist = []
            out["gmres_residuals"].append(gmr_hist)
            for igm in range(1, kmax + 1):
                v = jv(q[igm - 1], qn[igm - 1])
                vn = np.array([self._dot(dzdt, q[igm - 1])] +
                              [self._dot(dzds[j], q[igm - 1]) for j in range(len(dirs))])
                for j in range(igm):
                    h = self._dot(q[j], v) + float(qn[j] @ vn)
                    H[j, igm - 1] = h
                    v = v - h * q[j]
                    vn = vn - h * qn[j]
                hn = math.sqrt(self._dot(v, v) + float(vn @ vn))
                H[igm, igm - 1] = hn
                q[igm] = self._m(v / hn)
                qn[igm] = vn / hn
                Hm = H[:igm + 1, :igm]
                U, S, VH = np.linalg.svd(Hm, full_matrices=True)
                P = normb * U[0, :]
                yh = VH.T @ (P[:igm] / S)
                r = Hm @ yh
                r[0] -= normb
                gmr = float(np.sqrt(np.sum(r * r)) / normb)
                gmr_hist.append(gmr)
                if gmr <= self.gmtol:
                    igm_done = igm
                    break
            if igm_done == 0:
                out["gmres"] += kmax + 1
                out["status"] = "GMRES FAILED"
                break
            igm = igm_done
            out["gmres"] += igm
            # ----------------------------------------------------------- hookstep
            ihook, halve, dbl = 0, False, False
            save = None
            nfpred = nfplus = float("nan")
            zplus = zn = fnplus = None
            tplus, splus = tnewt, dict(s)
            mumid = 0.0
            while True:
                ihook += 1
                if ihook > self.ihookmax:
                    break
                xh = P[:igm] / S[:igm]
                normx = float(np.sqrt(np.sum(xh * xh)))
                mumid = 0.0
                if normx > ROOT2 * delta:
                    mu1, mu2 = 0.0, float(np.max(S[:igm]))
                    xh = P[:igm] * S[:igm] / (mu2 + S[:igm] ** 2)
                    normx = float(np.sqrt(np.sum(xh * xh)))
                    while not (normx < delta):
                        mu1, mu2 = mu2, 2.0 * mu2
                        xh = P[:igm] * S[:igm] / (mu2 + S[:igm] ** 2)
                        normx = float(np.sqrt(np.sum(xh * xh)))
                    mumid = mu2
                    while not (normx < ROOT2 * delta and normx > delta / ROOT2):
                        mumid = 0.5 * (mu2 + mu1)
                        xh = P[:igm] * S[:igm] / (mumid + S[:igm] ** 2)
                        normx = float(np.sqrt(np.sum(xh * xh)))
                        if normx > delta:
                            mu1 = mumid
                        else:
                            mu2 = mumid
                yh = VH[:igm, :igm].T @ xh
                diffz = self._m(sum(q[j] * float(yh[j]) for j in range(igm)))
                dx = qn[:igm].T @ yh  # (dT, ds...)
                jfdiff = jv(diffz, dx)
                fnpred = self._m(fn + jfdiff)
                nfpred = math.sqrt(self._dot(fnpred, fnpred))
                nbpredc = math.sqrt(self._dot(fn, fn))
                zplus = self._m(znewt + diffz)
                tplus = tnewt + float(dx[0])
                splus = dict(s)
                for j, a in enumerate(dirs):
                    splus[a] = s[a] + float(dx[1 + j])
                zn = self.phi(zplus, tplus, truedelt)
                fnplus = self._m(self._shift(zn, splus) - zplus)
                nfplus = math.sqrt(self._dot(fnplus, fnplus))
                if nfplus != nfplus or nfpred != nfpred:
                    delta /= 2.0
                    halve = True
                    continue
                if nfplus >= nbpredc:
                    if dbl:
                        zplus, tplus, splus, zn, fnplus, nfplus = save
                        delta /= 2.0
                        break
                    delta /= 2.0
                    halve = True
                else:
                    if halve:
                        break
                    if dbl and nfplus > save[5]:
                        zplus, tplus, splus, zn, fnplus, nfplus = save
                        delta /= 2.0
                        break
                    if mumid == 0.0:
                        break
                    if abs(nfpred - nfplus) < 0.1 * abs(nfplus - normfn) or nfplus < nfpred:
                        delta *= 2.0
                        dbl = True
                        save = (zplus, tplus, dict(splus), zn, fnplus, nfplus)
                    else:
                        break
            out["hook"] += ihook
            step = {"newton": ine, "gmres": igm, "gmr": gmr, "hook": ihook, "delta": delta,
                    "mu": mumid}
            if nfpred != nfpred or nfplus != nfplus:
                if truedelt < 0.1 * truedelt0:
                    out["status"] = "T-STEP FAILED"
                    out["steps"].append(step)
                    break
                truedelt /= 2.0
                out["steps"].append(step)
                continue
            if ihook > self.ihookmax:
                out["status"] = "H-STEP FAILED"
                out["steps"].append(step)
                break
            # ------------------------------------------------------------ update
            znn, znewt, tnewt, s = zn, zplus, tplus, splus
            fn, normfn = fnplus, nfplus
            normz = math.sqrt(self._dot(znn, znn) + self._dot(znewt, znewt))
            ner = normfn / normz
            step.update(T=tnewt, shifts=dict(s), ner=ner)
            out["steps"].append(step)
            rel = abs((ner - nerold) / ner)
            stalled = False
            if rel < 0.001:
                nercount += 1
                stalled = nercount > self.stall
            else:
                nercount = 0
            nerold = ner
            if stalled:
                out["status"] = "NEWTON STALLED"
                break
            if ner <= self.netol:
                out["status"] = "CONVERGED"
                break
            if tnewt < 0.1:
                out["status"] = "PERIOD TOO SMALL"
                break
        out.update(Z=znewt.cpu().numpy(), T=tnewt, shifts=dict(s), ner=ner, newton=ine,
                   integrations=self.integrations)
        return out
