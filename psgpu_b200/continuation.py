"""Arc-length continuation of 2D Kolmogorov periodic orbits in nu = 1/Re.

Restates the continuation driver around the reference's Newton solver
(2D_NavierStokes/src_RK4/src_gmres/main.F90:408-640 for the predictor and
the step-size control, 1780-1805 for the bookkeeping after convergence;
flags as parameters.F90:191-209 set them), with the corrector on the batched
GPU solver (psg_upo2d_set_arc): every branch is one guess of the batch, so
all branches step together.

Per branch and step:
* the first step is a natural one: nu <- nu - delta_v2 from the converged
  orbit (halving delta_v2 and retrying from the same orbit if Newton fails);
* later steps are pseudo-arclength ones: with the last two (three) converged
  points r1, r2 (r0) the branch tangent d(z, T, s, nu)/dr from the secant, the
  step Ndelta_r (twice the last secant on the second step, then at most the
  largest step taken, grown by 10 %, halved after a failure), the first-order
  (second step, or first_order) or second-order prediction, and the
  pseudo-arclength row <dZ/dr, z - Zr2> + ... = Ndelta_r as one more equation
  of the Newton solve, with nu one more unknown.
"""
from __future__ import annotations

import math

import numpy as np

from . import UPO2D


def _dot(a, b, mask):
    return float(np.sum((np.conj(a) * b).real[mask]))


class Continuation2D:
    def __init__(self, n, branches, dt, delta_v2, kmax=60, exact_jv=True, jv_precision=64,
                 first_order=False, full_second_order=False, drn_reset=False, netol=1e-10,
                 gmtol=1e-3, max_newton=30):
        """branches: converged orbits, dicts with Z, T, sx, and optionally sy, rsym,
        nu (viscosity).  delta_v2: the first, natural step in nu (the reference
        takes v2 - delta_v2)."""
        self.n, self.dt = n, dt
        self.first_order, self.full2 = first_order, full_second_order
        self.drn_reset = drn_reset
        self.netol, self.gmtol, self.max_newton = netol, gmtol, max_newton
        self.upo = UPO2D(len(branches), n, kmax=kmax, exact_jv=exact_jv,
                         jv_precision=jv_precision)
        self.mask = self.upo.grid.mask()
        self.B = []
        for b in branches:
            self.B.append({
                "start": (np.asarray(b["Z"], np.complex128), float(b["T"]), float(b["sx"])),
                "sy": float(b.get("sy", 0.0)), "rsym": int(b.get("rsym", 0)),
                "v2": float(b["nu"]), "delta_v2": float(delta_v2),
                "first": True, "second": False, "converged": True,
                "hist": [None, None, None],   # r0, r1, r2: (Z, T, S, v2)
                "delta_r1": 0.0, "delta_r2": 0.0, "ndelta": 0.0, "ndelta_max": 0.0,
                "points": [],
            })

    def close(self):
        self.upo.close()

    # ------------------------------------------------------------ predictor
    def _prepare(self, i, b):
        m = self.mask
        if b["first"]:
            # natural step in nu from the converged orbit (main.F90:412-428)
            if b["converged"]:
                b["v2"] -= b["delta_v2"]
            else:
                b["v2"] += b["delta_v2"]
                b["delta_v2"] /= 2.0
                b["v2"] -= b["delta_v2"]
            Z, T, S = b["start"]
            b["hist"][2] = (Z, T, S, b["v2"] + b["delta_v2"])
            b["converged"] = False
            self.upo.set_guess(i, Z, T=T, sx=S, sy=b["sy"], rsym=b["rsym"], nu=b["v2"], dt=self.dt)
            return
        (Z1, T1, S1, v1), (Z2, T2, S2, v2) = b["hist"][1], b["hist"][2]
        # secant, its length and the branch tangent (main.F90:454-465)
        dZ = Z2 - Z1
        dr2 = math.sqrt(_dot(dZ, dZ, m) + (S2 - S1) ** 2 + (v2 - v1) ** 2 + (T2 - T1) ** 2)
        b["delta_r2"] = dr2
        dZr, dTr, dSr, dvr = dZ / dr2, (T2 - T1) / dr2, (S2 - S1) / dr2, (v2 - v1) / dr2
        # step size (main.F90:467-485)
        if b["second"]:
            b["ndelta"] = 2.0 * dr2 if b["converged"] else b["ndelta"] / 2.0
            b["ndelta_max"] = b["ndelta"]
        else:
            if b["converged"]:
                b["ndelta"] = dr2 if dr2 < b["ndelta_max"] else b["ndelta_max"]
                if 1.1 * b["ndelta"] < b["ndelta_max"]:
                    b["ndelta"] *= 1.1
            else:
                b["ndelta"] /= 2.0
        b["converged"] = False
        N = b["ndelta"]
        if b["second"] or self.first_order:
            # first-order prediction (main.F90:488-505)
            Zp, Tp, Sp, vp = Z2 + dZr * N, T2 + dTr * N, S2 + dSr * N, v2 + dvr * N
        else:
            # second-order prediction from r0, r1, r2 (main.F90:508-560)
            Z0, T0, S0, v0 = b["hist"][0]
            drr = dr2 / (dr2 + b["delta_r1"])
            den1 = dr2 * (1.0 - drr)
            den2 = 0.5 * dr2 * dr2 * (1.0 - 1.0 / drr)

            def d1(x2, x1, x0):
                return ((1.0 - drr * drr) * x2 - x1 + drr * drr * x0) / den1

            def d2(x2, x1, x0):
                return ((drr - 1.0) * x2 + x1 - drr * x0) / den2

            Zp = Z2 + d1(Z2, Z1, Z0) * N + 0.5 * N * N * d2(Z2, Z1, Z0)
            Tp = T2 + d1(T2, T1, T0) * N + 0.5 * N * N * d2(T2, T1, T0)
            Sp = S2 + d1(S2, S1, S0) * N + 0.5 * N * N * d2(S2, S1, S0)
            vp = v2 + d1(v2, v1, v0) * N + 0.5 * N * N * d2(v2, v1, v0)
            if self.full2:
                dZr, dTr, dSr, dvr = (d1(Z2, Z1, Z0), d1(T2, T1, T0), d1(S2, S1, S0),
                                      d1(v2, v1, v0))
        if self.drn_reset:  # main.F90:567-572
            dz = Zp - Z2
            b["ndelta"] = math.sqrt(_dot(dz, dz, m) + (Sp - S2) ** 2 + (vp - v2) ** 2 +
                                    (Tp - T2) ** 2)
        b["v2"] = vp
        self.upo.set_guess(i, Zp, T=Tp, sx=Sp, sy=b["sy"], rsym=b["rsym"], nu=vp, dt=self.dt)
        self.upo.set_arc(i, dZr, Z2, dTr, dSr, dvr, T2, S2, v2, b["ndelta"])

    # --------------------------------------------------------------- a step
    def step(self):
        """one continuation step of every branch (one batched Newton solve);
        returns, per branch, the point reached (or None when Newton failed)"""
        for i, b in enumerate(self.B):
            self._prepare(i, b)
        self.upo.solve(max_newton=self.max_newton, tol=self.netol, gmres_tol=self.gmtol)
        out = []
        for i, b in enumerate(self.B):
            r = self.upo.get(i)
            if r["status"] != "CONVERGED":
                b["converged"] = False
                out.append(None)
                continue
            nu = self.upo.nu(i)
            # bookkeeping after convergence (main.F90:1780-1805)
            b["converged"] = True
            if b["second"]:
                b["second"] = False
            if b["first"]:
                b["first"] = False
                b["second"] = True
            b["hist"] = [b["hist"][1], b["hist"][2], (r["Z"], r["T"], r["sx"], nu)]
            b["delta_r1"] = b["delta_r2"]
            b["delta_r2"] = b["ndelta"]
            b["v2"] = nu
            pt = {"nu": nu, "re": 1.0 / nu, "T": r["T"], "sx": r["sx"], "residual": r["residual"],
                  "newton": r["newton"], "Z": r["Z"]}
            b["points"].append(pt)
            out.append(pt)
        return out

    def run(self, nsteps):
        for _ in range(nsteps):
            self.step()
        return [b["points"] for b in self.B]
