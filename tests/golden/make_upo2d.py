"""Makes tests/golden/upo2d_n32_re30.npz: recurrence-derived guesses for
relative periodic orbits of 2D Kolmogorov flow and the orbits the reference's
Newton-GMRES-hookstep converges them to.

Test infrastructure.  Everything here runs on the host: the FP64 CPU oracle
(oracle/psg_oracle.c, a restatement of the reference's 2D step
2D_NavierStokes/src_RK4/kernels.h:112-435 pinned by tests/golden/ns2d_*.npz)
integrates, and oracle/newton2d.py (the restatement of
2D_NavierStokes/src_RK4/src_gmres/main.F90:688-1823, forward-difference Jv
with eps = 1e-7, DGESDD) converges.

Case: [0, 2 pi]^2, 32^2 (K = 10), Re = 30 (nu = 1/30), forcing sin(4y),
dt = 0.005.  A seeded start (modes 1 <= |k| <= 8, enstrophy 1) is integrated
for 100 time units, then 3000 snapshots 0.1 apart are searched for near
recurrences: for every pair 3 <= T <= 20 apart, the residual
min |S(z(t+T)) - z(t)| / |z(t)| over x-shifts (128 trial shifts) and the
discrete symmetries y -> y + m pi/2 and the shift-reflect x -> -x with
y -> y + pi/4 + m pi/2 (the reference's RsymFLAG); local minima of the
residual in (t, T) below 0.25 are candidates, best first.  The six best
candidates are converged to NETOL = 1e-12; the first two that land on
distinct orbits (periods more than 1e-4 apart) are kept.

    python tests/golden/make_upo2d.py        # ~5 minutes on 6 host cores
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "upo2d_n32_re30.npz")

N, RE, DT, SEED = 32, 30.0, 0.005, 5
SPINUP, NSNAP, EVERY = 100.0, 3000, 20


def trajectory():
    sys.path.insert(0, ROOT)
    from oracle import pyoracle as O
    from psgpu_b200.fields import kolmogorov_ic2d
    nu = 1.0 / RE
    Z = kolmogorov_ic2d(N, SEED)
    Z, _ = O.ns2d_timestep(Z, N, nu, DT, int(round(SPINUP / DT)))
    snaps = np.zeros((NSNAP,) + Z.shape, np.complex128)
    for i in range(NSNAP):
        snaps[i] = Z
        Z, _ = O.ns2d_timestep(Z, N, nu, DT, EVERY)
    return snaps


def recurrences(snaps, tmin=3.0, tmax=20.0, thresh=0.25, nshift=128):
    from oracle.newton2d import grid2d
    kx, ky, LL = grid2d(N)
    S = snaps * LL
    M = len(S)
    svals = np.linspace(0.0, 2 * np.pi, nshift, endpoint=False)
    E = np.exp(-1j * kx[0][:, None] * svals[None, :])
    norms = np.sum(np.abs(S) ** 2, axis=(1, 2))
    syms = [(0, m * np.pi / 2) for m in range(4)] + [(1, np.pi / 4 + m * np.pi / 2) for m in range(4)]
    h = EVERY * DT
    lags = range(int(round(tmin / h)), int(round(tmax / h)) + 1)
    L0, L1 = lags.start, lags.stop
    res = np.full((M, L1), np.inf)
    arg = np.zeros((M, L1, 3))
    for L in lags:
        A, B = S[:M - L], S[L:]
        for rs, sy in syms:
            Bs = np.conj(B[:, ::-1, :]) if rs else B
            Bs = Bs * np.exp(-1j * ky[:, 0] * sy)[None, :, None] * LL
            cross = np.real(np.sum(np.conj(A) * Bs, axis=1) @ E)
            ib = np.argmax(cross, axis=1)
            r = np.sqrt(np.maximum(norms[:M - L] + norms[L:] - 2 * cross[np.arange(M - L), ib], 0)
                        / norms[:M - L])
            upd = r < res[:M - L, L]
            res[:M - L, L][upd] = r[upd]
            arg[:M - L, L][upd] = np.stack([np.full(upd.sum(), rs), np.full(upd.sum(), sy),
                                            svals[ib[upd]]], 1)
    cand = []
    for i in range(1, M - 1):
        for L in range(L0 + 1, L1 - 1):
            r = res[i, L]
            if r < thresh and r <= res[i - 1:i + 2, L - 1:L + 2].min():
                cand.append((r, i, L * h, *arg[i, L]))
    cand.sort()
    out = []
    for c in cand:  # one candidate per recurrence event
        if all(abs(c[1] - o[1]) > 20 or abs(c[2] - o[2]) > 0.5 for o in out):
            out.append(c)
    return out


def converge(job):
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    from oracle import pyoracle as O
    from oracle.newton2d import Newton2D
    Z, T, sx, sy, rsym = job
    nu = 1.0 / RE

    def phi(z, t, dt):
        ns = int(t / dt)
        return O.ns2d_timestep(z, N, nu, t / ns, ns)[0]

    def rhs(z):
        return O.ns2d_timederiv(z, N, nu)

    r = Newton2D(N, phi, rhs, gmresmax=60, netol=1e-12).solve(Z, T, sx, sy, rsym, DT, 40)
    return r


def main():
    sys.path.insert(0, ROOT)
    snaps = trajectory()
    cands = recurrences(snaps)
    jobs = [(snaps[int(c[1])], float(c[2]), float(c[5]), float(c[4]), int(c[3])) for c in cands[:6]]
    with mp.get_context("spawn").Pool(6) as p:
        res = p.map(converge, jobs)
    keep = []
    for j, c, r in zip(jobs, cands, res):
        if r.status == "CONVERGED" and all(abs(r.T - o[2].T) > 1e-4 for o in keep):
            keep.append((j, c, r))
        if len(keep) == 2:
            break
    rec = {"n": N, "re": RE, "dt": DT, "nguess": len(keep)}
    for k, (j, c, r) in enumerate(keep):
        assert r.status == "CONVERGED", (k, r.status, r.ner)
        rec.update({
            f"g{k}_Z": j[0], f"g{k}_T": j[1], f"g{k}_sx": j[2], f"g{k}_sy": j[3],
            f"g{k}_rsym": j[4], f"g{k}_rec_residual": c[0], f"g{k}_rec_time": c[1] * EVERY * DT,
            f"o{k}_Z": r.Z, f"o{k}_T": r.T, f"o{k}_sx": r.sx, f"o{k}_ner": r.ner,
            f"o{k}_newton": r.newton, f"o{k}_gmres": r.gmres, f"o{k}_hook": r.hook,
            f"o{k}_trace_gmres": np.array([s.gmres for s in r.steps]),
            f"o{k}_trace_hook": np.array([s.hook for s in r.steps]),
            f"o{k}_trace_ner": np.array([s.ner for s in r.steps]),
            f"o{k}_trace_T": np.array([s.T for s in r.steps]),
            f"o{k}_trace_delta": np.array([s.delta for s in r.steps]),
        })
        print(f"guess {k}: recurrence residual {c[0]:.3f}, T {j[1]:.2f} -> {r.status} "
              f"ner {r.ner:.2e} T {r.T:.6f} sx {r.sx:.6f} in {r.newton} Newton steps")
    np.savez_compressed(OUT, **rec)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
