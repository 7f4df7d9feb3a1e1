"""Generate golden input/output vectors from the reference's own CUDA step.

Runs on a machine with a GPU, after ``oracle/build_ref.sh`` has compiled the
reference's unmodified ``cuda.cu`` sources into ``oracle/_ref/libref_*.so``.
Each case feeds a seeded input through the reference's ``timestep_cuda_`` (FP64
cuFFT) with the argument lists its Fortran drivers build, and stores inputs,
parameters and outputs as ``.npz`` beside this script (or in ``--out``).

    python tests/golden/make_golden.py --out tests/golden

The fixtures pin the FP64 CPU oracle (tests/test_oracle_golden.py) and the
CUDA path (tests/test_parity_gpu.py) to the reference's behaviour.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from psgpu_b200.abi import TimestepLibrary  # noqa: E402
from psgpu_b200.fields import (Grid3D, kolmogorov_ic2d, random_vorticity3d,  # noqa: E402
                               taylor_green3d)


def _ref(flavour):
    return TimestepLibrary(os.path.join(ROOT, "oracle", "_ref", f"libref_{flavour}.so"), flavour)


def _rho3d(n, seed, amp=0.3):
    g = Grid3D(n)
    rng = np.random.default_rng(seed)
    kx, ky, kz = g.wavenumbers()
    wk = np.sqrt(kx * kx + ky * ky + kz * kz)
    sel = g.mask() & (wk <= 4.5)
    r = (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * sel
    return amp * r / math.sqrt(np.sum(np.abs(r) ** 2))


def cases():
    out = {}
    # ---- 2D RK4/CN (Kolmogorov forcing hard-coded at |ky| = 4) ----
    for n, seed, nstop in ((32, 11, 10), (128, 12, 40)):
        Z = kolmogorov_ic2d(n, seed)
        p = dict(n=n, nu=1 / 40, dt=0.005, nstop=nstop)
        Zo, t = _ref("ns2d").ns2d(Z, **p)
        out[f"ns2d_n{n}"] = dict(flavour="ns2d", Z_in=Z, Z_out=Zo, time=t, **p)
    # ---- 3D NS Heun/CN, forced at (0,kf,+-kf) ----
    for n, seed, kf, nstop, sol in ((16, 21, 2, 8, False), (32, 22, 4, 6, True)):
        xi, et, zt = random_vorticity3d(n, seed, kmin=0.5, kmax=n // 3 - 0.5, solenoidal=sol)
        p = dict(n=n, nu=1 / 20, dt=0.01, nstop=nstop, ampfor=-0.25 * kf * kf, kf=kf)
        # one step per call: the checked DNS build aborts on a filename buffer
        # overflow when NSTOP > 1 (see oracle/build_ref.sh)
        a, b, c, t, phys = _ref("ns3d").ns3d(xi, et, zt, steps_per_call=1, **p)
        out[f"ns3d_n{n}"] = dict(flavour="ns3d", xii_in=xi, eta_in=et, zet_in=zt,
                                 xii_out=a, eta_out=b, zet_out=c, phys_out=phys, time=t, **p)
    # ---- 3D Euler Heun ----
    n = 32
    xi, et, zt = taylor_green3d(n, 31, amp=1e-2)
    p = dict(n=n, dt=0.005, nstop=10)
    a, b, c, t, phys = _ref("euler3d").euler3d(xi, et, zt, **p)
    out["euler3d_n32"] = dict(flavour="euler3d", xii_in=xi, eta_in=et, zet_in=zt,
                              xii_out=a, eta_out=b, zet_out=c, phys_out=phys, time=t, **p)
    # ---- 3D Boussinesq RK4/CN ----
    bc = (
        ("bous3d_n16_ri1", 16, 41, dict(nu=1 / 50, dt=0.01, tend=0.1, ri=1.0, sc=1.0,
                                        theta=math.pi / 2, ampfor=-1.0, kf=2), True),
        ("bous3d_n16_tilt", 16, 42, dict(nu=1 / 30, dt=0.02, tend=0.13, ri=0.5, sc=0.7,
                                         theta=math.pi / 6, ampfor=-0.5, kf=1), True),
        ("bous3d_n32_ri0", 32, 43, dict(nu=1 / 1600, dt=1e-3, tend=0.0105, ri=0.0, sc=1.0,
                                        theta=0.0, ampfor=0.0, kf=4), False),
    )
    for name, n, seed, p, rnd in bc:
        if rnd:
            xi, et, zt = random_vorticity3d(n, seed, kmin=0.5, kmax=n // 3 - 0.5, solenoidal=True)
            rho = _rho3d(n, seed + 100)
        else:
            xi, et, zt = taylor_green3d(n, seed, amp=1e-3)
            rho = np.zeros_like(xi)
        a, b, c, r, t = _ref("bous3d").bous3d(xi, et, zt, rho, n=n, **p)
        out[name] = dict(flavour="bous3d", n=n, xii_in=xi, eta_in=et, zet_in=zt, rho_in=rho,
                         xii_out=a, eta_out=b, zet_out=c, rho_out=r, time=t, **p)
    # ---- Boussinesq time derivative ----
    n = 16
    xi, et, zt = random_vorticity3d(n, 51, kmin=0.5, kmax=4.5, solenoidal=False)
    rho = _rho3d(n, 151)
    p = dict(nu=1 / 50, ri=1.0, sc=1.0, theta=math.pi / 3, ampfor=-1.0, kf=2)
    a, b, c, r = _ref("bous3d").bous3d_timederiv(xi, et, zt, rho, n=n, **p)
    out["bous3d_deriv_n16"] = dict(flavour="bous3d_deriv", n=n, xii_in=xi, eta_in=et,
                                   zet_in=zt, rho_in=rho, xii_out=a, eta_out=b, zet_out=c,
                                   rho_out=r, **p)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for name, d in cases().items():
        path = os.path.join(args.out, name + ".npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in d.items()})
        print("wrote", path, flush=True)


if __name__ == "__main__":
    main()
