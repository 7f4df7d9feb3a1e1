"""Floquet multipliers of 2D orbits with the exact tangent.

The stability of a (relative) periodic orbit z = shift_s Phi_T(z) is given by
the eigenvalues of its monodromy operator M q = shift_s dPhi_T(z) q.  As the
reference's Newton solver does for its stability analysis
(2D_NavierStokes/src_RK4/src_gmres/main.F90:859-1037, ARPACK's Arnoldi on
finite-difference Jacobian-vector products), the leading multipliers come
from an Arnoldi iteration on M; here every product is one exact tangent
integration on the GPU (psg_upo2d_apply, mode 0) instead of a finite
difference, and the small Hessenberg eigenproblem is solved on the host.

The step is real-linear, not complex-linear (the kx = 0 modes are
Hermitian-completed), so the Krylov vectors are the real and imaginary parts
of the kept coefficients.
"""
from __future__ import annotations

import numpy as np

from . import UPO2D


def shift2d(grid, Z, sx: float, sy: float, rsym: int = 0):
    """the reference's shift (and shift-reflect) of a 2D state
    (2D_NavierStokes/src_RK4/src_gmres/main.F90:718-731):
    Z(kx, ky) exp(-i (kx sx + ky sy)), with rsym the reflection conj Z(kx, -ky) first"""
    kx, ky = grid.wavenumbers()
    W = Z
    if rsym:
        W = np.conj(Z[::-1, :])
    return W * np.exp(-1j * (kx * sx + ky * sy)) * grid.mask()


def floquet(upo: UPO2D, i: int, k: int = 30, sx: float | None = None, sy: float | None = None,
            rsym: int = 0, seed: int = 0):
    """Leading Floquet multipliers (sorted by modulus, largest first) of guess i's
    orbit at its current state and period, from k Arnoldi steps; the shift
    defaults to the guess's own.  Returns (multipliers, ritz residual
    estimates)."""
    g = upo.grid
    m = g.mask()
    nk = int(m.sum())
    info = upo.get(i)
    sx = info["sx"] if sx is None else sx
    sy = info["sy"] if sy is None else sy

    def to_real(Z):
        v = Z[m]
        return np.concatenate([v.real, v.imag])

    def to_cplx(x):
        Z = np.zeros(g.shape, np.complex128)
        Z[m] = x[:nk] + 1j * x[nk:]
        return Z

    def matvec(x):
        _, jq = upo.apply(i, 0, to_cplx(x))
        return to_real(shift2d(g, jq, sx, sy, rsym))

    rng = np.random.default_rng(seed)
    n = 2 * nk
    k = min(k, n)
    Q = np.zeros((n, k + 1))
    H = np.zeros((k + 1, k))
    q = rng.standard_normal(n)
    Q[:, 0] = q / np.linalg.norm(q)
    for j in range(k):
        w = matvec(Q[:, j])
        for r in range(2):  # modified Gram-Schmidt, twice
            for l in range(j + 1):
                h = Q[:, l] @ w
                H[l, j] += h
                w -= h * Q[:, l]
        H[j + 1, j] = np.linalg.norm(w)
        if H[j + 1, j] < 1e-14:
            k = j + 1
            break
        Q[:, j + 1] = w / H[j + 1, j]
    ev, vec = np.linalg.eig(H[:k, :k])
    order = np.argsort(-np.abs(ev))
    resid = np.abs(H[k, k - 1] * vec[k - 1, :]) if k < H.shape[0] else np.zeros(k)
    return ev[order], resid[order]
