"""Floquet multipliers from the Arnoldi iteration on the exact tangent,
against the eigenvalues of the full Jacobian of the same map built by central
differences of the oracle's FP64 step (32^2, a time-T map of a laminar-ish
Kolmogorov state at Re = 5, no shift): the leading multipliers agree to 1e-6."""
import numpy as np
import pytest

import psgpu_b200 as P
from oracle import pyoracle as O
from psgpu_b200.fields import Grid2D, kolmogorov_ic2d
from psgpu_b200.floquet import floquet, shift2d

pytestmark = pytest.mark.gpu


def test_floquet_matches_full_jacobian():
    n, nu, dt, T = 16, 1 / 5.0, 0.005, 0.5
    g = Grid2D(n)
    m = g.mask()
    nk = int(m.sum())
    Z = kolmogorov_ic2d(n, 3) * 0.3
    u = P.UPO2D(1, n, kmax=4)
    u.set_guess(0, Z, T=T, nu=nu, dt=dt)
    mult, _ = floquet(u, 0, k=2 * nk)
    # full Jacobian of Phi_T by central differences of the oracle step
    ns = int(round(T / dt))
    eps = 1e-6
    J = np.zeros((2 * nk, 2 * nk))
    for j in range(2 * nk):
        e = np.zeros(2 * nk)
        e[j] = 1.0
        q = np.zeros(g.shape, np.complex128)
        q[m] = e[:nk] + 1j * e[nk:]
        zp, _ = O.ns2d_timestep(Z + eps * q, n, nu, dt, ns)
        zm, _ = O.ns2d_timestep(Z - eps * q, n, nu, dt, ns)
        d = (zp - zm) / (2 * eps)
        J[:, j] = np.concatenate([d[m].real, d[m].imag])
    ref = np.linalg.eigvals(J)
    ref = ref[np.argsort(-np.abs(ref))]
    for a, b in zip(mult[:6], ref[:6]):
        assert abs(a - b) < 1e-6 * max(1.0, abs(b)), (a, b)


def test_shift_and_shift_reflect():
    """the shift is an isometry; the shift-reflect is the reference's formula
    exp(-i kx sx) exp(-i ky sy) conj(Z(kx, -ky)) on the kept modes
    (src_gmres/main.F90:718-731), which reads the unkept kx = 0, ky < 0 slots"""
    n = 32
    g = Grid2D(n)
    Z = kolmogorov_ic2d(n, 9)
    W = shift2d(g, Z, 0.3, np.pi / 2, 0)
    assert np.sum(np.abs(W) ** 2) == pytest.approx(np.sum(np.abs(Z * g.mask()) ** 2), rel=1e-12)
    R = shift2d(g, Z, 0.3, np.pi / 2, 1)
    K = n // 3
    m = g.mask()
    for iky in range(2 * K + 1):
        for ikx in range(K + 1):
            want = 0.0
            if m[iky, ikx]:
                want = np.exp(-1j * ikx * 0.3) * np.exp(-1j * (iky - K) * np.pi / 2) * \
                    np.conj(Z[2 * K - iky, ikx])
            assert R[iky, ikx] == pytest.approx(want, abs=1e-14)
