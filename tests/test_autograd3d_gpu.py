"""Gradient of terminal kinetic energy through the differentiable 3D trajectory
(torch.autograd.Function, checkpointed adjoint) against central finite
differences of the forward integration, FP64, on seeded directions.

Small case (32^3, 24 steps, checkpoints every 5 so that the last segment is
partial): directional derivatives agree to rel 1e-7 (central-difference
truncation with eps = 1e-4 of the state's norm); the FP32 engine's gradient
agrees with the FP64 one to rel 1e-4.
"""
import numpy as np
import pytest
import torch

import psgpu_b200 as P
from psgpu_b200.adjoint import Spectral3D, trajectory

pytestmark = pytest.mark.gpu

N, NU, DT, STEPS, EVERY = 32, 1 / 100, 5e-3, 24, 5


def _loss(u0, eng, sp):
    w0 = sp.curl(u0)
    wT = trajectory(w0, eng, DT, STEPS, EVERY)
    return sp.energy(sp.velocity(wT))


def _grad(precision, sp, u0):
    eng = P.NS3D(N, P.SCHEME_NS_RK4, precision=precision, nu=NU)
    u = u0.clone().requires_grad_(True)
    L = _loss(u, eng, sp)
    L.backward()
    return float(L.detach()), u.grad.detach().clone(), eng


def test_gradient_matches_central_differences():
    sp = Spectral3D(N)
    u0 = sp.random_velocity(3, energy=0.5)
    L, g, eng = _grad(64, sp, u0)
    eps = 1e-4
    for seed in range(4):
        v = sp.random_velocity(100 + seed, energy=1.0)
        with torch.no_grad():
            lp = float(_loss(u0 + eps * v, eng, sp))
            lm = float(_loss(u0 - eps * v, eng, sp))
        fd = (lp - lm) / (2 * eps)
        ad = float((g.real * v.real + g.imag * v.imag).sum())
        assert abs(ad - fd) <= 1e-7 * abs(fd) + 1e-12, (seed, ad, fd)


def test_fp32_gradient_matches_fp64():
    sp = Spectral3D(N)
    u0 = sp.random_velocity(5, energy=0.5)
    _, g64, _ = _grad(64, sp, u0)
    _, g32, _ = _grad(32, sp, u0)
    err = float((g32 - g64).abs().max() / g64.abs().max())
    assert err < 1e-4


def test_bous_gradient_matches_central_differences():
    """Boussinesq (Ri = 1, Sc = 1, gravity along z): gradient of the terminal
    kinetic plus potential energy with respect to the initial velocity and
    density"""
    sp = Spectral3D(N)
    u0 = sp.random_velocity(8, energy=0.5)
    rng = np.random.default_rng(9)
    r0 = torch.tensor((rng.standard_normal(sp.grid.shape) + 1j * rng.standard_normal(sp.grid.shape))
                      * sp.grid.mask() * 0.05, dtype=torch.complex128, device="cuda")
    eng = P.NS3D(N, P.SCHEME_BOUS_RK4, precision=64, nu=NU, ri=1.0, sc=1.0, theta=np.pi / 2)

    def loss(u, r):
        s0 = torch.cat([sp.curl(u), r[None]], 0)
        sT = trajectory(s0, eng, DT, STEPS, EVERY)
        return sp.energy(sp.velocity(sT[:3])) + (sT[3].real ** 2 + sT[3].imag ** 2).sum()

    u = u0.clone().requires_grad_(True)
    r = r0.clone().requires_grad_(True)
    L = loss(u, r)
    L.backward()
    eps = 1e-4
    for seed in range(3):
        vu = sp.random_velocity(200 + seed, energy=1.0)
        vr = torch.tensor(np.random.default_rng(300 + seed).standard_normal(sp.grid.shape) *
                          sp.grid.mask() * 0.1, dtype=torch.complex128, device="cuda")
        with torch.no_grad():
            fd = (float(loss(u0 + eps * vu, r0 + eps * vr)) - float(loss(u0 - eps * vu, r0 - eps * vr))) / (2 * eps)
        ad = float((u.grad.real * vu.real + u.grad.imag * vu.imag).sum() +
                   (r.grad.real * vr.real + r.grad.imag * vr.imag).sum())
        assert abs(ad - fd) <= 1e-7 * abs(fd) + 1e-12, (seed, ad, fd)
