"""Differentiable 3D trajectories: the RK4/CN step of `NS3D` behind a
`torch.autograd.Function`, with checkpointed recomputation.

The forward pass integrates the vorticity from w0 for `nsteps` steps and keeps
the state every `every` steps (FP64, reference layout, on the device).  The
backward pass walks the checkpoint segments in reverse: it recomputes the
segment's states from its checkpoint, then applies the exact adjoint of each
step (`psg_ns3d_linear`, PSG_LIN_ADJOINT_STEP) from the last state to the
first.  Memory: nsteps / every checkpoints plus `every` states.

Gradients follow torch's convention for complex tensors (dL/dRe + i dL/dIm),
which is the transpose in the real inner product of the stored coefficients
that the adjoint step implements.

Spectral helpers (curl, Biot-Savart, divergence-free random velocity) work on
the reference's truncated half-spectrum layout (IKTZ, IKTY, IKTX) and are
plain torch operations, so a loss can be written on velocities.
"""
from __future__ import annotations

import numpy as np
import torch

from . import NS3D, SCHEME_BOUS_RK4, SCHEME_NS_RK4
from .fields import Grid3D


def _ptrs(t):
    return [t[q].data_ptr() for q in range(t.shape[0])]


class _Trajectory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w0, engine, dt, nsteps, every):
        w = w0.detach().contiguous().to(torch.complex128)
        engine.upload_device(_ptrs(w))
        ckpts = []
        for n in range(nsteps):
            if n % every == 0:
                c = torch.empty_like(w)
                engine.download_device(_ptrs(c))
                ckpts.append(c)
            engine.step(dt, 1)
        out = torch.empty_like(w)
        engine.download_device(_ptrs(out))
        engine.sync()
        ctx.engine, ctx.dt, ctx.nsteps, ctx.every = engine, dt, nsteps, every
        ctx.ckpts = ckpts
        return out

    @staticmethod
    def backward(ctx, grad_out):
        eng, dt, nsteps, every = ctx.engine, ctx.dt, ctx.nsteps, ctx.every
        lam = grad_out.detach().contiguous().to(torch.complex128).clone()
        nseg = len(ctx.ckpts)
        for s in reversed(range(nseg)):
            n0 = s * every
            n1 = min(nsteps, n0 + every)
            states = [ctx.ckpts[s]]
            eng.upload_device(_ptrs(ctx.ckpts[s]))
            for _ in range(n0 + 1, n1):
                eng.step(dt, 1)
                z = torch.empty_like(lam)
                eng.download_device(_ptrs(z))
                states.append(z)
            for z in reversed(states):
                eng.upload_device(_ptrs(z))
                eng.linear(NS3D.LIN_ADJOINT_STEP, lam, dt, out=lam)
        eng.sync()
        ctx.ckpts = None
        return lam, None, None, None, None


def trajectory(w0: torch.Tensor, engine: NS3D, dt: float, nsteps: int, every: int = 20):
    """State after `nsteps` RK4/CN steps from w0 (CUDA complex128, shape
    (ncomp, IKTZ, IKTY, IKTX): the vorticity, and the density for the
    Boussinesq scheme), differentiable with respect to w0."""
    if engine.scheme not in (SCHEME_NS_RK4, SCHEME_BOUS_RK4):
        raise ValueError("the differentiable trajectory needs an RK4/CN scheme")
    if w0.shape[0] != engine.ncomp:
        raise ValueError(f"the engine's state has {engine.ncomp} components")
    return _Trajectory.apply(w0, engine, float(dt), int(nsteps), int(every))


class Spectral3D:
    """Wavenumbers and mask of a grid on a device, and the spectral operators of
    the step as torch functions on (3, IKTZ, IKTY, IKTX) complex tensors."""

    def __init__(self, n: int, device="cuda"):
        g = Grid3D(n)
        self.grid = g
        kx, ky, kz = g.wavenumbers()
        self.k = torch.tensor(np.stack([kx, ky, kz]), dtype=torch.float64, device=device)
        self.mask = torch.tensor(g.mask(), dtype=torch.float64, device=device)
        wk = kx * kx + ky * ky + kz * kz
        self.wkinv = torch.tensor(1.0 / np.maximum(wk, 1e-3), dtype=torch.float64, device=device)

    def cross_ik(self, x):
        """i k x x"""
        k = self.k
        c0 = k[1] * x[2] - k[2] * x[1]
        c1 = k[2] * x[0] - k[0] * x[2]
        c2 = k[0] * x[1] - k[1] * x[0]
        return 1j * torch.stack([c0, c1, c2]) * self.mask

    def curl(self, u):
        return self.cross_ik(u)

    def velocity(self, w):
        """Biot-Savart, u = i k x w / k^2"""
        return self.cross_ik(w) * self.wkinv

    def project(self, u):
        """divergence-free part, u - k (k.u) / k^2"""
        k = self.k
        div = (k * u).sum(0) * self.wkinv
        return (u - k * div) * self.mask

    def energy(self, u):
        """mean kinetic energy 1/2 <|u|^2> = sum over the stored modes |u_k|^2"""
        return (u.real ** 2 + u.imag ** 2).sum()

    def random_velocity(self, seed: int, energy: float = 0.5, k0: float = 4.0):
        """divergence-free random velocity with shell spectrum ~ k^4 exp(-2 (k/k0)^2)"""
        g = self.grid
        rng = np.random.default_rng(seed)
        z = rng.standard_normal((3,) + g.shape) + 1j * rng.standard_normal((3,) + g.shape)
        kx, ky, kz = g.wavenumbers()
        kk = np.sqrt(kx * kx + ky * ky + kz * kz)
        # per-mode amplitude: E(k) / (number of modes in the shell ~ k^2)
        amp = np.where(kk > 0, kk ** 2 * np.exp(-2.0 * (kk / k0) ** 2), 0.0)
        u = torch.tensor(z * np.sqrt(amp), dtype=torch.complex128, device=self.k.device)
        u = self.project(u)
        return u * np.sqrt(energy / float(self.energy(u)))
