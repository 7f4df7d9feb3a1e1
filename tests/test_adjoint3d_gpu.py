"""Tangent-linear and adjoint of the 3D RK4/CN step.

The linearised right-hand side and step are checked in FP64
  * tangent RHS against central differences of the engine's own time
    derivative (the nonlinear term is quadratic, so the central difference is
    exact up to round-off): rel 1e-9;
  * adjoint RHS and adjoint step by the dot-product identity
    <l, A d> = <A^T l, d> in the real inner product of the stored
    coefficients: rel 1e-11;
  * tangent step against central differences of the forward step
    (eps = 1e-5, truncation O(eps^2)): rel 1e-7;
and the FP32 engine's linearised step against the FP64 one: rel 2e-5.
"""
import numpy as np
import pytest
import torch

import psgpu_b200 as P
from psgpu_b200.fields import Grid3D, random_vorticity3d, taylor_green3d

pytestmark = pytest.mark.gpu

N, NU, DT = 32, 0.02, 2e-3


def _masked(seed, amp=1.0):
    g = Grid3D(N)
    rng = np.random.default_rng(seed)
    m = g.mask()
    v = [(rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * m for _ in range(3)]
    v = np.stack(v)
    return amp * v / np.sqrt(np.sum(np.abs(v) ** 2))


def _dot(a, b):
    a = a.cpu().numpy() if torch.is_tensor(a) else a
    b = b.cpu().numpy() if torch.is_tensor(b) else b
    return float(np.sum(a.real * b.real + a.imag * b.imag))


def _engine(z, precision=64):
    e = P.NS3D(N, P.SCHEME_NS_RK4, precision=precision, nu=NU)
    e.upload(*z)
    return e


def _base():
    xi, et, zt = random_vorticity3d(N, 21)
    return np.stack([xi, et, zt]) * 3.0


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _cuda(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_tangent_rhs_matches_central_difference():
    z = _base()
    d = _masked(1, amp=np.sqrt(np.sum(np.abs(z) ** 2)))
    e = _engine(z)
    jd = e.linear(P.NS3D.LIN_TANGENT_RHS, _cuda(d))
    torch.cuda.synchronize()
    g = Grid3D(N)
    kx, ky, kz = g.wavenumbers()
    wk = kx * kx + ky * ky + kz * kz
    derivs = []
    for s in (+1, -1):
        f = _engine(z + s * d)
        derivs.append(np.stack(f.timederiv()[:3]))
    fd = (derivs[0] - derivs[1]) / 2 + NU * wk * d * g.mask()
    assert _rel(jd.cpu().numpy(), fd) < 1e-9


@pytest.mark.parametrize("mode", [P.NS3D.LIN_ADJOINT_RHS, P.NS3D.LIN_ADJOINT_STEP])
def test_adjoint_dot_product(mode):
    z = _base()
    d, lam = _masked(2), _masked(3)
    tmode = P.NS3D.LIN_TANGENT_RHS if mode == P.NS3D.LIN_ADJOINT_RHS else P.NS3D.LIN_TANGENT_STEP
    e = _engine(z)
    jd = e.linear(tmode, _cuda(d), DT)
    e.upload(*z)
    jtl = e.linear(mode, _cuda(lam), DT)
    torch.cuda.synchronize()
    lhs, rhs = _dot(lam, jd), _dot(jtl, d)
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1e-300) + 1e-14 * np.linalg.norm(jd.cpu().numpy())


def test_tangent_step_matches_central_difference():
    z = _base()
    d = _masked(4, amp=np.sqrt(np.sum(np.abs(z) ** 2)))
    e = _engine(z)
    jd = e.linear(P.NS3D.LIN_TANGENT_STEP, _cuda(d), DT).cpu().numpy()
    eps = 1e-5
    outs = []
    for s in (+1, -1):
        f = _engine(z + s * eps * d)
        f.step(DT, 1)
        outs.append(np.stack(f.download()))
    fd = (outs[0] - outs[1]) / (2 * eps)
    assert _rel(jd, fd) < 1e-7
    # the engine's state advanced by one step, as a forward step would
    f = _engine(z)
    f.step(DT, 1)
    assert _rel(np.stack(e.download()), np.stack(f.download())) < 1e-13


@pytest.mark.parametrize("mode", [P.NS3D.LIN_TANGENT_STEP, P.NS3D.LIN_ADJOINT_STEP])
def test_fp32_linear_step_matches_fp64(mode):
    z = _base()
    d = _masked(5)
    r = {}
    for prec in (64, 32):
        e = _engine(z, prec)
        r[prec] = e.linear(mode, _cuda(d), DT).cpu().numpy()
    assert _rel(r[32], r[64]) < 2e-5


# ---------------------------------------------------------------- Boussinesq
# Ri = 1 (N = 1), Sc = 1 (Pr = 1), gravity along z (theta = 90 degrees)
RI, SC, THETA = 1.0, 1.0, np.pi / 2


def _bous_engine(z, precision=64):
    e = P.NS3D(N, P.SCHEME_BOUS_RK4, precision=precision, nu=NU, ri=RI, sc=SC, theta=THETA)
    e.upload(*z)
    return e


def _bous_base():
    w = _base()
    g = Grid3D(N)
    rho = random_vorticity3d(N, 33)[0] * g.mask()
    return np.concatenate([w, rho[None]], axis=0)


def _bous_masked(seed, amp=1.0):
    g = Grid3D(N)
    rng = np.random.default_rng(seed)
    v = np.stack([(rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * g.mask()
                  for _ in range(4)])
    return amp * v / np.sqrt(np.sum(np.abs(v) ** 2))


@pytest.mark.parametrize("mode", [P.NS3D.LIN_ADJOINT_RHS, P.NS3D.LIN_ADJOINT_STEP])
def test_bous_adjoint_dot_product(mode):
    z = _bous_base()
    d, lam = _bous_masked(12), _bous_masked(13)
    tmode = P.NS3D.LIN_TANGENT_RHS if mode == P.NS3D.LIN_ADJOINT_RHS else P.NS3D.LIN_TANGENT_STEP
    e = _bous_engine(z)
    jd = e.linear(tmode, _cuda(d), DT)
    e.upload(*z)
    jtl = e.linear(mode, _cuda(lam), DT)
    torch.cuda.synchronize()
    lhs, rhs = _dot(lam, jd), _dot(jtl, d)
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), 1e-300) + 1e-13 * np.linalg.norm(jd.cpu().numpy())


def test_bous_tangent_step_matches_central_difference():
    z = _bous_base()
    d = _bous_masked(14, amp=np.sqrt(np.sum(np.abs(z) ** 2)))
    e = _bous_engine(z)
    jd = e.linear(P.NS3D.LIN_TANGENT_STEP, _cuda(d), DT).cpu().numpy()
    eps = 1e-5
    outs = []
    for s in (+1, -1):
        f = _bous_engine(z + s * eps * d)
        f.step(DT, 1)
        outs.append(np.stack(f.download()))
    fd = (outs[0] - outs[1]) / (2 * eps)
    assert _rel(jd, fd) < 1e-7


@pytest.mark.parametrize("mode", [P.NS3D.LIN_TANGENT_STEP, P.NS3D.LIN_ADJOINT_STEP])
def test_bous_fp32_linear_step_matches_fp64(mode):
    z = _bous_base()
    d = _bous_masked(15)
    r = {}
    for prec in (64, 32):
        e = _bous_engine(z, prec)
        r[prec] = e.linear(mode, _cuda(d), DT).cpu().numpy()
    assert _rel(r[32], r[64]) < 5e-5


def test_bous_adjoint_step_dot_product_64():
    """the whole adjoint step at 64^3 (the scalar products' six x-pass outputs
    fill the intermediate buffer more than the forward step's do)"""
    n = 64
    g = Grid3D(n)
    rng = np.random.default_rng(41)
    m = g.mask()
    def rnd():
        return np.stack([(rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)) * m
                         for _ in range(4)])
    z, d, lam = rnd() * 0.05, rnd(), rnd()
    e = P.NS3D(n, P.SCHEME_BOUS_RK4, precision=64, nu=NU, ri=RI, sc=SC, theta=THETA)
    e.upload(*z)
    jd = e.linear(P.NS3D.LIN_TANGENT_STEP, _cuda(d), DT)
    e.upload(*z)
    jtl = e.linear(P.NS3D.LIN_ADJOINT_STEP, _cuda(lam), DT)
    torch.cuda.synchronize()
    lhs, rhs = _dot(lam, jd), _dot(jtl, d)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
