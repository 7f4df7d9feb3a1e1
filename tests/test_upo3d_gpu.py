"""The 3D Newton-GMRES-hookstep driver (psgpu_b200/upo3d.py) on the GPU engine.

* Its building blocks: Phi_T equals the Boussinesq drop-in's integration of
  the same span (the reference's Newton-solver step: full steps of dt while
  T - t > dt, then the remainder; the drop-in is checked against the
  reference in test_parity_gpu.py); the exact tangent of that integration
  equals the central difference of Phi_T to 1e-7.
  The tangent carries the stage input the engine's step hands on to the next
  step (its final stage before the divergence removal), so the check holds
  over many steps for inputs with a divergence too (a random q).
* Newton from a perturbed laminar state of forced Boussinesq flow at 16^3
  (Re = 2, Ri = 1: the laminar shear is stable) reaches the reference's
  NETOL = 1e-10 with the exact tangent and with the forward difference, and
  lands on the laminar state.  The shear is invariant under the x and z
  shifts and steady in time, so those unknowns are nearly degenerate and
  GMRES stalls on its way to the driver's GMTOL = 1e-7 (80 iterations were
  not always enough); the test asks for 1e-4, which Newton turns into the
  same final residual in a few more steps.
"""
import numpy as np
import pytest
import torch

import psgpu_b200 as P
from psgpu_b200.abi import TimestepLibrary
from psgpu_b200.fields import Grid3D, random_vorticity3d
from psgpu_b200.upo3d import UPO3D
from tests.golden_cases import relerr

pytestmark = pytest.mark.gpu

N, NU, DT, KF, AMP = 16, 0.5, 0.01, 1.0, -0.5


def _engine():
    return P.NS3D(N, P.SCHEME_BOUS_RK4, precision=64, nu=NU, ampfor=AMP, kf=KF, ri=1.0, sc=1.0,
                  theta=np.pi / 2)


def _laminar():
    g = Grid3D(N)
    z = np.zeros((4,) + g.shape, np.complex128)
    # zeta(0, kf, 0) of the steady shear: -nu kf^2 zeta + ampfor = 0
    z[2, g.kt, g.kt + int(KF), 0] = AMP / (NU * KF * KF)
    return z


def _perturbed(seed=3, amp=0.05):
    z = _laminar()
    xi, et, zt = random_vorticity3d(N, seed, kmin=1.0, kmax=4.0, solenoidal=True)
    rho = random_vorticity3d(N, seed + 1, kmin=1.0, kmax=4.0)[0]
    return z + amp * np.stack([xi, et, zt, 0.1 * rho])


def test_phi_and_tangent():
    eng = _engine()
    u = UPO3D(eng, DT)
    z = _perturbed()
    T = 0.255
    zt = torch.as_tensor(z).cuda()
    phi = u.phi(zt, T, DT).cpu().numpy()
    lib = TimestepLibrary(P.dropin_path("bous3d"), "bous3d")
    ref = lib.bous3d(*z, N, NU, DT, T, ri=1.0, sc=1.0, theta=np.pi / 2, ampfor=AMP, kf=KF)
    for a, b in zip(phi, ref[:4]):
        assert relerr(a, b) < 1e-12
    rng = np.random.default_rng(5)
    q = (rng.standard_normal(z.shape) + 1j * rng.standard_normal(z.shape)) * Grid3D(N).mask()
    q /= np.linalg.norm(q)
    jq = u.tangent(zt, torch.as_tensor(q).cuda(), T, DT).cpu().numpy()
    e = 1e-5
    zp = u.phi(torch.as_tensor(z + e * q).cuda(), T, DT).cpu().numpy()
    zm = u.phi(torch.as_tensor(z - e * q).cuda(), T, DT).cpu().numpy()
    fd = (zp - zm) / (2 * e)
    assert np.linalg.norm(jq - fd) / np.linalg.norm(fd) < 1e-7
    eng.close()


@pytest.mark.parametrize("jv", ["exact", "fd"])
def test_newton_converges_to_laminar_state(jv):
    eng = _engine()
    # the x and z shifts barely move the near-laminar state (its shear mode is
    # invariant under them) and it is nearly steady: GMRES tolerance 1e-4
    u = UPO3D(eng, DT, jv=jv, kmax=80, gmtol=1e-4)
    r = u.solve(_perturbed(), T=1.0, shifts={"x": 0.0, "z": 0.0}, max_newton=25)
    assert r["status"] == "CONVERGED", (r["status"], r["ner"], r["steps"])
    assert r["ner"] <= 1e-10
    lam = _laminar()
    # the laminar state up to the x/z translations the orbit may pick (they do
    # not move the kx = kz = 0 shear mode)
    assert relerr(r["Z"][2, :, :, 0], lam[2, :, :, 0]) < 1e-6
    eng.close()
