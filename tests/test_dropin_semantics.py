"""What an unchanged reference driver sees from the drop-in libraries.

* A call the library cannot serve (a box it does not support, no device, a
  failed device call) fills the state arrays with NaN.  The reference has no
  error channel; its Newton driver catches a failed integration by the NaN it
  leaves (2D_NavierStokes/src_RK4/src_gmres/main.F90:1527-1534, 1636-1665),
  whereas an untouched state would read as Phi_T(z) = z -- a false zero
  residual.  These calls fail on host-side checks (or for want of a device),
  so they run without a GPU.
* With no PSG_PRECISION in the environment the drop-ins compute in FP64, the
  reference's precision (the golden fixtures to 1e-10, on a GPU).
"""
import numpy as np
import pytest

import psgpu_b200 as P
from psgpu_b200.abi import TimestepLibrary
from psgpu_b200.fields import kolmogorov_ic2d, random_vorticity3d
from tests.golden_cases import cases, relerr


def _lib(flavour):
    try:
        P.lib()
        return TimestepLibrary(P.dropin_path(flavour), flavour)
    except (P.PsgError, OSError) as e:
        pytest.skip(f"drop-in {flavour} not loadable: {e}")


def _all_nan(*arrays):
    return all(np.isnan(a.view(np.float64)).all() for a in arrays)


def _state3(n, seed=3):
    return random_vorticity3d(n, seed)


def test_ns2d_unsupported_box_fills_nan():
    Z, _ = _lib("ns2d").ns2d(kolmogorov_ic2d(32, 1), 32, 1 / 40, 0.005, 3, alpha=0.5)
    assert _all_nan(Z)


def test_ns3d_unsupported_box_fills_nan():
    xi, et, zt = _state3(16)
    a, b, c, _, _ = _lib("ns3d").ns3d(xi, et, zt, 16, 1 / 40, 0.01, 1, alpha=0.5)
    assert _all_nan(a, b, c)


def test_euler3d_unsupported_box_fills_nan():
    xi, et, zt = _state3(16)
    a, b, c, _, _ = _lib("euler3d").euler3d(xi, et, zt, 16, 0.01, 1, alpha=0.5)
    assert _all_nan(a, b, c)


def test_bous3d_unsupported_box_fills_nan():
    L = _lib("bous3d")
    xi, et, zt = _state3(16)
    r = L.bous3d(xi, et, zt, np.zeros_like(xi), 16, 1 / 40, 0.01, 0.03, alpha=0.5)
    assert _all_nan(*r[:4])
    d = L.bous3d_timederiv(xi, et, zt, np.zeros_like(xi), 16, 1 / 40, alpha=0.5)
    assert _all_nan(*d)


def test_ns3d_newton_unsupported_grid_fills_nan(monkeypatch):
    # the Newton-solver build's grid is compiled in (PSG_NEWTON_N here); 48 is not a supported grid
    monkeypatch.setenv("PSG_NEWTON_N", "48")
    xi, et, zt = _state3(48)
    a, b, c, _ = _lib("ns3d_newton").ns3d_newton(xi, et, zt, 48, 1 / 40, 0.01, 1)
    assert _all_nan(a, b, c)


def _gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu(), reason="checks the no-device path")
def test_no_device_fills_nan():
    Z, _ = _lib("ns2d").ns2d(kolmogorov_ic2d(32, 1), 32, 1 / 40, 0.005, 3)
    assert _all_nan(Z)
    xi, et, zt = _state3(16)
    r = _lib("bous3d").bous3d(xi, et, zt, np.zeros_like(xi), 16, 1 / 40, 0.01, 0.03)
    assert _all_nan(*r[:4])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(cases()))
def test_default_precision_is_fp64(name, monkeypatch):
    """Every golden fixture through its drop-in with no PSG_PRECISION set: 1e-10."""
    monkeypatch.delenv("PSG_PRECISION", raising=False)
    d = cases()[name]
    fl, n, tol = d["flavour"], int(d["n"]), 1e-10
    if fl == "ns2d":
        Z, _ = _lib("ns2d").ns2d(d["Z_in"], n, d["nu"], d["dt"], int(d["nstop"]))
        assert relerr(Z, d["Z_out"]) < tol
    elif fl == "ns3d":
        r = _lib("ns3d").ns3d(d["xii_in"], d["eta_in"], d["zet_in"], n, d["nu"], d["dt"],
                              int(d["nstop"]), ampfor=d["ampfor"], kf=d["kf"])
        for x, k in zip(r[:3], ("xii_out", "eta_out", "zet_out")):
            assert relerr(x, d[k]) < tol, k
    elif fl == "euler3d":
        r = _lib("euler3d").euler3d(d["xii_in"], d["eta_in"], d["zet_in"], n, d["dt"],
                                    int(d["nstop"]))
        for x, k in zip(r[:3], ("xii_out", "eta_out", "zet_out")):
            assert relerr(x, d[k]) < tol, k
    elif fl == "bous3d":
        r = _lib("bous3d").bous3d(d["xii_in"], d["eta_in"], d["zet_in"], d["rho_in"], n, d["nu"],
                                  d["dt"], d["tend"], ri=d["ri"], sc=d["sc"], theta=d["theta"],
                                  ampfor=d["ampfor"], kf=d["kf"])
        for x, k in zip(r[:4], ("xii_out", "eta_out", "zet_out", "rho_out")):
            assert relerr(x, d[k]) < tol, k
    elif fl == "bous3d_deriv":
        r = _lib("bous3d").bous3d_timederiv(d["xii_in"], d["eta_in"], d["zet_in"], d["rho_in"], n,
                                            d["nu"], ri=d["ri"], sc=d["sc"], theta=d["theta"],
                                            ampfor=d["ampfor"], kf=d["kf"])
        for x, k in zip(r, ("xii_out", "eta_out", "zet_out", "rho_out")):
            assert relerr(x, d[k]) < tol, k
