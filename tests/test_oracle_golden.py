"""The FP64 CPU oracle against golden vectors produced by the reference's own
CUDA timestep_cuda_ (FP64 cuFFT) on a B200.  This pins the oracle: every
flavour, the step-count and final-step rules, the physical-field output and the
Boussinesq time derivative agree to FP64 round-off."""
import pytest

from oracle import pyoracle as O
from tests.golden_cases import cases, relerr

CASES = cases()
TOL = 1e-12


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference(name):
    d = CASES[name]
    fl, n = d["flavour"], int(d["n"])
    if fl == "ns2d":
        Z, t = O.ns2d_timestep(d["Z_in"], n, d["nu"], d["dt"], int(d["nstop"]))
        assert relerr(Z, d["Z_out"]) < TOL
        assert t == pytest.approx(d["time"], rel=1e-14)
    elif fl in ("ns3d", "euler3d"):
        if fl == "ns3d":
            a, b, c, t, ph = O.ns3d_timestep(d["xii_in"], d["eta_in"], d["zet_in"], n, d["nu"],
                                             d["dt"], int(d["nstop"]), ampfor=d["ampfor"],
                                             kfy=float(d["kf"]), want_phys=True)
        else:
            a, b, c, t, ph = O.euler3d_timestep(d["xii_in"], d["eta_in"], d["zet_in"], n, d["dt"],
                                                int(d["nstop"]), want_phys=True)
        for x, k in ((a, "xii_out"), (b, "eta_out"), (c, "zet_out")):
            assert relerr(x, d[k]) < TOL, k
        assert relerr(ph, d["phys_out"]) < TOL
        assert t == pytest.approx(d["time"], rel=1e-12)
    elif fl == "bous3d":
        r = O.bous3d_timestep(d["xii_in"], d["eta_in"], d["zet_in"], d["rho_in"], n, d["nu"],
                              d["dt"], d["tend"], ri=d["ri"], sc=d["sc"], theta=d["theta"],
                              ampfor=d["ampfor"], kfy=float(d["kf"]))
        for x, k in zip(r[:4], ("xii_out", "eta_out", "zet_out", "rho_out")):
            assert relerr(x, d[k]) < TOL, k
        assert r[4] == pytest.approx(d["time"], rel=1e-14)
    elif fl == "bous3d_deriv":
        r = O.bous3d_timederiv(d["xii_in"], d["eta_in"], d["zet_in"], d["rho_in"], n, d["nu"],
                               ri=d["ri"], sc=d["sc"], theta=d["theta"], ampfor=d["ampfor"],
                               kfy=float(d["kf"]))
        for x, k in zip(r, ("xii_out", "eta_out", "zet_out", "rho_out")):
            assert relerr(x, d[k]) < TOL, k
    else:
        pytest.fail(f"unknown flavour {fl}")


def test_planted_mistake_is_caught():
    """A wrong viscosity in the oracle must break agreement with the fixture."""
    d = CASES["ns2d_n32"]
    Z, _ = O.ns2d_timestep(d["Z_in"], int(d["n"]), d["nu"] * 1.01, d["dt"], int(d["nstop"]))
    assert relerr(Z, d["Z_out"]) > 1e-8
