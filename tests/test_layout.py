"""Host-side layout logic: wavenumbers, masks, index maps and initial
conditions (no GPU).  The numpy builders of psgpu_b200.fields must agree with
the oracle's restatement of the Fortran drivers."""
import numpy as np
import pytest

from oracle import pyoracle as O
from psgpu_b200.fields import (Grid2D, Grid3D, kolmogorov_ic2d, random_vorticity3d,
                               taylor_green3d, to_physical3d)


@pytest.mark.parametrize("n", [16, 32, 64, 128])
def test_maps_3d(n):
    g = Grid3D(n)
    assert (g.ikf() == O.ikf3d(n)).all()
    assert (g.ikn() == O.ikn3d(n)).all()
    kx, ky, kz, LL = O.layout3d(n)
    assert (LL.reshape(g.shape).astype(bool) == g.mask()).all()
    # ikF and ikN are inverse on the box: padded(ikN[ik]) == ik
    ikf, ikn = g.ikf(), g.ikn()
    assert (ikf[ikn] == np.arange(g.nkt)).all()


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256])
def test_maps_2d(n):
    g = Grid2D(n)
    assert (g.ikf() == O.ikf2d(n)).all()
    assert (g.ikn() == O.ikn2d(n)).all()
    kx, ky, LL = O.layout2d(n)
    assert (LL.reshape(g.shape).astype(bool) == g.mask()).all()
    ikf, ikn = g.ikf(), g.ikn()[: g.nkt]
    assert (ikf[ikn] == np.arange(g.nkt)).all()


def test_sizes_of_the_configs():
    assert Grid2D(128).nkt == 3655
    assert Grid2D(64).nkt == 946
    assert Grid2D(256).nkt == 14706
    assert Grid3D(256).nkt == 2514726
    assert Grid3D(128).nkt == 310675


def test_taylor_green_physical():
    n = 32
    x = np.arange(n) * 2 * np.pi / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    xi, et, zt = taylor_green3d(n, 0, amp=0.0)
    ref = [-np.cos(X) * np.sin(Y) * np.sin(Z), -np.sin(X) * np.cos(Y) * np.sin(Z),
           2 * np.sin(X) * np.sin(Y) * np.cos(Z)]
    for F, r in zip((xi, et, zt), ref):
        assert np.abs(to_physical3d(F, n) - r).max() < 1e-13


def test_taylor_green_perturbation_divergence_free():
    n = 32
    g = Grid3D(n)
    xi, et, zt = taylor_green3d(n, 5, amp=1e-3)
    kx, ky, kz = g.wavenumbers()
    div = kx * xi + ky * et + kz * zt
    assert np.abs(div).max() < 1e-15
    assert not g.mask()[~g.mask()].any()
    assert np.abs(xi[~g.mask()]).max() == 0


def test_kolmogorov_ic_enstrophy():
    Z = kolmogorov_ic2d(128, 3)
    g = Grid2D(128)
    assert 2 * np.sum(np.abs(Z[g.mask()]) ** 2) == pytest.approx(1.0, rel=1e-12)
    kx, ky = g.wavenumbers()
    wk = np.sqrt(kx * kx + ky * ky)
    assert np.abs(Z[(wk > 8) | (wk < 1)]).max() == 0


def test_random_vorticity_solenoidal():
    n = 32
    g = Grid3D(n)
    a = random_vorticity3d(n, 1, solenoidal=True)
    kx, ky, kz = g.wavenumbers()
    assert np.abs(kx * a[0] + ky * a[1] + kz * a[2]).max() < 1e-14
