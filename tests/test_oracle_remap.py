"""The oracle's host lon-lat <-> Gauss remap pinned to the reference's own
checks (tests/test_remap.f90:22-95) on the CPU: a constant is preserved to
1e-10, a zonal sin(lat) field comes through within 2e-2 with the northern
Gauss row first, the mass rescale makes the Gauss quadrature integral equal
the source area integral to 1e-10, and the bilinear leg returns sin(lat)
within 5e-2. Also: the host longitude window (-180..180 or 0..360) does not
change the result."""
import numpy as np
import pytest

from oracle import orc
from oracle.remap import Remap

LMAX, NLON, NLAT_S = 32, 72, 36


@pytest.fixture(scope="module")
def setup():
    p = orc.default_params()
    p.lmax, p.nlat, p.nphi = LMAX, 2 * LMAX, 4 * LMAX
    p.ne_layer[:4] = [2, 4, 4, 3]
    o = orc.Oracle(p)
    colat, w = o.grid()
    lon = -180.0 + (np.arange(NLON) + 0.5) * 360.0 / NLON
    lat = -90.0 + (np.arange(NLAT_S) + 0.5) * 180.0 / NLAT_S
    return o, colat, w, lon, lat, Remap(lon, lat, colat, p.nphi)


def test_remap_reference_properties(setup):
    o, colat, w, lon, lat, R = setup
    g = R.to_gauss(np.full((NLAT_S, NLON), 7.0), w, False)
    assert np.abs(g - 7.0).max() <= 1e-10
    f = np.sin(np.radians(lat))[:, None] * np.ones(NLON)
    g = R.to_gauss(f, w, False)
    latg = 90.0 - np.degrees(colat)
    assert np.abs(g - np.sin(np.radians(latg))[:, None]).max() <= 2e-2
    assert g[0, 0] > 0.0 and g[-1, 0] < 0.0  # north row first
    f = 1.0 + 0.5 * np.cos(np.radians(lat))[:, None] * np.cos(np.radians(lon))[None, :]
    g = R.to_gauss(f, w, True)
    isrc = (f * R.area_s).sum() / R.area_s.sum()
    idst = o.surface_integral(np.ascontiguousarray(g.reshape(-1))) / (4.0 * np.pi)
    assert abs(isrc - idst) <= 1e-10 * abs(isrc)
    gs = np.sin(np.radians(latg))[:, None] * np.ones(4 * LMAX)
    assert np.abs(R.to_ll(gs) - np.sin(np.radians(lat))[:, None]).max() <= 5e-2


def test_remap_longitude_window(setup):
    o, colat, w, lon, lat, R = setup
    rng = np.random.default_rng(3)
    f = rng.standard_normal((NLAT_S, NLON))
    shift = NLON // 2  # the same cells listed from 0 to 360 degrees
    lon2 = np.concatenate([lon[shift:], lon[:shift] + 360.0])
    f2 = np.concatenate([f[:, shift:], f[:, :shift]], axis=1)
    R2 = Remap(lon2, lat, colat, 4 * LMAX)
    assert np.abs(R.to_gauss(f, w, True) - R2.to_gauss(f2, w, True)).max() <= 1e-13
