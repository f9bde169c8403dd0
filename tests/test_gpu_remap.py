"""Host-grid coupling on the GPU (vg_remap_*, vg_set_reference_ll,
vg_update_ll) against the oracle.

The remap legs match the oracle's restatement to 1e-12 (random fields, with
and without the mass rescale), and satisfy the reference's own checks
(tests/test_remap.f90:22-95). The coupled path of tests/test_couple_remap.f90
(a regular 96 x 48 host grid, a northern land cap over deep ocean, a 2 km ice
cap held for 12 intervals of 2 kyr) returns rsl and z_bed on the host grid
equal to the oracle's (host fields remapped in, the Gauss-grid update,
rsl remapped out) to 1e-10, with the reference's physical checks: ocean mass
conserved to 1e-10, the bed subsides more than 10 m under the ice, the ocean
draws down."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from oracle import orc
from oracle.remap import Remap as OrcRemap

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def regular(nlon, nlat):
    lon = -180.0 + (np.arange(nlon) + 0.5) * 360.0 / nlon
    lat = -90.0 + (np.arange(nlat) + 0.5) * 180.0 / nlat
    return lon, lat


def pair(lmax, nlon, nlat, mk_layers=None):
    out = []
    for mk in (vlib.default_params, orc.default_params):
        p = mk()
        p.lmax, p.nlat, p.nphi = lmax, 2 * lmax, 4 * lmax
        p.ne_layer[:4] = [3, 8, 8, 5]
        out.append(vlib.Model(p) if mk is vlib.default_params else orc.Oracle(p))
    return out


def test_remap_legs_match_oracle_and_reference_checks():
    L, NLON, NS = 32, 72, 36
    g, o = pair(L, NLON, NS)
    lon, lat = regular(NLON, NS)
    colat, w = o.grid()
    R, Ro = vlib.Remap(g, lon, lat), OrcRemap(lon, lat, colat, 4 * L)
    rng = np.random.default_rng(9)
    f = 1000.0 + 300.0 * rng.standard_normal((NS, NLON))
    for mass in (False, True):
        assert rel(R.to_gauss(f, mass), Ro.to_gauss(f, w, mass)) < 1e-12
    gf = rng.standard_normal((2 * L, 4 * L))
    assert rel(R.to_ll(gf), Ro.to_ll(gf)) < 1e-12
    # the reference's checks, on the GPU
    assert np.abs(R.to_gauss(np.full((NS, NLON), 7.0)) - 7.0).max() <= 1e-10
    latg = 90.0 - np.degrees(colat)
    gz = R.to_gauss(np.sin(np.radians(lat))[:, None] * np.ones(NLON))
    assert np.abs(gz - np.sin(np.radians(latg))[:, None]).max() <= 2e-2
    assert gz[0, 0] > 0.0 and gz[-1, 0] < 0.0
    fb = 1.0 + 0.5 * np.cos(np.radians(lat))[:, None] * np.cos(np.radians(lon))[None, :]
    gb = R.to_gauss(fb, True)
    isrc = (fb * Ro.area_s).sum() / Ro.area_s.sum()
    idst = o.surface_integral(np.ascontiguousarray(gb.reshape(-1))) / (4.0 * np.pi)
    assert abs(isrc - idst) <= 1e-10 * abs(isrc)
    gs = np.sin(np.radians(latg))[:, None] * np.ones(4 * L)
    assert np.abs(R.to_ll(gs) - np.sin(np.radians(lat))[:, None]).max() <= 5e-2


def test_host_grid_coupling_matches_oracle():
    L, NLON, NS, NSTEP = 16, 96, 48, 12
    g, o = pair(L, NLON, NS)
    lon, lat = regular(NLON, NS)
    colat, w = o.grid()
    z_eq = np.where(lat[:, None] > 40.0, 500.0, -4000.0) * np.ones(NLON)
    h_eq = np.zeros((NS, NLON))
    ice = np.where(lat[:, None] > 55.0, 2000.0, 0.0) * np.ones(NLON)
    R = vlib.Remap(g, lon, lat)
    R.set_reference(z_eq, h_eq)
    Ro = OrcRemap(lon, lat, colat, 4 * L)
    o.set_reference(np.ascontiguousarray(Ro.to_gauss(z_eq, w, False).reshape(-1)),
                    np.ascontiguousarray(Ro.to_gauss(h_eq, w, True).reshape(-1)))
    worst = 0.0
    for _ in range(NSTEP):
        rsl, zb = R.update(ice, 2000.0)
        o.update(np.ascontiguousarray(Ro.to_gauss(ice, w, True).reshape(-1)), 2000.0)
        worst = max(worst, g.info().worst_mass_resid)
    rsl_o = Ro.to_ll(o.fields()[0].reshape(2 * L, 4 * L))
    assert rel(rsl, rsl_o) < 1e-10
    assert rel(zb, z_eq - rsl_o) < 1e-10
    jice = int(np.argmin(np.abs(lat - 70.0)))
    joc = int(np.argmin(np.abs(lat + 50.0)))
    assert worst <= 1e-10
    assert z_eq[jice, 0] - zb[jice, 0] > 10.0  # subsidence under the ice
    assert rsl[joc, 0] < 0.0  # ocean drawdown
