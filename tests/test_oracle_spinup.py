"""The oracle's spin-up relaxation (solid_earth_spinup's relax_hold) against the
checks of the reference's tests/test_spinup.f90 on the same setup (lmax 16,
32 x 64 grid, bed 500 m north of 50 deg colatitude and -4000 m elsewhere, a
2 km polar cap north of 30 deg, a 500 kyr cap): the held load relaxes the bed
far beyond a single cold 2 kyr step and leaves it near stationary."""
import numpy as np

from oracle import orc

RATE_TOL = 1e-3  # equil_rate_tol [m/yr] (src/vilma_params.f90)


def setup():
    p = orc.default_params()
    p.lmax, p.nlat, p.nphi = 16, 32, 64
    o = orc.Oracle(p)
    colat, _ = o.grid()
    cd = np.rad2deg(colat)[:, None] * np.ones((1, p.nphi))
    z_eq = np.where(cd < 50.0, 500.0, -4000.0).reshape(-1)
    ice = np.where(cd < 30.0, 2000.0, 0.0).reshape(-1)
    o.set_reference(z_eq, np.zeros_like(z_eq))
    jice = int(np.argmin(np.abs(np.rad2deg(colat) - 15.0)))
    return o, z_eq, ice, jice * p.nphi


def test_spinup_relaxes_to_equilibrium():
    o, z_eq, ice, at = setup()
    o.update(ice, 2.0e3)
    cold_step = z_eq[at] - o.fields()[1][at]
    o, z_eq, ice, at = setup()
    t_done, passes, converged = o.spinup(ice, 5.0e5, RATE_TOL)
    assert converged and 0 < passes <= 60 and 0 < t_done <= 5.0e5
    zb = o.fields()[1]
    spin_sub = z_eq[at] - zb[at]
    o.update(ice, 2.0e3)
    follow = abs(o.fields()[1][at] - zb[at])
    assert spin_sub >= 50.0 and spin_sub >= 1.5 * cold_step, (spin_sub, cold_step)
    assert follow <= 0.1 * cold_step, (follow, cold_step)


def test_spinup_zero_cap_does_nothing():
    o, z_eq, ice, at = setup()
    assert o.spinup(ice, 0.0, RATE_TOL) == (0.0, 0, False)
    assert np.array_equal(o.fields()[1], z_eq)


def test_pre_spinup_1d_phase():
    """tests/test_spinup.f90 check (2): the 1-D pre-equilibration alone
    (pre_spinup_1d, equil_time_max = 0) drives appreciable subsidence."""
    o, z_eq, ice, at = setup()
    t_done, passes, converged, passes_1d = o.spinup(ice, 0.0, RATE_TOL, pre_1d=True, with_1d=True)
    assert (t_done, passes, converged) == (0.0, 0, False) and 0 < passes_1d <= 60
    assert z_eq[at] - o.fields()[1][at] >= 50.0


def test_pre_spinup_1d_restores_the_3d_field():
    """With lateral viscosity, the 1-D phase runs on the lateral mean and the
    genuinely 3-D elements are back afterwards."""
    from fastearth3d_b200 import synth

    w = synth.Workload("s", 12, 16, 100.0, 2, 2, "sawtooth", sle=True, visc3d=True, seed=8)
    o = orc.Oracle(w.params(orc.default_params))
    zb, hi = w.reference()
    o.set_reference(zb, hi)
    o.enable_visc3d(w.pert(o.p))
    ne3d = o.info().ne3d
    assert ne3d > 0
    out = o.spinup(w.ice_at(400), 2000.0, RATE_TOL, pre_1d=True, with_1d=True)
    assert out[3] > 0 and out[1] > 0
    assert o.info().ne3d == ne3d
