"""Restart through the C-ABI in the reference's restart content
(src/vilma_io.f90:414-569): memory stress tau (NLAM, ne, nk) and time, the
diagnostic fields h_ice, rsl, z_bed, C_ocean, and with rotation the polar
motion and both degree-2 channels' memory. A run continued from a restart
must continue bit for bit."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth

pytestmark = pytest.mark.gpu


def new_model(w):
    m = vlib.Model(w.params(vlib.default_params))
    zb, hi = w.reference()
    m.set_reference(zb, hi)
    if w.visc3d:
        m.enable_visc3d(w.pert(m.p))
    return m


@pytest.mark.parametrize("visc3d", [False, True])
def test_restart_continues_bit_for_bit(visc3d):
    w = synth.Workload("rs", 16, 20, 100.0, 6, 3, "sawtooth", sle=True, visc3d=visc3d, seed=21, rotation=True)
    a = new_model(w)
    for step in range(1, 4):
        a.update(w.ice_at(step * 250), w.dt_yr)
    # restart record
    tau, t = a.state()
    rsl, zb, C, _ = a.fields()
    rot = a.rotation_state()
    ice_carried = w.ice_at(3 * 250)
    b = new_model(w)
    b.set_state(tau, t)
    b.set_fields(h_ice=ice_carried, rsl=rsl, z_bed=zb, C_ocean=C)
    b.set_rotation_state(*rot)
    for step in range(4, 7):
        ice = w.ice_at(step * 250)
        a.update(ice, w.dt_yr)
        b.update(ice, w.dt_yr)
        ra, rb = a.fields()[0], b.fields()[0]
        assert np.array_equal(ra, rb)
    assert a.rotation()[0] == b.rotation()[0]
    sa, _ = a.state()
    sb, _ = b.state()
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)


def test_trapezoidal_restart_continues_bit_for_bit():
    """The trapezoidal scheme also carries the controller's dt_try and the
    start-of-step load sigma_n across a restart (restore_sigma,
    src/vilma_io.f90:599-615)."""
    w = synth.Workload("rt", 16, 20, 200.0, 6, 3, "sawtooth", sle=True, visc3d=True, seed=23)

    def trap_model():
        p = w.params(vlib.default_params)
        p.scheme = 2
        m = vlib.Model(p)
        zb, hi = w.reference()
        m.set_reference(zb, hi)
        m.enable_visc3d(w.pert(m.p))
        return m

    a = trap_model()
    for step in range(1, 3):
        a.update(w.ice_at(step * 300), w.dt_yr)
    tau, t = a.state()
    rsl, zb, C, _ = a.fields()
    dt_try, sig_n, primed = a.step_state()
    assert primed and dt_try > 0
    b = trap_model()
    b.set_state(tau, t)
    b.set_fields(h_ice=w.ice_at(2 * 300), rsl=rsl, z_bed=zb, C_ocean=C)
    b.set_step_state(dt_try, sig_n, primed)
    for step in range(3, 5):
        ice = w.ice_at(step * 300)
        a.update(ice, w.dt_yr)
        b.update(ice, w.dt_yr)
        assert np.array_equal(a.fields()[0], b.fields()[0])
    for x, y in zip(a.state()[0], b.state()[0]):
        assert np.array_equal(x, y)
