"""vg_advance (stepper_advance, src/vilma_timestep.f90:79-105, for hosts that
run their own interval driver) against the oracle's stepper_advance: three
intervals with a host-given rotational-feedback term s_rot held across each
(rsl, C and the converged load to 1e-10, identical ocean function), and with
no s_rot the same results as vg_update bit for bit."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from oracle import orc

pytestmark = pytest.mark.gpu


def test_advance_with_host_s_rot_matches_oracle():
    w = synth.Workload("a", 16, 20, 100.0, 3, 3, "sawtooth", sle=True, visc3d=True, seed=12)
    g, o = vlib.Model(w.params(vlib.default_params)), orc.Oracle(w.params(orc.default_params))
    zb, hi = w.reference()
    colat, _ = o.grid()
    lon = 2 * np.pi * np.arange(w.nphi) / w.nphi
    s_rot = (0.8 * np.sin(2 * colat)[:, None] * np.cos(lon - 0.3)[None, :]).reshape(-1)  # a degree-2 order-1 term
    for m in (g, o):
        m.set_reference(zb, hi)
        m.enable_visc3d(w.pert(m.p))
    ice_prev = hi
    for step in range(1, 4):
        ice = w.ice_at(step * 300)
        t0, t1 = (step - 1) * w.dt_yr, step * w.dt_yr
        rg, cg, sg = g.advance_interval(ice_prev, ice, t0, t1, s_rot)
        ro, co, so = o.advance_interval(ice_prev, ice, t0, t1, s_rot)
        assert np.array_equal(cg, co)
        assert np.abs(rg - ro).max() <= 1e-10 * np.abs(ro).max()
        assert np.abs(sg - so).max() <= 1e-10 * np.abs(so).max()
        ice_prev = ice
    assert g.info().time_yr == pytest.approx(3 * w.dt_yr)


def test_advance_without_s_rot_is_update():
    w = synth.Workload("a", 16, 20, 100.0, 3, 3, "sawtooth", sle=True, visc3d=False, seed=13)
    a, b = vlib.Model(w.params(vlib.default_params)), vlib.Model(w.params(vlib.default_params))
    zb, hi = w.reference()
    for m in (a, b):
        m.set_reference(zb, hi)
    ice_prev = hi
    for step in range(1, 3):
        ice = w.ice_at(step * 300)
        a.update(ice, w.dt_yr)
        rb, _, _ = b.advance_interval(ice_prev, ice, (step - 1) * w.dt_yr, step * w.dt_yr)
        assert np.array_equal(a.fields()[0], rb)
        ice_prev = ice
