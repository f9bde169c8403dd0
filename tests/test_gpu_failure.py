"""Failure paths of the time step, driven in forms that fault and hang no GPU:

* the forward-Euler guard's reject branch (src/vilma_timestep.f90:204-224):
  a Maxwell-CFL ceiling above the stability limit with a tight growth bound
  makes sub-steps grow the memory too fast; the device rejects, restores and
  halves exactly where the oracle does;
* the guard's collapse: a memory state with NaN (set through the restart
  entry point on the host) is never accepted, the sub-step halves until it
  collapses, and the call returns a nonzero status with the reference's
  message instead of stopping;
* a singular radial operator (a solid earth with no density and no rigidity):
  the band LU meets an exact zero pivot (src/vilma_band.f90:81) and vg_create
  returns a status, as the oracle does;
* the bounded device waits: with the wait limit set to zero the fused
  sea-level loop's grid barriers run out, the kernel returns early with its
  status bit, the update reports the error, and the device stays usable."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from oracle import orc
from parity_util import check_models

pytestmark = pytest.mark.gpu


def pair(w, **kw):
    ps = []
    for mk in (vlib.default_params, orc.default_params):
        p = w.params(mk)
        for k, v in kw.items():
            setattr(p, k, v)
        ps.append(p)
    return vlib.Model(ps[0]), orc.Oracle(ps[1])


def test_guard_rejects_and_recovers_like_the_oracle():
    # 2-kyr intervals under cfl 20: one sub-step with M ~ 11 in the upper
    # mantle, |1 - M| > guard_growth 2 -> reject, halve, recover (10 rejects)
    w = synth.Workload("t", 16, 20, 2000.0, 4, 2, "sawtooth", sle=True, visc3d=False, seed=21)
    g, o = pair(w, cfl=20.0, guard_growth=2.0)
    for m in (g, o):
        m.set_reference(*w.reference())
    for step in (8, 9, 10, 11):
        ice = w.ice_at(step)
        g.update(ice, w.dt_yr)
        o.update(ice, w.dt_yr)
    assert o.info().n_reject > 0
    check_models(g, o)


def test_guard_collapse_returns_status():
    w = synth.Workload("t", 12, 16, 100.0, 2, 2, "ramp", sle=False, visc3d=False, seed=22)
    g, o = pair(w)
    for m in (g, o):
        m.set_reference(*w.reference())
        m.update(w.ice_at(40), w.dt_yr)
    state, t = g.state()
    state = [a.copy() for a in state]
    state[0][5] = np.nan
    msgs = []
    for m in (g, o):
        m.set_state(state, t)
        with pytest.raises(Exception) as ei:
            m.update(w.ice_at(41), w.dt_yr)
        msgs.append(str(ei.value))
    for s in msgs:
        assert "explicit guard sub-step collapsed" in s, s
    assert g.info().n_reject == o.info().n_reject > 30


def test_singular_operator_returns_status():
    layers = [(rb, rt, 0.0, 0.0, eta, rh) if i < 3 else synth.EARTH4[i]
              for i, (rb, rt, _rho, _mu, eta, rh) in enumerate(synth.EARTH4)]
    errs = []
    for mk, cls in ((vlib.default_params, vlib.Model), (orc.default_params, orc.Oracle)):
        p = mk()
        p.lmax, p.nlat, p.nphi = 8, 9, 18
        from fastearth3d_b200.abi import set_layers

        set_layers(p, layers)
        for i, c in enumerate((2, 3, 3, 3)):
            p.ne_layer[i] = c
        with pytest.raises(Exception) as ei:
            cls(p)
        errs.append(str(ei.value))
    assert "zero pivot" in errs[0] and "band LU factorization failed" in errs[1], errs


def test_wait_limit_runs_out_and_reports():
    w = synth.Workload("t", 24, 24, 100.0, 2, 3, "sawtooth", sle=True, visc3d=False, seed=23)
    g = vlib.Model(w.params(vlib.default_params))
    g.set_reference(*w.reference())
    with pytest.raises(Exception):
        vlib.Model._c(g, vlib.lib().vg_set_wait_limit(g.h, -1.0))
    g._c(vlib.lib().vg_set_wait_limit(g.h, 0.0))
    with pytest.raises(Exception) as ei:
        g.update(w.ice_at(200), w.dt_yr)
    assert "timed out" in str(ei.value), str(ei.value)
    g.close()
    # the device is still usable: a fresh model matches the oracle
    g2 = vlib.Model(w.params(vlib.default_params))
    o2 = orc.Oracle(w.params(orc.default_params))
    for m in (g2, o2):
        m.set_reference(*w.reference())
        m.update(w.ice_at(200), w.dt_yr)
    check_models(g2, o2)
