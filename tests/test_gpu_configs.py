"""Device FP64 path against the oracle at the benchmark configurations'
full sizes, through the C-ABI, on the same seeded inputs:

  configuration 1  1-D, lmax 64 (65 x 130), 60 radial elements, ice ramp,
                   no ocean, 10 intervals of 50 yr
  configuration 2  1-D, lmax 128 (129 x 258), 100 elements, sea-level
                   equation with migrating coastlines and rotation, 4
                   intervals of 100 yr
  configuration 3  lateral viscosity, lmax 128 (129 x 258), 100 elements
                   (54 of them 3-D), sea-level equation, 3 intervals of 50
                   yr with 3 Maxwell sub-steps each (the timed workload of
                   bench.py)

Outputs (rsl, z_bed, the load spectrum) to 1e-10 relative to their maximum,
the memory to 1e-8, identical ocean function, sub-step counts and
accepted / rejected sub-steps (parity_util)."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from oracle import orc
from parity_util import TOL, check_models

pytestmark = pytest.mark.gpu


def run_pair(w, steps):
    g = vlib.Model(w.params(vlib.default_params))
    o = orc.Oracle(w.params(orc.default_params))
    if w.visc3d:
        pert = w.pert(g.p)
        g.enable_visc3d(pert)
        o.enable_visc3d(pert)
        assert g.info().ne3d == o.info().ne3d > 0
    zb, hi = w.reference()
    g.set_reference(zb, hi)
    o.set_reference(zb, hi)
    for s in steps:
        ice = w.ice_at(s)
        g.update(ice, w.dt_yr)
        o.update(ice, w.dt_yr)
    return g, o


def test_config1_full_size():
    w = synth.workloads()["c1_1d_l64"]
    assert (w.lmax, w.nlat, w.nphi, w.n_elem) == (64, 65, 130, 60)
    g, o = run_pair(w, range(40, 401, 40))  # the 20-kyr ramp in 10 intervals
    check_models(g, o)
    assert g.info().n_sub_last == 1


def test_config2_full_size_with_rotation():
    w = synth.workloads()["c2_1d_sle_l128"]
    assert (w.lmax, w.n_elem, w.sle, w.rotation) == (128, 100, True, True)
    g, o = run_pair(w, (300, 301, 302, 303))
    check_models(g, o)
    mg, _ = g.rotation()
    mo, _ = o.rotation()
    assert abs(mg - mo) <= TOL * abs(mo)
    assert g.info().worst_mass_resid < 1e-10
    ig, io = g.info(), o.info()
    assert (ig.n_outer_last, ig.n_inner_last, ig.n_coast_flip_last) == (io.n_outer_last, io.n_inner_last,
                                                                         io.n_coast_flip_last)


def test_config3_full_size_3d():
    w = synth.workloads()["c3_3d_l128"]
    assert (w.lmax, w.n_elem, w.visc3d, w.sle) == (128, 100, True, True)
    g, o = run_pair(w, (400, 401, 402))
    errs = check_models(g, o)
    assert g.info().n_sub_last == o.info().n_sub_last == 3
    assert g.info().ne3d == 54
    print("config 3 FP64 vs oracle:", errs)
