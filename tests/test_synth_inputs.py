"""The seeded synthetic inputs that stand in for the benchmark workloads have
the shapes, sizes and value distributions the workloads are stated with:
the 4-layer earth, the ice caps and their histories, the topography's mean
and spread, the lateral log-viscosity's spread and clip, and the ensemble's
parameter ranges."""
import numpy as np

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import VG_RHEOL_ELASTIC, VG_RHEOL_FLUID, VG_RHEOL_MAXWELL


def test_earth_layers():
    (l0, l1, l2, core) = synth.EARTH4
    assert l0[:2] == (6301.0e3, 6371.0e3) and l0[2:4] == (3300.0, 0.7e11) and l0[5] == VG_RHEOL_ELASTIC
    assert l1[:2] == (5701.0e3, 6301.0e3) and l1[2:5] == (3450.0, 0.9e11, 5e20) and l1[5] == VG_RHEOL_MAXWELL
    assert l2[:2] == (3480.0e3, 5701.0e3) and l2[2:5] == (4900.0, 2.0e11, 2e21) and l2[5] == VG_RHEOL_MAXWELL
    assert core[1] == 3480.0e3 and core[2] == 10900.0 and core[5] == VG_RHEOL_FLUID


def test_workload_sizes():
    ws = synth.workloads()
    c1, c2, c3 = ws["c1_1d_l64"], ws["c2_1d_sle_l128"], ws["c3_3d_l128"]
    assert (c1.lmax, c1.nlat, c1.nphi, c1.n_elem, c1.dt_yr, c1.history) == (64, 65, 130, 60, 50.0, "ramp")
    assert not c1.sle and not c1.visc3d and not c1.rotation
    assert (c2.lmax, c2.nlat, c2.nphi, c2.n_elem, c2.dt_yr) == (128, 129, 258, 100, 100.0)
    assert c2.sle and c2.rotation and not c2.visc3d and c2.history == "sawtooth"
    assert (c3.lmax, c3.n_elem, c3.dt_yr) == (128, 100, 50.0) and c3.sle and c3.visc3d
    for w in (c1, c2, c3):
        p = w.params(vlib.default_params)
        assert sum(p.ne_layer[i] for i in range(4)) == w.n_elem


def test_topography_and_lateral_viscosity():
    c3 = synth.workloads()["c3_3d_l128"]
    assert abs(c3.topo.mean() - (-1500.0)) < 1e-6 and abs(c3.topo.std() - 2500.0) < 1e-6
    f = synth.random_sh_field(c3.seed + 2, 32, c3.lmax, c3.nlat, c3.nphi, 0.4, 0.0)
    assert abs(f.std() - 0.4) < 1e-12 and abs(f.mean()) < 1e-12
    assert np.array_equal(c3.pert2d, np.clip(f, -1.0, 1.0))
    assert np.abs(c3.pert2d).max() <= 1.0


def test_ice_caps_and_histories():
    c3 = synth.workloads()["c3_3d_l128"]
    ice = c3.ice_full
    assert ice.min() >= 0.0 and 1000.0 <= ice.max() <= 6 * 3000.0
    assert np.allclose(synth.ramp(np.array([0.0, 10000.0, 20000.0, 30000.0])), [0.0, 0.5, 1.0, 1.0])
    s = synth.sawtooth(np.array([0.0, 45000.0, 90000.0, 95000.0, 100000.0]))
    assert np.allclose(s, [0.0, 0.5, 1.0, 0.5, 0.0])
    assert np.allclose(c3.ice_at(900).reshape(ice.shape), ice * synth.sawtooth(900 * c3.dt_yr))


def test_ensemble_ranges():
    ms = synth.ensemble()
    assert len(ms) == 32
    assert {m.lmax for m in ms} <= {64, 96, 128, 192, 256}
    assert sum(m.visc3d for m in ms) == 16
    for m in ms:
        assert 1e20 <= m.eta_um <= 1e21 and 1e21 <= m.eta_lm <= 1e23 and 50.0 <= m.litho_km <= 120.0
        assert m.n_elem == {64: 60, 96: 80}.get(m.lmax, 100)
