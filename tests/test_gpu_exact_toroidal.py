"""The toroidal channels (toroidal = 1) on the exact tensor-core 3-D path
(visc3d_precision = EXACT_TC) against the FP64 3-D path and the oracle.

With W carried, the exact stages take ten synthesis products (P.X4, D.X4,
H.X5, G.X5 beside the spheroidal six, each added to its dyadic component in
the inverse stage) and ten analysis quadratures (wD.RP, wP.(m/sin)RT, wG.TP,
wH.(TT - PP) beside the six). Stated tolerances, as for the spheroidal exact
path: rsl and z_bed within 1e-9 of the FP64 path on full updates with the sea
level at lmax 12 and 33 (odd: no equatorial row), the spheroidal and the
toroidal memory within 1e-8 (the internal state amplifies last-bit
differences), identical ocean function and sub-step counts; within 1e-9 of
the oracle at lmax 12; the lmax-128 3-D workload of the benchmark with W
carried, rsl within 1e-8 of the FP64 path over 6 intervals.
"""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import VG_VISC3D_EXACT_TC, VG_VISC3D_FP64
from oracle import orc

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    return np.abs(a - b).max() / s if s > 0 else np.abs(a - b).max()


def build(mk, w, precision=None):
    p = w.params(mk.default_params)
    p.toroidal = 1
    if precision is not None:
        p.visc3d_precision = precision
    m = vlib.Model(p) if mk is vlib else orc.Oracle(p)
    m.set_reference(*w.reference())
    m.enable_visc3d(w.pert(m.p))
    return m


def run(ms, w, steps):
    for s in steps:
        ice = w.ice_at(s)
        for m in ms:
            m.update(ice, w.dt_yr)


@pytest.mark.parametrize("lmax,ne", [(12, 16), (33, 24)])
def test_exact_toroidal_vs_fp64(lmax, ne):
    w = synth.Workload("tor_exact", lmax, ne, 100.0, 4, 2, "sawtooth", sle=True, visc3d=True, seed=5)
    ex = build(vlib, w, VG_VISC3D_EXACT_TC)
    fp = build(vlib, w, VG_VISC3D_FP64)
    assert ex.info().ne3d == fp.info().ne3d > 0
    run((ex, fp), w, (80, 160, 240, 320))
    re_, ze, ce, _ = ex.fields()
    rf, zf, cf, _ = fp.fields()
    assert np.array_equal(ce, cf)
    assert ex.info().n_sub_last == fp.info().n_sub_last
    assert rel(re_, rf) < 1e-9 and rel(ze, zf) < 1e-9, (rel(re_, rf), rel(ze, zf))
    for a, b in zip(ex.state()[0], fp.state()[0]):
        assert rel(a, b) < 1e-8
    te, tf = ex.state_tor(), fp.state_tor()
    assert max(np.abs(x).max() for x in tf) > 0.0
    worst = max(rel(a, b) for a, b in zip(te, tf))
    print("lmax %d: rsl %.2e, toroidal memory %.2e" % (lmax, rel(re_, rf), worst))
    assert worst < 1e-8
    assert rel(ex.toroidal(), fp.toroidal()) < 1e-8


def test_exact_toroidal_vs_oracle():
    w = synth.Workload("tor_exact", 12, 16, 100.0, 4, 2, "sawtooth", sle=True, visc3d=True, seed=7)
    ex = build(vlib, w, VG_VISC3D_EXACT_TC)
    o = build(orc, w)
    run((ex, o), w, (80, 160, 240))
    assert rel(ex.fields()[0], o.fields()[0]) < 1e-9
    for a, b in zip(ex.state_tor(), o.state_tor()):
        assert rel(a, b) < 1e-8


def test_exact_toroidal_full_size_rsl_within_1e8():
    w = synth.workloads()["c3_3d_l128"]
    ex = build(vlib, w, VG_VISC3D_EXACT_TC)
    fp = build(vlib, w, VG_VISC3D_FP64)
    worst = 0.0
    for s in range(400, 406):
        run((ex, fp), w, (s,))
        worst = max(worst, rel(ex.fields()[0], fp.fields()[0]))
        assert ex.info().n_sub_last == fp.info().n_sub_last
    print("lmax-128 3-D workload with W, 6 intervals: rsl %.3e" % worst)
    assert worst <= 1e-8
