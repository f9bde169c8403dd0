"""vg_spinup (solid_earth_spinup's relaxation) against the oracle on the
reference test's setup (tests/test_spinup.f90), and full-update parity on the
reference-native radial mesh (per-layer element counts unset: the depth-target
rule of src/vilma_radial_fe.f90:140-224 gives 14 + 60 + 56 + 87 = 217 elements
for the default earth)."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from oracle import orc

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    return np.abs(a - b).max() / s if s > 0 else np.abs(a - b).max()


def spin_setup(mk, model):
    p = mk()
    p.lmax, p.nlat, p.nphi = 16, 32, 64
    m = model(p)
    return m, p


def test_spinup_parity_with_oracle():
    g, pg = spin_setup(vlib.default_params, vlib.Model)
    o, po = spin_setup(orc.default_params, orc.Oracle)
    colat, _ = o.grid()
    cd = np.rad2deg(colat)[:, None] * np.ones((1, pg.nphi))
    z_eq = np.where(cd < 50.0, 500.0, -4000.0).reshape(-1)
    ice = np.where(cd < 30.0, 2000.0, 0.0).reshape(-1)
    for m in (g, o):
        m.set_reference(z_eq, np.zeros_like(z_eq))
    rg = g.spinup(ice, 5.0e5, 1e-3)
    ro = o.spinup(ice, 5.0e5, 1e-3)
    assert rg[1:] == ro[1:] and abs(rg[0] - ro[0]) <= 1e-9 * ro[0], (rg, ro)
    assert rg[2]  # came to rest before the cap
    (rsg, zg, cg, _), (rso, zo, co, _) = g.fields(), o.fields()
    assert np.array_equal(cg, co)
    assert rel(zg, zo) < 1e-10 and rel(rsg, rso) < 1e-10
    assert g.spinup(ice, 0.0, 1e-3) == (0.0, 0, False)


def test_pre_spinup_1d_parity_3d():
    """The 1-D pre-equilibration on the lateral mean of a 3-D field, then the
    full-model phase with the field restored: passes, model time and fields
    as the oracle's."""
    w = synth.Workload("s", 12, 16, 100.0, 2, 2, "sawtooth", sle=True, visc3d=True, seed=8)
    g, o = vlib.Model(w.params(vlib.default_params)), orc.Oracle(w.params(orc.default_params))
    zb, hi = w.reference()
    for m in (g, o):
        m.set_reference(zb, hi)
        m.enable_visc3d(w.pert(m.p))
    ne3d = g.info().ne3d
    rg = g.spinup(w.ice_at(400), 2000.0, 1e-3, pre_1d=True, with_1d=True)
    ro = o.spinup(w.ice_at(400), 2000.0, 1e-3, pre_1d=True, with_1d=True)
    assert rg[1:] == ro[1:] and abs(rg[0] - ro[0]) <= 1e-9 * ro[0], (rg, ro)
    assert rg[3] > 0 and g.info().ne3d == ne3d
    (rsg, zg, cg, _), (rso, zo, co, _) = g.fields(), o.fields()
    assert np.array_equal(cg, co)
    assert rel(zg, zo) < 1e-10 and rel(rsg, rso) < 1e-10


def test_reference_native_mesh_parity():
    w = synth.Workload("t", 16, 0, 100.0, 2, 2, "sawtooth", sle=True, visc3d=False, seed=4)
    ps = []
    for mk in (vlib.default_params, orc.default_params):
        p = w.params(mk)
        for i in range(16):
            p.ne_layer[i] = 0  # the reference's depth-target rule
        ps.append(p)
    g, o = vlib.Model(ps[0]), orc.Oracle(ps[1])
    assert g.info().ne == o.info().ne == 217
    zb, hi = w.reference()
    for m in (g, o):
        m.set_reference(zb, hi)
    for step in (1, 2):
        ice = w.ice_at(step * 300)
        g.update(ice, w.dt_yr)
        o.update(ice, w.dt_yr)
    (rg, zg, cg, sg), (ro, zo, co, so) = g.fields(), o.fields()
    assert np.array_equal(cg, co)
    assert rel(rg, ro) < 1e-10 and rel(zg, zo) < 1e-10 and rel(sg, so) < 1e-10
