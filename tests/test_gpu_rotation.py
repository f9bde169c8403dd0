"""Rotational feedback on the device (src/vilma_rotation.f90, coupled as
src/vilma_coupling.f90:399-424) against the oracle's restatement, which is
pinned to the Spada 2011 Test 3/2 polar motion (tests/test_oracle_golden.py).
FP64 path: 1e-10 relative on rsl, z_bed and the polar motion."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from oracle import orc

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    return np.abs(a - b).max() / s if s > 0 else np.abs(a - b).max()


def models(w):
    g = vlib.Model(w.params(vlib.default_params))
    o = orc.Oracle(w.params(orc.default_params))
    zb, hi = w.reference()
    for m in (g, o):
        m.set_reference(zb, hi)
    if w.visc3d:
        pert = w.pert(g.p)
        g.enable_visc3d(pert)
        o.enable_visc3d(pert)
    return g, o


def test_rotation_constants_match_oracle():
    w = synth.Workload("rot", 16, 20, 100.0, 2, 2, "sawtooth", sle=True, visc3d=False, seed=7, rotation=True)
    g, o = models(w)
    _, lg = g.rotation()
    _, lo = o.rotation()
    assert rel(lg, lo) < TOL


@pytest.mark.parametrize("lmax,visc3d", [(16, False), (24, True)])
def test_rotation_update_parity(lmax, visc3d):
    w = synth.Workload("rot", lmax, 20, 100.0, 4, 3, "sawtooth", sle=True, visc3d=visc3d, seed=11, rotation=True)
    g, o = models(w)
    for step in range(1, 5):
        ice = w.ice_at(step * 300)
        g.update(ice, w.dt_yr)
        o.update(ice, w.dt_yr)
        mg, _ = g.rotation()
        mo, _ = o.rotation()
        assert abs(mg - mo) <= TOL * abs(mo)
        rg, zg, Cg, _ = g.fields()
        ro, zo, Co, _ = o.fields()
        assert rel(rg, ro) < TOL and rel(zg, zo) < TOL
        assert np.array_equal(Cg, Co)
    assert abs(mg) > 0.0


def test_rotation_changes_sea_level():
    """The centrifugal term is really fed into the sea-level equation: the same
    run without rotation gives a different rsl (at the degree-2 order-1 level)."""
    kw = dict(sle=True, visc3d=False, seed=11)
    w1 = synth.Workload("rot", 16, 20, 100.0, 3, 3, "sawtooth", rotation=True, **kw)
    w0 = synth.Workload("rot", 16, 20, 100.0, 3, 3, "sawtooth", rotation=False, **kw)
    a, _ = models(w1)
    b, _ = models(w0)
    for step in range(1, 4):
        a.update(w1.ice_at(step * 300), w1.dt_yr)
        b.update(w0.ice_at(step * 300), w0.dt_yr)
    ra, rb = a.fields()[0], b.fields()[0]
    assert rel(ra, rb) > 1e-8
