"""The trapezoidal scheme (scheme = "trap") on the GPU against the oracle: the
sea-level <-> memory co-convergence, the endpoint drift, the 1-D and 3-D
trapezoid advance and the step-doubling controller, through vg_update on the
same seeded inputs. FP64 path: 1e-10 relative on rsl, z_bed and the load, the
controller's decisions (accepted and rejected steps) identical. The split
tensor-core 3-D path against the FP64 path: 1e-6 on rsl (as for forward Euler)
with every trial step accepted, so both take the same steps."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import VG_VISC3D_FP64, VG_VISC3D_SPLIT_TC
from oracle import orc

pytestmark = pytest.mark.gpu
TOL = 1e-10
TOL_STATE = 1e-8


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    d = np.abs(a - b).max()
    return d / s if s > 0 else d


def trap_params(w, mk, **kw):
    p = w.params(mk)
    p.scheme = 2
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def run_pair(w, n_steps, stride, **kw):
    g = vlib.Model(trap_params(w, vlib.default_params, **kw))
    o = orc.Oracle(trap_params(w, orc.default_params, **kw))
    zb, hi = w.reference()
    for m in (g, o):
        m.set_reference(zb, hi)
    if w.visc3d:
        g.enable_visc3d(w.pert(g.p))
        o.enable_visc3d(w.pert(o.p))
    for step in range(1, n_steps + 1):
        ice = w.ice_at(step * stride)
        g.update(ice, w.dt_yr)
        o.update(ice, w.dt_yr)
    return g, o


def check(g, o):
    rg, zg, cg, sg = g.fields()
    ro, zo, co, so = o.fields()
    assert np.array_equal(cg, co), "ocean function differs"
    assert rel(rg, ro) < TOL
    assert rel(zg, zo) < TOL
    assert rel(sg, so) < TOL
    (stg, tg), (sto, to) = g.state(), o.state()
    for a, b in zip(stg, sto):
        assert rel(a, b) < TOL_STATE
    assert abs(tg - to) <= 1e-9 * abs(to)
    ig, io = g.info(), o.info()
    assert (ig.n_accept, ig.n_reject, ig.n_sub_last) == (io.n_accept, io.n_reject, io.n_sub_last)


def test_trap_update_parity_with_sea_level():
    w = synth.Workload("t", 16, 24, 200.0, 6, 3, "sawtooth", sle=True, visc3d=False, seed=3)
    g, o = run_pair(w, 4, stride=60)
    assert o.info().n_accept >= 4 and o.info().n_reject > 0  # the controller both accepts and rejects
    check(g, o)


def test_trap_visc3d_parity():
    w = synth.Workload("t", 12, 16, 100.0, 4, 2, "sawtooth", sle=True, visc3d=True, seed=5)
    g, o = run_pair(w, 3, stride=80)
    assert g.info().ne3d > 0
    check(g, o)


def test_trap_split_tc_vs_fp64():
    w = synth.Workload("t", 32, 40, 50.0, 8, 3, "sawtooth", sle=True, visc3d=True, seed=5)
    ms = []
    for prec in (VG_VISC3D_FP64, VG_VISC3D_SPLIT_TC):
        p = trap_params(w, vlib.default_params, rtol=1e30, atol=1e30, visc3d_precision=prec)
        m = vlib.Model(p)
        zb, hi = w.reference()
        m.set_reference(zb, hi)
        m.enable_visc3d(w.pert(m.p))
        ms.append(m)
    worst = 0.0
    for step in range(1, 6):
        ice = w.ice_at(step * 400)
        for m in ms:
            m.update(ice, w.dt_yr)
        (r0, *_), (r1, *_) = ms[0].fields(), ms[1].fields()
        worst = max(worst, np.abs(r1 - r0).max() / np.abs(r0).max())
    assert ms[0].info().n_accept == ms[1].info().n_accept == 5
    assert worst < 1e-6, worst
