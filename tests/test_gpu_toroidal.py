"""The toroidal degree of freedom (toroidal = 1) on the GPU against the oracle.

Response level (the protocol of tests/test_toroidal.f90: a held 1 km Y20
load over M3-L70-V01 whose Maxwell layers carry delta sin^2(theta) cos(2 phi))
through vg_response_*: uplift U(a) and the toroidal W(a) to 1e-10 relative,
with the GPU's own selection rule (U real / W imaginary at even m, nothing at
odd m) and the axisymmetric null. Full updates (sea level, FE and trapezoidal
schemes) on a laterally varying synthetic earth: rsl, the spheroidal and the
toroidal memory to the same tolerances as the spheroidal 3-D tests, the
trapezoidal controller's decisions identical. Restart with the toroidal
memory continues bit for bit; the combination the product does not carry
(the two-term TF32 tensor-core precision) fails loudly.
"""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import M3L70V01, VG_VISC3D_SPLIT_TC, set_layers
from oracle import orc

pytestmark = pytest.mark.gpu
TOL = 1e-10
TOL_STATE = 1e-8
LMAX, NSTEP = 12, 40


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    d = np.abs(a - b).max()
    return d / s if s > 0 else d


def lm_of(L):
    ls, ms = [], []
    for m in range(L + 1):
        for l in range(m, L + 1):
            ls.append(l)
            ms.append(m)
    return np.array(ls), np.array(ms)


def run_held(model, p, delta, axisym, colat):
    lon = 2 * np.pi * np.arange(p.nphi) / p.nphi
    st, ct = np.sin(colat)[:, None], np.cos(colat)[:, None]
    pat = ct * ct + 0 * lon[None, :] if axisym else st * st * np.cos(2 * lon)[None, :]
    elem_layers = []
    for i in range(p.n_layer - 1, -1, -1):
        elem_layers += [i] * p.ne_layer[i]
    pert = np.zeros((len(elem_layers), p.nlat, p.nphi))
    for e, L in enumerate(elem_layers):
        if M3L70V01[L][5] == 1:
            pert[e] = delta * pat
    model.enable_visc3d(pert.reshape(-1))
    s = np.zeros(model.nlm, complex)
    s[synth.lmidx(LMAX, 2, 0)] = 1.0e3
    for _ in range(NSTEP):
        model.begin_step()
        model.apply(s)
        model.advance(s)
    model.begin_step()
    u, _ = model.apply(s)
    return u, model.toroidal()


def held_pair(delta, axisym):
    out = []
    for mk in (vlib.default_params, orc.default_params):
        p = mk()
        set_layers(p, M3L70V01)
        p.lmax, p.nlat, p.nphi = LMAX, 3 * LMAX, 3 * LMAX
        p.ne_layer[:5] = [3, 6, 4, 8, 2]
        p.toroidal = 1
        p.dt_init = 40.0 * synth.SEC_PER_YEAR
        m = vlib.Model(p) if mk is vlib.default_params else orc.Oracle(p)
        m.set_dt(p.dt_init)
        o = orc.Oracle(p) if mk is vlib.default_params else m
        colat, _ = o.grid()
        out.append(run_held(m, p, delta, axisym, colat))
    return out


def test_held_load_toroidal_parity_and_selection_rule():
    (ug, tg), (uo, to) = held_pair(0.2, False)
    assert np.abs(to).max() > 1e-6 * np.abs(uo).max()  # W is driven
    assert rel(ug, uo) < TOL
    assert rel(tg, to) < TOL
    ls, ms = lm_of(LMAX)
    odd = ms % 2 == 1
    wmax, umax = np.abs(tg).max(), np.abs(ug).max()
    err = max(np.abs(ug[odd]).max() / umax, np.abs(tg[odd]).max() / wmax)
    ev = ~odd & (ls >= 1)
    err = max(err, np.abs(ug[ev].imag).max() / umax, np.abs(tg[ev].real).max() / wmax)
    assert err < 1e-10


def test_held_load_axisymmetric_null():
    (ug, tg), _ = held_pair(0.2, True)
    assert np.abs(tg).max() / np.abs(ug).max() <= 1e-12


def tor_params(w, mk, scheme=0, **kw):
    p = w.params(mk)
    p.toroidal = 1
    p.scheme = scheme
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def run_update_pair(w, n_steps, stride, scheme):
    g = vlib.Model(tor_params(w, vlib.default_params, scheme))
    o = orc.Oracle(tor_params(w, orc.default_params, scheme))
    zb, hi = w.reference()
    for m in (g, o):
        m.set_reference(zb, hi)
        m.enable_visc3d(w.pert(m.p))
    for step in range(1, n_steps + 1):
        ice = w.ice_at(step * stride)
        g.update(ice, w.dt_yr)
        o.update(ice, w.dt_yr)
    return g, o


def check_update(g, o):
    rg, zg, cg, sg = g.fields()
    ro, zo, co, so = o.fields()
    assert np.array_equal(cg, co), "ocean function differs"
    assert rel(rg, ro) < TOL
    assert rel(zg, zo) < TOL
    (stg, _), (sto, _) = g.state(), o.state()
    for a, b in zip(stg, sto):
        assert rel(a, b) < TOL_STATE
    tgm, tom = g.state_tor(), o.state_tor()
    assert tgm is not None and tom is not None
    assert max(np.abs(x).max() for x in tom) > 0.0
    for a, b in zip(tgm, tom):
        assert rel(a, b) < TOL_STATE
    assert rel(g.toroidal(), o.toroidal()) < TOL_STATE


def test_toroidal_update_parity_fe():
    w = synth.Workload("tor", 12, 16, 100.0, 4, 2, "sawtooth", sle=True, visc3d=True, seed=5)
    g, o = run_update_pair(w, 4, stride=80, scheme=0)
    assert g.info().ne3d > 0
    check_update(g, o)


def test_toroidal_update_parity_trap():
    w = synth.Workload("tor", 12, 16, 100.0, 4, 2, "sawtooth", sle=True, visc3d=True, seed=5)
    g, o = run_update_pair(w, 3, stride=80, scheme=2)
    check_update(g, o)
    ig, io = g.info(), o.info()
    assert (ig.n_accept, ig.n_reject, ig.n_sub_last) == (io.n_accept, io.n_reject, io.n_sub_last)


def test_toroidal_restart_continues_bit_for_bit():
    w = synth.Workload("tor", 12, 16, 100.0, 4, 2, "sawtooth", sle=True, visc3d=True, seed=7)

    def model():
        m = vlib.Model(tor_params(w, vlib.default_params))
        zb, hi = w.reference()
        m.set_reference(zb, hi)
        m.enable_visc3d(w.pert(m.p))
        return m

    a = model()
    for step in range(1, 3):
        a.update(w.ice_at(step * 250), w.dt_yr)
    tau, t = a.state()
    ttor = a.state_tor()
    rsl, zb, C, _ = a.fields()
    b = model()
    b.set_state(tau, t)
    b.set_state_tor(ttor)
    b.set_fields(h_ice=w.ice_at(2 * 250), rsl=rsl, z_bed=zb, C_ocean=C)
    for step in range(3, 5):
        ice = w.ice_at(step * 250)
        a.update(ice, w.dt_yr)
        b.update(ice, w.dt_yr)
        assert np.array_equal(a.fields()[0], b.fields()[0])
    for x, y in zip(a.state_tor(), b.state_tor()):
        assert np.array_equal(x, y)


def test_toroidal_refusals():
    w = synth.Workload("tor", 12, 16, 100.0, 4, 2, "sawtooth", sle=True, visc3d=True, seed=5)
    m = vlib.Model(tor_params(w, vlib.default_params, visc3d_precision=VG_VISC3D_SPLIT_TC))
    zb, hi = w.reference()
    m.set_reference(zb, hi)
    with pytest.raises(RuntimeError, match="toroidal"):
        m.enable_visc3d(w.pert(m.p))
    g = vlib.Model(tor_params(w, vlib.default_params))
    g.set_reference(zb, hi)
    g.enable_visc3d(w.pert(g.p))
    off = vlib.Model(w.params(vlib.default_params))  # toroidal = 0: nothing carried
    off.set_reference(zb, hi)
    off.enable_visc3d(w.pert(off.p))
    assert off.state_tor() is None
    assert np.abs(off.toroidal()).max() == 0.0
