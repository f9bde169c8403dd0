"""The autotuner (vg_autotune): it times its candidates from the handle's own
state and puts that state back, applies and caches its choices per model key,
a second handle of the same key reads them from the cache, and every choice
(both warp splits of the exact stages, every sea-level loop CTA count) gives
the same results bit for bit."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import VG_VISC3D_EXACT_TC

pytestmark = pytest.mark.gpu


def workload():
    return synth.Workload("tune", 32, 40, 50.0, 1000, 4, "sawtooth", sle=True, visc3d=True, seed=9)


def make(w):
    p = w.params(vlib.default_params)
    p.visc3d_precision = VG_VISC3D_EXACT_TC
    m = vlib.Model(p)
    m.set_reference(*w.reference())
    m.enable_visc3d(w.pert(m.p))
    for s in (100, 101):
        m.update(w.ice_at(s), w.dt_yr)
    return m


def run(m, w, steps=range(102, 108)):
    for s in steps:
        m.update(w.ice_at(s), w.dt_yr)
    return m.fields()[0], m.state()[0]


def test_autotune_caches_and_keeps_state(tmp_path):
    w = workload()
    cache = tmp_path / "tune.txt"
    a = make(w)
    before = a.fields()
    s_before = a.state()[0]
    assert a.autotune(w.dt_yr, cache) is False
    for x, y in zip(before, a.fields()):
        assert np.array_equal(x, y)
    for x, y in zip(s_before, a.state()[0]):
        assert np.array_equal(x, y)
    ncw, ctas = a.tuning()
    assert all(c in (4, 8) for c in ncw) and ctas >= 0
    text = cache.read_text()
    assert "lmax=32" in text and "ncw=" in text
    b = make(w)
    assert b.autotune(w.dt_yr, cache) is True
    assert b.tuning() == (ncw, ctas)
    # a tuned handle continues exactly like an untuned one
    ra, sa = run(a, w)
    rb, sb = run(make(w), w)
    assert np.array_equal(ra, rb)
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("ncw,ctas", [((4, 4, 4, 4), 33), ((8, 4, 8, 4), 296), ((4, 8, 4, 8), 0)])
def test_every_choice_gives_the_same_bits(tmp_path, ncw, ctas):
    w = workload()
    ref = make(w)
    # the cache key of this model, written by a tuning run of its own
    probe = make(w)
    path = tmp_path / "probe.txt"
    probe.autotune(w.dt_yr, path)
    key_line = path.read_text().splitlines()[0].split(" | ")[0]
    forced = tmp_path / "forced.txt"
    forced.write_text("%s | ncw=%d,%d,%d,%d sle_ctas=%d\n" % ((key_line,) + tuple(ncw) + (ctas,)))
    m = make(w)
    assert m.autotune(w.dt_yr, forced) is True
    assert m.tuning() == (list(ncw), ctas)
    r1, s1 = run(m, w)
    r0, s0 = run(ref, w)
    assert np.array_equal(r1, r0)
    for x, y in zip(s1, s0):
        assert np.array_equal(x, y)


def test_tuned_full_size_workload_continues_bit_for_bit(tmp_path):
    """The lmax-128 3-D workload of the benchmark, tuned after four intervals,
    continues exactly like an untuned handle (the drift skip gate's scale,
    the per-slot norms and the rest of the driver state are put back)."""
    w = synth.workloads()["c3_3d_l128"]

    def build():
        p = w.params(vlib.default_params)
        p.visc3d_precision = VG_VISC3D_EXACT_TC
        m = vlib.Model(p)
        m.set_reference(*w.reference())
        m.enable_visc3d(w.pert(m.p))
        for s in range(400, 404):
            m.update(w.ice_at(s), w.dt_yr)
        return m

    a, b = build(), build()
    a.autotune(w.dt_yr, tmp_path / "tune.txt")
    for s in range(404, 410):
        a.update(w.ice_at(s), w.dt_yr)
        b.update(w.ice_at(s), w.dt_yr)
    for x, y in zip(a.fields()[:3], b.fields()[:3]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("toroidal,scheme", [(1, 0), (0, 2), (1, 2)])
def test_tuning_keeps_toroidal_and_trapezoidal_state(tmp_path, toroidal, scheme):
    """Tuning from a state that carries the toroidal memory or the
    trapezoidal scheme's carried step and sigma_n puts those back too: the
    tuned handle continues bit for bit like an untuned one."""
    w = workload()

    def build():
        p = w.params(vlib.default_params)
        p.visc3d_precision = VG_VISC3D_EXACT_TC
        p.toroidal = toroidal
        p.scheme = scheme
        m = vlib.Model(p)
        m.set_reference(*w.reference())
        m.enable_visc3d(w.pert(m.p))
        for s in (100, 101):
            m.update(w.ice_at(s), w.dt_yr)
        return m

    a, b = build(), build()
    a.autotune(w.dt_yr, tmp_path / "tune.txt")
    for s in range(102, 106):
        a.update(w.ice_at(s), w.dt_yr)
        b.update(w.ice_at(s), w.dt_yr)
    assert np.array_equal(a.fields()[0], b.fields()[0])
    for x, y in zip(a.state()[0], b.state()[0]):
        assert np.array_equal(x, y)
    if toroidal:
        for x, y in zip(a.state_tor(), b.state_tor()):
            assert np.array_equal(x, y)
