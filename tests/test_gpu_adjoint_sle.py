"""The adjoint of the coupled time step (vg_sle_misfit_grad): the gradient of
an rsl misfit at land sites over intervals of vg_update (forward-Euler
sub-steps, the sea-level equation with its migrating coastline, lateral
viscosity on the FP64 path) with respect to the interval-end ice thickness on
the Gauss grid and to the spectrum of the lateral log10-viscosity field,
against central finite differences (h = 1e-6 relative) along 20 seeded random
directions each, of both the GPU forward (vg_sle_misfit) and the oracle's
forward (its own update, the CPU restatement of the reference). With the
forward's discrete decisions fixed the misfit is quadratic in the ice, so the
differences are exact up to rounding; in the viscosity they carry an O(h^2)
truncation. Stated tolerance: 1e-6 relative to the larger of the two
directional derivatives (and to the gradient's scale along the direction, so
that a direction the misfit barely sees is not judged on its rounding)."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import VG_VISC3D_FP64
from oracle import orc

pytestmark = pytest.mark.gpu

LMAX, NE, DT, NSTEPS, NSITE, FIRST = 32, 40, 50.0, 8, 60, 160
TOL = 1e-6


def workload():
    return synth.Workload("adj_sle", LMAX, NE, DT, 1000, 4, "sawtooth", sle=True, visc3d=True, seed=31)


def spectrum(rng, lmax_field, scale):
    nlm = (LMAX + 1) * (LMAX + 2) // 2
    q = np.zeros(nlm, complex)
    for m in range(lmax_field + 1):
        for l in range(max(m, 1), lmax_field + 1):
            q[synth.lmidx(LMAX, l, m)] = scale / l * (rng.standard_normal() + (1j * rng.standard_normal() if m else 0))
    return q


def build(kind, w, q, toroidal=0):
    mk = vlib if kind == "gpu" else orc
    p = w.params(mk.default_params)
    p.skip_tol = 0.0
    p.toroidal = toroidal
    if kind == "gpu":
        p.visc3d_precision = VG_VISC3D_FP64
    m = vlib.Model(p) if kind == "gpu" else orc.Oracle(p)
    m.set_reference(*w.reference())
    w.pert2d = synth.synthesize(q, LMAX, w.nlat, w.nphi)
    m.enable_visc3d(w.pert(p))
    return m


def run_misfit(m, ice, sites, obs):
    """J by plain updates and field reads (the public interval call)."""
    J = 0.0
    for n in range(len(ice)):
        m.update(ice[n], DT)
        r = m.fields()[0]
        J += float(np.sum((r[sites] - obs[n]) ** 2))
    return J


@pytest.fixture(scope="module")
def case():
    w = workload()
    rng = np.random.default_rng(17)
    q0 = spectrum(rng, 12, 0.25)
    ice = np.stack([w.ice_at(FIRST + n + 1) for n in range(NSTEPS)])
    land = np.flatnonzero(w.topo.reshape(-1) > 0.0)
    sites = rng.choice(land, NSITE, replace=False).astype(np.int32)
    # observations: a truth run with a stronger lateral field and 5 % less ice, plus noise
    truth = build("gpu", w, 1.3 * q0)
    obs = np.zeros((NSTEPS, NSITE))
    for n in range(NSTEPS):
        truth.update(0.95 * ice[n], DT)
        obs[n] = truth.fields()[0][sites] + 0.05 * rng.standard_normal(NSITE)
    return w, rng, q0, ice, sites, obs


def test_sle_misfit_equals_updates_and_oracle(case):
    w, rng, q0, ice, sites, obs = case
    g = build("gpu", w, q0)
    before = g.fields()
    J = g.sle_misfit(ice, DT, sites, obs)
    after = g.fields()
    for a, b in zip(before, after):  # the handle's state is put back
        assert np.array_equal(a, b)
    assert g.info().ne3d > 0
    Ju = run_misfit(build("gpu", w, q0), ice, sites, obs)
    Jo = run_misfit(build("orc", w, q0), ice, sites, obs)
    assert abs(J - Ju) <= 1e-14 * J, (J, Ju)  # the same fields; the sums differ in order
    assert abs(J - Jo) <= 1e-10 * J, (J, Jo)


def test_sle_gradient_checkpoints_and_state(case):
    w, rng, q0, ice, sites, obs = case
    g = build("gpu", w, q0)
    s0, _ = g.state()
    out = [g.sle_misfit_grad(ice, DT, sites, obs, ckpt_every=c, want_pert=True) for c in (1, 3, NSTEPS)]
    for o in out[1:]:
        assert o[0] == out[0][0]
        for a, b in zip(o[1:], out[0][1:]):
            assert np.array_equal(a, b)
    s1, _ = g.state()
    for a, b in zip(s0, s1):
        assert np.array_equal(a, b)
    J, gi, gp, gq = out[0]
    assert J == g.sle_misfit(ice, DT, sites, obs)
    assert np.abs(gi).max() > 0 and np.abs(gq).max() > 0
    # the spectral gradient is the synthesis transpose of the grid gradient summed over the 3-D elements
    nlm = gq.size
    for lm in (synth.lmidx(LMAX, 3, 0), synth.lmidx(LMAX, 5, 2)):
        e = np.zeros(nlm, complex)
        e[lm] = 1.0
        f = synth.synthesize(e, LMAX, w.nlat, w.nphi)
        assert abs(np.sum(gp * f[None]) - gq[lm].real) <= 1e-9 * np.abs(gq).max()


def directional(gi, d):
    return float(np.sum(gi * d))


def check(fd, ad, scale, worst):
    err = abs(fd - ad) / max(abs(fd), abs(ad), scale)
    worst.append(err)
    assert err <= TOL, (fd, ad, scale)


@pytest.mark.parametrize("forward", ["gpu", "oracle"])
def test_sle_gradient_ice_vs_central_differences(case, forward):
    w, rng, q0, ice, sites, obs = case
    g = build("gpu", w, q0)
    J, gi = g.sle_misfit_grad(ice, DT, sites, obs, ckpt_every=3)
    gi = gi.reshape(NSTEPS, -1)
    rs = np.random.default_rng(101)
    h = 1e-6
    worst = []
    for _ in range(20):
        # smooth-ish direction: the ice pattern with random per-interval weights plus white noise on the caps
        d = rs.standard_normal((NSTEPS, 1)) * ice + 100.0 * rs.standard_normal(ice.shape) * (ice > 0)
        ad = directional(gi, d)
        scale = np.sqrt(np.sum(gi * gi) * np.sum(d * d)) * 1e-3
        if forward == "gpu":
            jp = g.sle_misfit(ice + h * d, DT, sites, obs)
            jm = g.sle_misfit(ice - h * d, DT, sites, obs)
        else:
            jp = run_misfit(build("orc", w, q0), ice + h * d, sites, obs)
            jm = run_misfit(build("orc", w, q0), ice - h * d, sites, obs)
        check((jp - jm) / (2 * h), ad, scale, worst)
    print("ice gradient vs central differences of the %s forward: worst relative error %.2e" % (forward, max(worst)))


@pytest.mark.parametrize("forward", ["gpu", "oracle"])
def test_sle_gradient_viscosity_vs_central_differences(case, forward):
    w, rng, q0, ice, sites, obs = case
    g = build("gpu", w, q0)
    J, gi, gp, gq = g.sle_misfit_grad(ice, DT, sites, obs, ckpt_every=4, want_pert=True)
    rs = np.random.default_rng(202)
    h = 1e-6
    worst = []
    for _ in range(20):
        dq = spectrum(rs, 12, 1.0)  # coefficients to degree 12 of the lateral field
        ad = float(np.sum(gq.real * dq.real + gq.imag * dq.imag))
        scale = np.sqrt(np.sum(np.abs(gq) ** 2) * np.sum(np.abs(dq) ** 2)) * 1e-3
        if forward == "gpu":
            jp = build("gpu", w, q0 + h * dq).sle_misfit(ice, DT, sites, obs)
            jm = build("gpu", w, q0 - h * dq).sle_misfit(ice, DT, sites, obs)
        else:
            jp = run_misfit(build("orc", w, q0 + h * dq), ice, sites, obs)
            jm = run_misfit(build("orc", w, q0 - h * dq), ice, sites, obs)
        check((jp - jm) / (2 * h), ad, scale, worst)
    print("viscosity gradient vs central differences of the %s forward: worst relative error %.2e" % (
        forward, max(worst)))


@pytest.mark.parametrize("forward", ["gpu", "oracle"])
def test_sle_gradient_with_toroidal_channels_vs_central_differences(case, forward):
    """With toroidal = 1 the lateral viscosity also drives W, and the reverse
    sweep runs its transposes (the lambda 3, 4 advance, the W drift, the
    ten-product 3-D chain): the viscosity gradient against central
    differences along 10 seeded directions, of the GPU and the oracle
    forwards with W carried."""
    w, rng, q0, ice, sites, obs = case
    g = build("gpu", w, q0, toroidal=1)
    assert g.state_tor() is not None
    J, gi, gp, gq = g.sle_misfit_grad(ice, DT, sites, obs, ckpt_every=3, want_pert=True)
    rs = np.random.default_rng(303)
    h = 1e-6
    worst = []
    for _ in range(10):
        dq = spectrum(rs, 12, 1.0)
        ad = float(np.sum(gq.real * dq.real + gq.imag * dq.imag))
        scale = np.sqrt(np.sum(np.abs(gq) ** 2) * np.sum(np.abs(dq) ** 2)) * 1e-3
        if forward == "gpu":
            jp = build("gpu", w, q0 + h * dq, toroidal=1).sle_misfit(ice, DT, sites, obs)
            jm = build("gpu", w, q0 - h * dq, toroidal=1).sle_misfit(ice, DT, sites, obs)
        else:
            jp = run_misfit(build("orc", w, q0 + h * dq, toroidal=1), ice, sites, obs)
            jm = run_misfit(build("orc", w, q0 - h * dq, toroidal=1), ice, sites, obs)
        check((jp - jm) / (2 * h), ad, scale, worst)
    print("viscosity gradient with W vs central differences of the %s forward: worst relative error %.2e" % (
        forward, max(worst)))
