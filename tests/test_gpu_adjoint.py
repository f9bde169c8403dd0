"""The hand-written adjoint of the response-level time step (vg_misfit_grad):
its gradient of the rsl misfit with respect to the load history against
central finite differences of the FP64 GPU forward (vg_misfit) along seeded
random directions, and its independence of the checkpoint interval. The
forward is linear in the load, so central differences are exact up to
rounding; the stated tolerance is 1e-6 relative."""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth

pytestmark = pytest.mark.gpu


def setup(lmax=12, nsteps=10, nsite=40, seed=3):
    p = vlib.default_params()
    p.lmax, p.nlat, p.nphi = lmax, lmax + 1, 2 * (lmax + 1)
    for i, c in enumerate([2, 6, 5, 3]):
        p.ne_layer[i] = c
    m = vlib.Model(p)
    rng = np.random.default_rng(seed)
    nlm = m.nlm

    def load_history(scale):
        s = (rng.standard_normal((nsteps, nlm)) + 1j * rng.standard_normal((nsteps, nlm))) * scale
        s[:, : lmax + 1] = s[:, : lmax + 1].real  # m = 0 coefficients of a real field
        return s

    sigma = load_history(1e3)
    truth = load_history(1e3)
    sites = rng.choice(m.ng, size=nsite, replace=False)
    dt = 100.0 * synth.SEC_PER_YEAR
    obs = np.zeros((nsteps, nsite))
    # observations: the forward's rsl for the truth history (misfit of zero obs gives -rsl)
    J0 = m.misfit(truth, dt, sites, obs)
    assert J0 > 0
    return m, sigma, truth, sites, dt, rng


def test_adjoint_gradient_vs_central_differences():
    m, sigma, truth, sites, dt, rng = setup()
    obs = 0.01 * rng.standard_normal((len(sigma), len(sites)))
    J, g = m.misfit_grad(sigma, dt, sites, obs, ckpt_every=4)
    assert abs(J - m.misfit(sigma, dt, sites, obs)) <= 1e-12 * J
    for _ in range(20):  # 20 seeded random directions
        d = rng.standard_normal(sigma.shape) + 1j * rng.standard_normal(sigma.shape)
        d[:, : m.p.lmax + 1] = d[:, : m.p.lmax + 1].real
        h = 1e-3 * np.abs(sigma).max() / np.abs(d).max()
        jp = m.misfit(sigma + h * d, dt, sites, obs)
        jm = m.misfit(sigma - h * d, dt, sites, obs)
        fd = (jp - jm) / (2 * h)
        ad = np.sum(g.real * d.real + g.imag * d.imag)
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-300), (fd, ad)


def test_adjoint_checkpoint_interval_and_state_kept():
    m, sigma, truth, sites, dt, rng = setup(nsteps=7)
    obs = np.zeros((len(sigma), len(sites)))
    s0, _ = m.state()
    J1, g1 = m.misfit_grad(sigma, dt, sites, obs, ckpt_every=1)
    J3, g3 = m.misfit_grad(sigma, dt, sites, obs, ckpt_every=3)
    J7, g7 = m.misfit_grad(sigma, dt, sites, obs, ckpt_every=7)
    assert J1 == J3 == J7
    assert np.array_equal(g1, g3) and np.array_equal(g1, g7)
    s1, _ = m.state()
    for a, b in zip(s0, s1):
        assert np.array_equal(a, b)


def setup_3d(lmax=10, nsteps=5, nsite=30, seed=5, toroidal=0):
    """A model whose Maxwell elements are all carried as 3-D, with a seeded
    lateral log-viscosity field; returns a factory so finite differences can
    rebuild the model with a perturbed field."""
    rng = np.random.default_rng(seed)

    def make(pert):
        p = vlib.default_params()
        p.lmax, p.nlat, p.nphi = lmax, lmax + 1, 2 * (lmax + 1)
        for i, c in enumerate([2, 4, 3, 3]):
            p.ne_layer[i] = c
        p.visc3d_tol = -1.0  # every Maxwell element 3-D
        p.toroidal = toroidal
        m = vlib.Model(p)
        m.enable_visc3d(pert)
        return m

    m0 = make(np.zeros((12, lmax + 1, 2 * (lmax + 1))))
    th = np.linspace(0.1, 3.0, lmax + 1)[:, None]
    ph = np.linspace(0, 2 * np.pi, 2 * (lmax + 1), endpoint=False)[None, :]
    base = 0.3 * np.sin(2 * th) * np.cos(2 * ph) + 0.1 * rng.standard_normal((lmax + 1, 2 * (lmax + 1)))
    pert = np.stack([base * (1 + 0.05 * e) for e in range(m0.ne)])
    sig = (rng.standard_normal((nsteps, m0.nlm)) + 1j * rng.standard_normal((nsteps, m0.nlm))) * 1e3
    sig[:, : lmax + 1] = sig[:, : lmax + 1].real
    sites = rng.choice(m0.ng, size=nsite, replace=False)
    obs = 0.01 * rng.standard_normal((nsteps, nsite))
    return make, pert, sig, sites, obs, 50.0 * synth.SEC_PER_YEAR, rng


@pytest.mark.parametrize("toroidal", [0, 1])
def test_adjoint_3d_log_viscosity_gradient_vs_central_differences(toroidal):
    """With toroidal = 1 the lateral viscosity also drives W: the reverse
    sweep runs the lambda 3, 4 advance, the W drift and the ten-product 3-D
    chain transposed."""
    make, pert, sig, sites, obs, dt, rng = setup_3d(toroidal=toroidal)
    m = make(pert)
    assert m.info().ne3d > 0
    if toroidal:
        assert m.state_tor() is not None
    J, gs, gp = m.misfit_grad(sig, dt, sites, obs, ckpt_every=2, want_pert=True)
    assert abs(J - m.misfit(sig, dt, sites, obs)) <= 1e-12 * J
    h = 1e-4
    for _ in range(20):  # 20 seeded random directions
        d = rng.standard_normal(pert.shape)
        fd = (make(pert + h * d).misfit(sig, dt, sites, obs) - make(pert - h * d).misfit(sig, dt, sites, obs)) / (2 * h)
        ad = np.sum(gp * d)
        assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)
    # the load gradient through the 3-D transposes
    for _ in range(20):
        d = rng.standard_normal(sig.shape) + 1j * rng.standard_normal(sig.shape)
        d[:, : m.p.lmax + 1] = d[:, : m.p.lmax + 1].real
        hs = 1e-3 * np.abs(sig).max() / np.abs(d).max()
        fd = (m.misfit(sig + hs * d, dt, sites, obs) - m.misfit(sig - hs * d, dt, sites, obs)) / (2 * hs)
        ad = np.sum(gs.real * d.real + gs.imag * d.imag)
        assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


@pytest.mark.parametrize("toroidal", [0, 1])
def test_adjoint_3d_checkpoint_interval_and_state_kept(toroidal):
    """The 3-D reverse sweep reads each step's longitude grid: kept from the
    forward sweep for the last segment, recomputed from a checkpoint for the
    others. Every interval gives the same gradients, bit for bit, and the
    handle's memory (the toroidal one too) is left as it was."""
    make, pert, sig, sites, obs, dt, rng = setup_3d(nsteps=5, toroidal=toroidal)
    m = make(pert)
    m.set_dt(dt)
    for _ in range(2):  # a state with memory in it, toroidal included
        m.begin_step()
        m.advance(sig[0])
    s0, _ = m.state()
    t0 = m.state_tor()
    out = [m.misfit_grad(sig, dt, sites, obs, ckpt_every=c, want_pert=True) for c in (1, 2, 5, 9)]
    J0, gs0, gp0 = out[0]
    for J, gs, gp in out[1:]:
        assert J == J0
        assert np.array_equal(gs, gs0) and np.array_equal(gp, gp0)
    s1, _ = m.state()
    for a, b in zip(s0, s1):
        assert np.array_equal(a, b)
    if toroidal:
        for a, b in zip(t0, m.state_tor()):
            assert np.array_equal(a, b)
