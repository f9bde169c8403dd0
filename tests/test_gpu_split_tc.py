"""The split-precision tensor-core 3-D advance (visc3d_precision = SPLIT_TC)
against the plain FP64 GPU path on the same inputs.

The split path computes the four stress-product contractions with two-term
TF32 operands on tcgen05 tensor cores (FP32 accumulation), so its results are
held to stated tolerances, not to the FP64 path's 1e-10:
  * one 3-D memory advance: 1e-5 relative to the state's maximum;
  * six held-load advances (errors accumulate with the state): 1e-4;
  * laterally uniform perturbation through the split path vs the 1-D path
    (the FP64 analytic limit of tests/test_response_3d.f90): 1e-4.
Orders and sizes cover an odd lmax (no equatorial row, unequal even/odd order
counts) and lmax 160 (two N tiles in the longitude stages).
"""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import VG_VISC3D_FP64, VG_VISC3D_SPLIT_TC

pytestmark = pytest.mark.gpu


def model(lmax, ne_layer, prec, **kw):
    p = vlib.default_params()
    p.lmax, p.nlat, p.nphi = lmax, lmax + 1, 2 * (lmax + 1)
    for i, c in enumerate(ne_layer):
        p.ne_layer[i] = c
    for k, v in kw.items():
        setattr(p, k, v)
    p.visc3d_precision = prec
    return vlib.Model(p)


def lateral_pert(m, seed):
    rng = np.random.default_rng(seed)
    nlat, nphi = m.p.nlat, m.p.nphi
    th = np.linspace(0.1, 3.0, nlat)[:, None]
    ph = np.linspace(0, 2 * np.pi, nphi, endpoint=False)[None, :]
    f = 0.4 * np.sin(2 * th) * np.cos(3 * ph) + 0.3 * np.cos(th) * np.sin(ph)
    f = f + 0.1 * rng.standard_normal((nlat, nphi))
    return np.stack([f * (1.0 + 0.1 * e) for e in range(m.ne)])


def rand_sigma(rng, nlm, lmax, scale=1e4):
    s = (rng.standard_normal(nlm) + 1j * rng.standard_normal(nlm)) * scale
    s[: lmax + 1] = s[: lmax + 1].real
    return s


def state_err(a, b):
    sa, _ = a.state()
    sb, _ = b.state()
    mx = max(np.abs(x).max() for x in sb)
    return max(np.abs(x - y).max() for x, y in zip(sa, sb)) / mx


@pytest.mark.parametrize("lmax", [16, 33, 160])
def test_split_tc_advance_vs_fp64(lmax):
    kw = dict(skip_tol=0.0, dt_init=50 * synth.SEC_PER_YEAR)
    g64 = model(lmax, [2, 6, 5, 3], VG_VISC3D_FP64, **kw)
    gtc = model(lmax, [2, 6, 5, 3], VG_VISC3D_SPLIT_TC, **kw)
    pert = lateral_pert(g64, 21)
    g64.enable_visc3d(pert)
    gtc.enable_visc3d(pert)
    assert gtc.info().ne3d == g64.info().ne3d > 0
    sigma = rand_sigma(np.random.default_rng(8), g64.nlm, lmax)
    errs = []
    for _ in range(6):
        for m in (g64, gtc):
            m.begin_step()
            m.advance(sigma)
        errs.append(state_err(gtc, g64))
        ua, na = gtc.apply(sigma)
        ub, nb = g64.apply(sigma)
        assert np.isfinite(ua).all() and np.isfinite(na).all()
    assert errs[0] < 1e-5, errs
    assert max(errs) < 1e-4, errs


def test_split_tc_uniform_equals_1d():
    kw = dict(skip_tol=0.0, dt_init=50 * synth.SEC_PER_YEAR)
    g3 = model(24, [2, 5, 4, 3], VG_VISC3D_SPLIT_TC, visc3d_tol=-1.0, **kw)
    g1 = model(24, [2, 5, 4, 3], VG_VISC3D_FP64, visc3d_tol=10.0, **kw)
    pert = np.full((g3.ne, 25, 50), 0.3)
    g3.enable_visc3d(pert)
    g1.enable_visc3d(pert)
    assert g3.info().ne3d > 0 and g1.info().ne3d == 0
    sigma = rand_sigma(np.random.default_rng(11), g3.nlm, 24)
    for _ in range(5):
        for m in (g3, g1):
            m.begin_step()
            m.advance(sigma)
    assert state_err(g3, g1) < 1e-4


def test_split_tc_update_rsl_error():
    """Full solid_earth_update steps (sea level, sub-steps) at lmax 32 on the
    3-D workload's earth: the split path's rsl and z_bed against the FP64 GPU
    path. The stated tolerance of the split path on rsl is 1e-6 relative to
    max |rsl| over these steps."""
    w = synth.Workload("t", 32, 40, 50.0, 8, 3, "sawtooth", sle=True, visc3d=True, seed=5)
    ms = []
    for prec in (VG_VISC3D_FP64, VG_VISC3D_SPLIT_TC):
        p = w.params(vlib.default_params)
        p.visc3d_precision = prec
        m = vlib.Model(p)
        zb, hi = w.reference()
        m.set_reference(zb, hi)
        m.enable_visc3d(w.pert(m.p))
        ms.append(m)
    worst = 0.0
    for step in range(1, 9):
        ice = w.ice_at(step * 400)
        for m in ms:
            m.update(ice, w.dt_yr)
        (r0, z0, *_), (r1, z1, *_) = ms[0].fields(), ms[1].fields()
        worst = max(worst, np.abs(r1 - r0).max() / np.abs(r0).max())
        assert np.abs(z1 - z0).max() / np.abs(z0).max() < 1e-6
        assert ms[0].info().n_sub_last == ms[1].info().n_sub_last
    assert worst < 1e-6, worst
