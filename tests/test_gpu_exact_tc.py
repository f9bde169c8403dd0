"""The exact-product tensor-core 3-D advance (visc3d_precision = EXACT_TC)
against the plain FP64 GPU path and the reference's analytic limit.

EXACT_TC runs the four stress-product contractions on tcgen05 tensor cores
with 8-bit digit slices of 40-bit fixed-point operands and exact int32
accumulation (five digit levels), FP64 between the stages. Stated
tolerances:
  * one 3-D memory advance and six held-load advances with a white load
    spectrum: 1e-8 relative to the state's maximum and to the surface
    displacement's at lmax 16 and 33, 2e-8 at lmax 160 (the state,
    internal, amplifies last-bit differences as on the FP64 path; measured
    2e-10 ... 5e-9 at lmax 16 and 33, up to 1.2e-8 at lmax 160);
  * the reference's uniform-viscosity sweep (tests/test_response_3d.f90:
    25-30, 218-250), p from -0.4 to 10, both degree-1 frames: 1e-9, the
    reference's own tolerance;
  * full updates (sea level, sub-steps) at lmax 32: rsl and z_bed 1e-9;
  * the lmax-128 3-D workload of the benchmark, 30 intervals: rsl within
    1e-8 of the FP64 path (relative to max |rsl|), z_bed 1e-10, identical
    sub-step counts.
Orders and sizes cover an odd lmax (no equatorial row, unequal even/odd order
counts) and lmax 160 (three N tiles in the longitude stages).
"""
import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import VG_VISC3D_EXACT_TC, VG_VISC3D_FP64
from sweep_util import PSWEEP, TOL as SWEEP_TOL, sweep_errors

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


# Response spectra after each advance, relative to their largest entry. The
# fixed point keeps 38 bits below each row group's largest value, so the error
# of a K-term product grows with the number of latitudes and orders summed: a
# white load spectrum at lmax 160 reaches 1.1e-8 (the 1e-8 rsl bound of the
# lmax-128 configuration is asserted over 30 intervals in the full-size test).
# The memory state, read back after each advance, carries the same error
# (1.2e-8 after the first advance at lmax 160).
APPLY_TOL = {16: 1e-8, 33: 1e-8, 160: 2e-8}
STATE_TOL = APPLY_TOL


@pytest.mark.parametrize("lmax", [16, 33, 160])
def test_exact_tc_advance_vs_fp64(lmax):
    kw = dict(skip_tol=0.0, dt_init=50 * synth.SEC_PER_YEAR)
    g64 = model(lmax, [2, 6, 5, 3], VG_VISC3D_FP64, **kw)
    gtc = model(lmax, [2, 6, 5, 3], VG_VISC3D_EXACT_TC, **kw)
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
        assert np.abs(ua - ub).max() <= APPLY_TOL[lmax] * np.abs(ub).max()
    print("exact_tc state error per advance:", ["%.2e" % e for e in errs])
    assert max(errs) < STATE_TOL[lmax], errs


@pytest.mark.parametrize("deg1_cm", [False, True])
@pytest.mark.parametrize("p_pert", PSWEEP)
def test_exact_tc_uniform_sweep(p_pert, deg1_cm):
    emem, eupl = sweep_errors(vlib.Model, vlib.default_params, p_pert, deg1_cm, precision=VG_VISC3D_EXACT_TC)
    assert emem <= SWEEP_TOL and eupl <= SWEEP_TOL, (emem, eupl)


def run_pair(w, steps):
    ms = []
    for prec in (VG_VISC3D_FP64, VG_VISC3D_EXACT_TC):
        p = w.params(vlib.default_params)
        p.visc3d_precision = prec
        m = vlib.Model(p)
        zb, hi = w.reference()
        m.set_reference(zb, hi)
        m.enable_visc3d(w.pert(m.p))
        ms.append(m)
    worst_r = worst_z = 0.0
    for step in steps:
        ice = w.ice_at(step)
        for m in ms:
            m.update(ice, w.dt_yr)
        (r0, z0, *_), (r1, z1, *_) = ms[0].fields(), ms[1].fields()
        worst_r = max(worst_r, np.abs(r1 - r0).max() / np.abs(r0).max())
        worst_z = max(worst_z, np.abs(z1 - z0).max() / np.abs(z0).max())
        assert ms[0].info().n_sub_last == ms[1].info().n_sub_last
    return worst_r, worst_z


def test_exact_tc_update_rsl_error():
    w = synth.Workload("t", 32, 40, 50.0, 8, 3, "sawtooth", sle=True, visc3d=True, seed=5)
    wr, wz = run_pair(w, [s * 400 for s in range(1, 9)])
    assert wr < 1e-9 and wz < 1e-9, (wr, wz)


def test_exact_tc_full_size_rsl_within_1e8():
    w = synth.workloads()["c3_3d_l128"]
    wr, wz = run_pair(w, range(400, 430))
    print("lmax-128 3-D workload, 30 intervals: rsl %.3e, z_bed %.3e" % (wr, wz))
    assert wr <= 1e-8 and wz <= 1e-10, (wr, wz)
