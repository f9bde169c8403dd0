"""The laterally-uniform viscosity sweep of the reference's 3-D response test
(tests/test_response_3d.f90:25-30, 63-81, 101-120, 218-250): a spatially
constant log10 perturbation p routed through the pseudo-spectral 3-D memory
advance must reproduce a 1-D run on an earth whose Maxwell viscosities are
scaled by 10^p, for p in PSWEEP (soft to the stiff M ~ 1e-11 regime the
increment form exists for), in the centre-of-figure and centre-of-mass
degree-1 frames. Shared by the oracle (CPU) and the device tests; `make`
builds a model from params for either side."""
import numpy as np

from fastearth3d_b200.abi import M3L70V01, VG_RHEOL_MAXWELL, set_layers

PSWEEP = (-0.4, 2.0, 4.0, 6.0, 8.0, 10.0)
LMAX = 8
NSTEP = 25
DT_S = 20.0 * 31556926.0  # 20 yr (the reference test's 0.02 kyr)
TOL = 1.0e-9


def lmidx(lmax, l, m):
    return m * (lmax + 1) - m * (m - 1) // 2 + (l - m)


def build_load(lmax=LMAX):
    """The test's deterministic non-axisymmetric load: every (l, m), l >= 1."""
    nlm = (lmax + 1) * (lmax + 2) // 2
    s = np.zeros(nlm, complex)
    for l in range(1, lmax + 1):
        for m in range(0, l + 1):
            if m == 0:
                s[lmidx(lmax, l, m)] = 1000.0 / (l * l)
            else:
                s[lmidx(lmax, l, m)] = 700.0 / (l * l) + 1j * 400.0 / (l * (m + 1))
    return s


def params(default_params, p_pert, deg1_cm, three_d, precision=0):
    """M3-L70-V01 on its native radial mesh, lmax 8 on a 24 x 24 Gauss grid
    (nlat = nphi = 3 lmax, as the test), 20-yr steps. The 1-D model carries
    eta * 10^p in its Maxwell layers; the 3-D one gets p as a lateral field."""
    p = default_params()
    p.lmax, p.nlat, p.nphi = LMAX, 3 * LMAX, 3 * LMAX
    layers = list(M3L70V01)
    if not three_d:
        layers = [(rb, rt, rho, mu, eta * 10.0 ** p_pert if rh == VG_RHEOL_MAXWELL else eta, rh)
                  for (rb, rt, rho, mu, eta, rh) in layers]
    set_layers(p, layers)
    for i in range(len(p.ne_layer)):
        p.ne_layer[i] = 0
    p.deg1_cm = 1 if deg1_cm else 0
    p.skip_tol = 0.0
    p.dt_init = DT_S
    p.visc3d_tol = -1.0  # every Maxwell element through the pseudo-spectral path
    p.visc3d_precision = precision
    return p


def sweep_errors(make, default_params, p_pert, deg1_cm, precision=0):
    """(relative memory error, relative uplift error) of the 3-D path against
    the 1-D run over NSTEP begin / apply / commit steps."""
    m3 = make(params(default_params, p_pert, deg1_cm, True, precision))
    m1 = make(params(default_params, p_pert, deg1_cm, False))
    pert = np.full((m3.ne, 3 * LMAX, 3 * LMAX), p_pert)
    m3.enable_visc3d(pert)
    assert m3.info().ne3d > 0 and m1.info().ne3d == 0
    slm = build_load()
    nk, ne = m3.nk, m3.ne
    dmem = smem = dupl = supl = 0.0
    for _ in range(NSTEP):
        m3.begin_step()
        u3, _n3 = m3.apply(slm)
        m1.begin_step()
        u1, _n1 = m1.apply(slm)
        dupl = max(dupl, float(np.abs(u3 - u1).max()))
        supl = max(supl, float(np.abs(u1).max()))
        m3.advance(slm)
        m1.advance(slm)
        s3, _ = m3.state()
        s1, _ = m1.state()
        for a, b in zip(s3, s1):
            da = (np.asarray(a) - np.asarray(b)).reshape(nk, ne, 4).copy()
            da[:2, :, 3] = 0.0  # lambda 6 at the degree-1 slots (orders 0, 1)
            dmem = max(dmem, float(np.abs(da).max()))
        for b in s1[0::2]:  # A, B, C real parts, as the test's scale
            smem = max(smem, float(np.abs(b).max()))
    return dmem / max(smem, 1e-300), dupl / max(supl, 1e-300)
