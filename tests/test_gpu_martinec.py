"""The GPU time step against the Martinec et al. (2018) sea-level benchmark.

Cases C2, D3, E2 and F1 of the reference's benchmark data (SBK letter = the
paper's case letter + 1; tests/test_benchmark_sle.f90:1-38, 183-242), run
through vg_update on M3-L70-V01 at lmax 128 on the 256 x 512 Gauss grid,
20-yr steps:

* a sqrt ice cap (alpha = 10 deg) at colatitude 25, longitude 75: 1500 m held
  from the first step (C2: Heaviside, 500 steps), or 500 m grown linearly over
  10 kyr and held 5 kyr (D3, E2, F1: 750 steps);
* an exponential basin bmax - b0 exp(-psi^2 / 2 sigma^2), sigma = 26 deg, as the
  reference topography (C2: 760 / 1200 m at colatitude 100, longitude 320;
  the others 3800 / 6000 m at colatitude 35, longitude 25);
* a fixed ocean geometry (C2, D3) or a migrating coastline (E2, F1), the
  subgrid coast, warm-started fixed point with 20 inner iterations;
* F1 iterates the reference topography so the deformed present-day surface
  lands on the basin: topo0 <- topo0 - (topo0 - rsl - basin) / 2 until the
  mean misfit is below 1 m (at most 12 passes; :127-146).

The final state is read along the four profiles of each case (circles of
constant longitude or colatitude, :305-336): vertical displacement u and geoid
N from the converged load through vg_response_apply (the last step's frozen
drift, as the reference's resp%horizontal reuses it), the horizontal
displacement from V = gv sigma + dV, the sea surface N + esl and the sea level
rsl. The reference bounds the peak-normalised maximum errors by u 30 %,
horizontal 35 % of the peak vector, N 12 %, sea surface 8 % and sea level
12 % (:59-67); this test holds the tighter bounds this implementation
reaches with margin (u 8 %, horizontal 3 %, N 10 %, sea surface 1.5 %, sea
level 2.5 %). The spectral point evaluator used for the profiles is checked
against the library's own synthesis at grid nodes first, and the first steps
of case E2 (growing ice, migrating coast) against the oracle."""
import os

import numpy as np
import pytest

from fastearth3d_b200 import lib as vlib
from fastearth3d_b200 import synth
from fastearth3d_b200.abi import M3L70V01, set_layers

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
L, NLAT, NPHI = 128, 256, 512
DEG = np.pi / 180.0
NGROW, NHOLD = 500, 250
G_REF = 9.815  # the benchmark's reference gravity (col5 = -N g)
TOL = {"u": 0.08, "h": 0.03, "N": 0.10, "ss": 0.015, "sle": 0.025}

# case: (h0, basin colat, basin lon, bmax, b0, fixed ocean, Heaviside, spin-up, profile fixes)
CASES = {
    "C2": (1500.0, 100.0, 320.0, 760.0, 1200.0, True, True, False, (75.0, 25.0, -40.0, 100.0)),
    "D3": (500.0, 35.0, 25.0, 3800.0, 6000.0, True, False, False, (75.0, 25.0, 25.0, 35.0)),
    "E2": (500.0, 35.0, 25.0, 3800.0, 6000.0, False, False, False, (75.0, 25.0, 25.0, 35.0)),
    "F1": (500.0, 35.0, 25.0, 3800.0, 6000.0, False, False, True, (75.0, 25.0, 25.0, 35.0)),
}
PTYPE = ("Z", "Y", "Z", "Y")  # Z: fixed longitude, col1 = colatitude; Y: fixed colatitude, col1 = longitude


def gauss_grid():
    x, w = np.polynomial.legendre.leggauss(NLAT)
    order = np.argsort(-x)  # north first
    return np.arccos(x[order]), w[order], 2.0 * np.pi * np.arange(NPHI) / NPHI


def distance(colat, lon, c0, l0):
    """Great-circle distance between the grid (colat[:, None], lon[None, :]) and a point."""
    cd = np.cos(colat)[:, None] * np.cos(c0) + np.sin(colat)[:, None] * np.sin(c0) * np.cos(lon[None, :] - l0)
    return np.arccos(np.clip(cd, -1.0, 1.0))


def lm_index(l, m):
    return m * (L + 1) - m * (m - 1) // 2 + (l - m)


def plm(theta):
    """Orthonormal associated Legendre functions without the Condon-Shortley
    phase, P[lm, point] (m-major lm order), and their theta derivatives."""
    x, s = np.cos(theta), np.sin(theta)
    nlm = (L + 1) * (L + 2) // 2
    P = np.zeros((nlm, len(theta)))
    D = np.zeros_like(P)
    pmm = np.full(len(theta), 1.0 / np.sqrt(4.0 * np.pi))
    for m in range(L + 1):
        if m > 0:
            pmm = pmm * np.sqrt((2 * m + 1) / (2.0 * m)) * s
        prev2, prev = np.zeros_like(x), pmm
        P[lm_index(m, m)] = pmm
        for l in range(m + 1, L + 1):
            if l == m + 1:
                cur = np.sqrt(2.0 * m + 3.0) * x * prev
            else:
                a = np.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
                b = np.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
                cur = a * (x * prev - b * prev2)
            P[lm_index(l, m)] = cur
            prev2, prev = prev, cur
        for l in range(m, L + 1):
            below = P[lm_index(l - 1, m)] if l > m else 0.0
            c = np.sqrt((2.0 * l + 1.0) / (2.0 * l - 1.0) * (l * l - m * m)) if l > m else 0.0
            D[lm_index(l, m)] = (l * x * P[lm_index(l, m)] - c * below) / s
    return P, D


def mvec():
    return np.concatenate([np.full(L + 1 - m, m) for m in range(L + 1)])


def evaluate(q, theta, lon, horizontal=False):
    """f = sum_l q_l0 Y_l0 + 2 Re sum_{m>0} q_lm Y_lm at the points; with
    horizontal, the gradient components (d/dtheta, 1/sin(theta) d/dlon)."""
    P, D = plm(theta)
    m = mvec()[:, None]
    wgt = np.where(m == 0, 1.0, 2.0)
    e = np.exp(1j * m * lon[None, :])
    qe = wgt * q[:, None] * e
    if not horizontal:
        return (qe * P).real.sum(0)
    vth = (qe * D).real.sum(0)
    vph = (1j * m * qe * P).real.sum(0) / np.sin(theta)
    return vth, vph


def profile_points(k, c1, pfix):
    if PTYPE[k] == "Z":
        th, lo = c1 * DEG, np.full_like(c1, pfix[k] * DEG)
    else:
        th, lo = np.full_like(c1, pfix[k] * DEG), c1 * DEG
    # the pole rows of the colatitude profiles: evaluate a hair inside the sphere's axis
    return np.clip(th, 1e-7, np.pi - 1e-7), lo


def make_model(topo0, fixed_ocean, mk=vlib.default_params, cls=vlib.Model, scheme=0):
    p = mk()
    p.scheme = scheme  # 0: forward Euler ("fe"), 2: trapezoidal ("trap")
    set_layers(p, M3L70V01)
    p.lmax, p.nlat, p.nphi = L, NLAT, NPHI
    p.dt_init = 20.0 * synth.SEC_PER_YEAR
    p.sle_n_inner = 20
    p.sle_fixed_ocean = int(fixed_ocean)
    p.sle_subgrid = 1
    p.sle_warm_start = 1
    m = cls(p)
    m.set_reference(topo0, np.zeros_like(topo0))
    return m


def run_history(topo0, case, scheme=0):
    h0, _, _, _, _, fixed, heaviside, _, _ = CASES[case]
    colat, w, lon = gauss_grid()
    cd = np.cos(distance(colat, lon, 25.0 * DEG, 75.0 * DEG))
    m = make_model(topo0, fixed, scheme=scheme)
    nsteps = NGROW if heaviside else NGROW + NHOLD
    ice = np.zeros((NLAT, NPHI))
    for istep in range(1, nsteps + 1):
        frac = 1.0 if heaviside else min(1.0, istep / NGROW)
        ca = np.cos(frac * 10.0 * DEG)
        ice = np.where(cd >= ca, frac * h0 * np.sqrt(np.maximum((cd - ca) / (1.0 - ca), 0.0)), 0.0)
        m.update(ice, 20.0)
        if scheme == 0:
            assert m.info().n_sub_last == 1  # one 20-yr response step per interval, as the reference
    return m, ice


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLD, "martinec2018.npz"))


def test_point_evaluator_matches_library_synthesis():
    colat, _, lon = gauss_grid()
    m = make_model(np.full((NLAT, NPHI), 1000.0), False)
    rng = np.random.default_rng(5)
    q = (rng.standard_normal(m.nlm) + 1j * rng.standard_normal(m.nlm)) / (1.0 + mvec())
    q[mvec() == 0] = q[mvec() == 0].real
    f = m.synthesis(q).reshape(NLAT, NPHI)
    rows, cols = np.array([0, 40, 127, 128, 200, 255]), np.array([0, 77, 256, 300, 411, 511])
    got = evaluate(q, colat[rows], lon[cols])
    assert np.abs(got - f[rows, cols]).max() <= 1e-10 * np.abs(f).max()
    # the gradient against a centred difference of the same series
    th, lo, eps = colat[rows], lon[cols], 1e-6
    vth, vph = evaluate(q, th, lo, horizontal=True)
    dth = (evaluate(q, th + eps, lo) - evaluate(q, th - eps, lo)) / (2 * eps)
    dph = (evaluate(q, th, lo + eps) - evaluate(q, th, lo - eps)) / (2 * eps) / np.sin(th)
    assert np.abs(vth - dth).max() <= 1e-5 * np.abs(vth).max()
    assert np.abs(vph - dph).max() <= 1e-5 * np.abs(vph).max()


@pytest.mark.parametrize("case,scheme", [("C2", 0), ("D3", 0), ("E2", 0), ("F1", 0), ("E2", 2)])
def test_martinec2018_sea_level_case(case, scheme, golden):
    """scheme 2: the trapezoidal scheme with its step-doubling controller
    (adaptive sub-steps within each 20-yr interval) on the same case."""
    h0, bcol, blon, bmax, b0, fixed, heaviside, spin, pfix = CASES[case]
    colat, w, lon = gauss_grid()
    psi = distance(colat, lon, bcol * DEG, blon * DEG)
    basin = bmax - b0 * np.exp(-psi * psi / (2.0 * (26.0 * DEG) ** 2))
    area = (2.0 * np.pi / NPHI) * w[:, None] * np.ones(NPHI)
    topo0 = basin.copy()
    for _ in range(12 if spin else 1):
        m, ice = run_history(topo0, case, scheme)
        rsl, _, C_oc, sigma = m.fields()
        rsl = rsl.reshape(NLAT, NPHI)
        if not spin:
            break
        dtopo = (topo0 - rsl) - basin
        misfit = (area * np.abs(dtopo)).sum() / (4.0 * np.pi)
        if misfit < 1.0:
            break
        topo0 = topo0 - 0.5 * dtopo
    if spin:
        assert misfit < 1.0
    C_oc = C_oc.reshape(NLAT, NPHI)
    assert C_oc.min() >= 0.0 and C_oc.max() <= 1.0 and C_oc.max() > 0.0

    # the final state's fields, spectrally
    u_lm, N_lm = m.apply(sigma)
    gu, gn, gv = m.gains()
    dV = m.drift()[2]
    V_lm = np.zeros(m.nlm, complex)
    k = 0
    for l in range(1, L + 1):
        for mm in range(l + 1):
            V_lm[lm_index(l, mm)] = gv[l] * sigma[lm_index(l, mm)] + dV[k]
            k += 1
    rsl_lm = m.analysis(rsl.reshape(-1))
    N_grid = m.synthesis(N_lm).reshape(NLAT, NPHI)
    u_grid = m.synthesis(u_lm).reshape(NLAT, NPHI)
    # the sea-level equation's decomposition rsl = N - u + esl holds on the whole
    # grid (trapezoidal: up to the sea-level <-> memory co-convergence tolerance,
    # the stored drift being the last endpoint pass's)
    shift = rsl - (N_grid - u_grid)
    esl = float((area * shift).sum() / (4.0 * np.pi))
    tol_dec = 1e-6 if scheme == 0 else 1e-3
    assert np.abs(shift - esl).max() <= tol_dec * np.abs(rsl).max(), np.abs(shift - esl).max()

    errs = {}
    for k in range(4):
        ref = golden[f"{case}_fig{10 + k}"].astype(np.float64)
        th, lo = profile_points(k, ref[:, 0], pfix)
        um = evaluate(u_lm, th, lo)
        nm = evaluate(N_lm, th, lo)
        sle = evaluate(rsl_lm, th, lo)
        vth, vph = evaluate(V_lm, th, lo, horizontal=True)
        ss = nm + esl
        nref = -ref[:, 4] / G_REF
        hpk = np.sqrt(ref[:, 2] ** 2 + ref[:, 3] ** 2).max()
        e = {
            "u": np.abs(um - ref[:, 1]).max() / np.abs(ref[:, 1]).max(),
            "h": max(np.abs(vth - ref[:, 2]).max(), np.abs(vph - ref[:, 3]).max()) / hpk,
            "N": np.abs(nm - nref).max() / np.abs(nref).max(),
            "ss": np.abs(ss - ref[:, 5]).max() / np.abs(ref[:, 5]).max(),
            "sle": np.abs(sle - ref[:, 6]).max() / np.abs(ref[:, 6]).max(),
        }
        errs[f"fig{10 + k}"] = e
    print(case, "scheme", scheme, "esl", esl, {f: {c: round(100 * v, 2) for c, v in e.items()} for f, e in errs.items()})
    for f, e in errs.items():
        for c, v in e.items():
            assert v <= TOL[c], (case, f, c, v)


def test_martinec2018_e2_first_steps_match_oracle():
    """Case E2's first 12 steps (the cap growing over the near basin, the coast
    migrating): rsl, ocean function and load equal the oracle's to 1e-10."""
    from oracle import orc

    _, bcol, blon, bmax, b0, fixed, _, _, _ = CASES["E2"]
    colat, _, lon = gauss_grid()
    psi = distance(colat, lon, bcol * DEG, blon * DEG)
    basin = np.ascontiguousarray(bmax - b0 * np.exp(-psi * psi / (2.0 * (26.0 * DEG) ** 2)))
    cd = np.cos(distance(colat, lon, 25.0 * DEG, 75.0 * DEG))
    g = make_model(basin, fixed)
    o = make_model(basin, fixed, orc.default_params, orc.Oracle)
    C_first = None
    for istep in range(1, 13):
        frac = istep / 12.0  # a faster ramp than the benchmark's, to move the coast within the window
        ca = np.cos(frac * 10.0 * DEG)
        ice = np.where(cd >= ca, frac * 500.0 * np.sqrt(np.maximum((cd - ca) / (1.0 - ca), 0.0)), 0.0)
        g.update(ice, 20.0)
        o.update(np.ascontiguousarray(ice), 20.0)
        if C_first is None:
            C_first = g.fields()[2]
    fg, fo = g.fields(), o.fields()
    for a, b in ((fg[0], fo[0]), (fg[2], fo[2]), (fg[3], fo[3])):
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1.0)
    assert np.abs(fg[2] - C_first).max() > 0.0  # the coast moved
