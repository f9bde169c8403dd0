"""The oracle's trapezoidal scheme (scheme = "trap") against the properties the
reference's own tests establish for it (the reference has no golden vectors
for this path; tests/test_sle_couple_order.f90 and tests/test_timestep.f90):

  * with the sea-level <-> memory coupling iterated to convergence, the
    trapezoidal rule is 2nd order in dt for the rsl field under a fast ice ramp
    with a fixed ocean; forward Euler is 1st order;
  * a single coupling pass (sle_max_mem_iter = 1) falls back to ~1st order;
  * the step-doubling controller: tightening rtol lowers the error monotonically.

A fixed step is taken by making every trial step pass the controller (rtol,
atol huge): each update interval is then one coarse step and two accepted half
steps. Earth: the 4-layer default, a few elements per layer; lmax 12.
"""
import numpy as np
import pytest

from fastearth3d_b200 import synth
from oracle import orc

T_RAMP = 800.0  # yr


def make(scheme, lmax=12, mem_iter=30, rtol=1e30, atol=1e30, dt_yr=100.0):
    p = orc.default_params()
    p.lmax, p.nlat, p.nphi = lmax, lmax + 1, 2 * (lmax + 1)
    for i, c in enumerate([2, 5, 4, 3]):
        p.ne_layer[i] = c
    p.scheme = scheme
    p.sle_fixed_ocean = 1
    p.rtol, p.atol = rtol, atol
    p.sle_max_mem_iter = mem_iter
    p.couple_tol = 1e-10
    p.sle_tol = 1e-12
    p.sle_n_inner = 60
    p.dt_init = dt_yr * synth.SEC_PER_YEAR
    o = orc.Oracle(p)
    nlat, nphi = lmax + 1, 2 * (lmax + 1)
    th = np.linspace(0.05, np.pi - 0.05, nlat)[:, None]
    ph = np.linspace(0, 2 * np.pi, nphi, endpoint=False)[None, :]
    bump = np.exp(-((th - 0.6) ** 2 + (ph - 1.0) ** 2) / 0.5)
    topo = -2000.0 + 3000.0 * bump
    cap = 2000.0 * np.exp(-((th - 0.6) ** 2 + (ph - 1.0) ** 2) / 0.1) * (topo > 0)
    o.set_reference(topo.reshape(-1), np.zeros(nlat * nphi))
    return o, cap.reshape(-1)


def ramp(o, cap, dt_yr):
    n = int(round(T_RAMP / dt_yr))
    for k in range(1, n + 1):
        o.update(cap * min(1.0, k * dt_yr / T_RAMP), dt_yr)
    return o.fields()[0]


def errors(scheme, **kw):
    o, cap = make(scheme, dt_yr=5.0, **kw)
    ref = ramp(o, cap, 5.0)
    out = []
    for dt in (80.0, 40.0, 20.0):
        o, cap = make(scheme, dt_yr=dt, **kw)
        out.append(np.abs(ramp(o, cap, dt) - ref).max())
    return np.array(out)


def orders(e):
    return np.log2(e[:-1] / e[1:])


def test_trap_second_order_with_converged_coupling():
    e = errors(2)
    assert np.all(orders(e) > 1.8), (e, orders(e))
    fe = errors(0)
    assert np.all((orders(fe) > 0.8) & (orders(fe) < 1.4)), (fe, orders(fe))
    assert e[-1] < 1e-2 * fe[-1]


def test_trap_single_coupling_pass_is_first_order():
    e = errors(2, mem_iter=1)
    assert np.all((orders(e) > 0.8) & (orders(e) < 1.3)), (e, orders(e))


def test_trap_controller_rtol_monotone():
    o, cap = make(2, dt_yr=5.0)
    ref = ramp(o, cap, 5.0)
    errs, steps = [], []
    for rtol in (1e-2, 1e-3, 1e-4):
        o, cap = make(2, rtol=rtol, atol=1e-3)
        errs.append(np.abs(ramp(o, cap, 200.0) - ref).max())
        steps.append(o.info().n_accept)
    assert errs[0] > errs[1] > errs[2], errs
    assert steps[0] < steps[1] < steps[2], steps
