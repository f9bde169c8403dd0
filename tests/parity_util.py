"""Shared comparison of a device model with the oracle after the same calls.

Tolerance: 1e-10 relative to the field's maximum for outputs of the FP64
path; the Maxwell memory (internal state) to 1e-8, because its strain is a
difference of neighbouring nodal displacements that amplifies last-ulp
differences (FMA contraction, summation order) by about r/h ~ 600. Discrete
decisions (ocean function, accepted / rejected sub-steps, sub-step count)
must agree exactly."""
import numpy as np

TOL = 1e-10
TOL_STATE = 1e-8


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    d = np.abs(a - b).max()
    s = np.abs(b).max()
    return d / s if s > 0 else d


def check_models(g, o, tol=TOL, tol_state=TOL_STATE):
    rg, zg, cg, sg = g.fields()
    ro, zo, co, so = o.fields()
    assert np.array_equal(cg, co), "ocean function differs"
    assert rel(rg, ro) < tol, ("rsl", rel(rg, ro))
    assert rel(zg, zo) < tol, ("z_bed", rel(zg, zo))
    assert rel(sg, so) < tol, ("sigma", rel(sg, so))
    stg, _ = g.state()
    sto, _ = o.state()
    for a, b in zip(stg, sto):
        assert rel(a, b) < tol_state, ("state", rel(a, b))
    ig, io = g.info(), o.info()
    assert (ig.n_accept, ig.n_reject, ig.n_sub_last) == (io.n_accept, io.n_reject, io.n_sub_last)
    assert abs(ig.bsl - io.bsl) <= 1e-10 * max(1.0, abs(io.bsl))
    return {"rsl": rel(rg, ro), "z_bed": rel(zg, zo), "sigma": rel(sg, so)}
