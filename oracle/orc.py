"""ctypes binding of the CPU oracle (liboracle.so) — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this;
the product library never does. The C API mirrors include/vilma_gpu.h with an
`orc_` prefix, so both sides are driven by the same calls.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from fastearth3d_b200.abi import VgInfo, VgParams

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_P = C.POINTER(C.c_double)
_VP = C.c_void_p


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        for name, args in [
            ("orc_params_default", [C.POINTER(VgParams)]),
            ("orc_create", [C.POINTER(VgParams), C.POINTER(_VP)]),
            ("orc_destroy", [_VP]),
            ("orc_set_threads", [C.c_int]),
            ("orc_set_reference", [_VP, _P, _P, _P]),
            ("orc_enable_visc3d", [_VP, _P]),
            ("orc_advance", [_VP, _P, _P, C.c_double, C.c_double, _P, _P, _P, _P]),
            ("orc_enable_visc3d_from_nodes", [_VP, _P, C.c_double, C.c_double, C.c_double]),
            ("orc_update", [_VP, _P, C.c_double]),
            ("orc_spinup", [_VP, _P, C.c_double, C.c_double, C.c_int, _P, C.POINTER(C.c_int), C.POINTER(C.c_int),
                            C.POINTER(C.c_int)]),
            ("orc_get_fields", [_VP, _P, _P, _P, _P]),
            ("orc_get_rotation", [_VP, _P, _P]),
            ("orc_rotation_update", [_VP, _P, C.c_double]),
            ("orc_rotation_inertia", [_VP, _P, _P]),
            ("orc_get_info", [_VP, C.POINTER(VgInfo)]),
            ("orc_response_set_dt", [_VP, C.c_double]),
            ("orc_response_begin_step", [_VP]),
            ("orc_response_apply", [_VP, _P, _P, _P]),
            ("orc_response_advance", [_VP, _P]),
            ("orc_get_gains", [_VP, _P, _P, _P]),
            ("orc_get_drift", [_VP, _P, _P, _P]),
            ("orc_get_state", [_VP, _P, _P, _P, _P, _P, _P, _P]),
            ("orc_set_state", [_VP, _P, _P, _P, _P, _P, _P, C.c_double]),
            ("orc_sht_analysis", [_VP, _P, _P]),
            ("orc_sht_synthesis", [_VP, _P, _P]),
            ("orc_love_numbers", [C.POINTER(VgParams), C.c_int, C.c_int, _P, _P, _P]),
            ("orc_band_dense_solve", [C.c_int, _P, _P, _P]),
            ("orc_dense_operator", [C.POINTER(VgParams), C.c_int, C.c_int, _P, C.POINTER(C.c_int)]),
            ("orc_tensor_synth", [_VP, _P, _P, C.c_int]),
            ("orc_tensor_analysis", [_VP, _P, _P, C.c_int]),
            ("orc_get_toroidal", [_VP, _P]),
            ("orc_get_state_tor", [_VP, _P, _P, _P, _P, _P, _P, C.POINTER(C.c_int)]),
            ("orc_toroidal_operator", [C.POINTER(VgParams), C.c_int, _P, C.POINTER(C.c_int)]),
            ("orc_grid", [_VP, _P, _P]),
            ("orc_mesh", [_VP, _P, C.POINTER(C.c_int)]),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.orc_last_error.argtypes = [_VP]
        L.orc_last_error.restype = C.c_char_p
        L.orc_surface_integral.argtypes = [_VP, _P]
        L.orc_surface_integral.restype = C.c_double
        _lib = L
    return _lib


def ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_P)


def set_threads(n):
    """OpenMP threads of the oracle's parallel loops."""
    _check(lib().orc_set_threads(int(n)))


def default_params():
    p = VgParams()
    lib().orc_params_default(C.byref(p))
    return p


def _check(rc, h=None):
    if rc != 0:
        raise RuntimeError(lib().orc_last_error(h).decode())


def love_numbers(p, jmin, jmax):
    n = jmax - jmin + 1
    h, l, k = np.zeros(n), np.zeros(n), np.zeros(n)
    _check(lib().orc_love_numbers(C.byref(p), jmin, jmax, ptr(h), ptr(l), ptr(k)))
    return h, l, k


def band_dense_solve(A, b):
    A = np.asfortranarray(A, dtype=np.float64)
    n = A.shape[0]
    flat = np.ascontiguousarray(A.T.reshape(-1))  # column-major flattening
    x = np.zeros(n)
    _check(lib().orc_band_dense_solve(n, ptr(flat), ptr(np.ascontiguousarray(b, dtype=np.float64)), ptr(x)))
    return x


def toroidal_operator(p, j):
    """Dense toroidal W operator of degree j (nr x nr), nothing pinned."""
    nr = C.c_int(0)
    _check(lib().orc_toroidal_operator(C.byref(p), j, None, C.byref(nr)))
    A = np.zeros(nr.value * nr.value)
    _check(lib().orc_toroidal_operator(C.byref(p), j, ptr(A), C.byref(nr)))
    return A.reshape(nr.value, nr.value).T.copy()


def dense_operator(p, j, with_uniq=True):
    nd = C.c_int(0)
    lib().orc_dense_operator(C.byref(p), j, int(with_uniq), None, C.byref(nd))
    flat = np.zeros(nd.value * nd.value)
    lib().orc_dense_operator(C.byref(p), j, int(with_uniq), ptr(flat), C.byref(nd))
    return flat.reshape(nd.value, nd.value).T  # column-major -> A[i, k]


class Oracle:
    """One oracle model instance (solid_earth_init/update restated on the CPU)."""

    def __init__(self, p):
        self.p = p
        h = _VP()
        _check(lib().orc_create(C.byref(p), C.byref(h)))
        self.h = h
        info = self.info()
        self.nlm, self.nk, self.ne, self.nr = info.nlm, info.nk, info.ne, info.nr
        self.ng = p.nphi * p.nlat

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def _c(self, rc):
        _check(rc, self.h)

    def info(self):
        i = VgInfo()
        self._c(lib().orc_get_info(self.h, C.byref(i)))
        return i

    def set_reference(self, z_bed_eq, h_ice_eq, h_ice_init=None):
        self._c(lib().orc_set_reference(self.h, ptr(z_bed_eq), ptr(h_ice_eq), ptr(h_ice_init)))

    def enable_visc3d(self, pert):
        self._c(lib().orc_enable_visc3d(self.h, ptr(np.ascontiguousarray(pert, dtype=np.float64))))

    def advance_interval(self, ice0, ice1, t0_yr, t1_yr, s_rot=None):
        """stepper_advance driven directly: (rsl, C, sigma_lm) at t1."""
        rsl, Cf, sig = np.zeros(self.ng), np.zeros(self.ng), np.zeros(2 * self.nlm)
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (ice0, ice1)]
        sr = None if s_rot is None else np.ascontiguousarray(s_rot, dtype=np.float64)
        self._c(lib().orc_advance(self.h, ptr(a[0]), ptr(a[1]), t0_yr, t1_yr, ptr(sr), ptr(rsl), ptr(Cf), ptr(sig)))
        return rsl, Cf, sig[0::2] + 1j * sig[1::2]

    def enable_visc3d_from_nodes(self, visc_node, lid_depth=0.0, lid_log10max=0.0, log10_cap=0.0):
        v = np.ascontiguousarray(visc_node, dtype=np.float64)
        self._c(lib().orc_enable_visc3d_from_nodes(self.h, ptr(v), lid_depth, lid_log10max, log10_cap))

    def update(self, h_ice, dt_yr):
        self._c(lib().orc_update(self.h, ptr(np.ascontiguousarray(h_ice, dtype=np.float64)), dt_yr))

    def spinup(self, h_ice_lgm, t_max_yr, rate_tol, pre_1d=False, with_1d=False):
        t = C.c_double(0.0)
        n, ok, n1 = C.c_int(0), C.c_int(0), C.c_int(0)
        ice = np.ascontiguousarray(h_ice_lgm, dtype=np.float64)
        self._c(lib().orc_spinup(self.h, ptr(ice), t_max_yr, rate_tol, 1 if pre_1d else 0, C.byref(t), C.byref(n),
                                 C.byref(ok), C.byref(n1)))
        out = (t.value, n.value, bool(ok.value))
        return out + (n1.value,) if with_1d else out

    def fields(self):
        rsl, zb, Cf = np.zeros(self.ng), np.zeros(self.ng), np.zeros(self.ng)
        sig = np.zeros(2 * self.nlm)
        self._c(lib().orc_get_fields(self.h, ptr(rsl), ptr(zb), ptr(Cf), ptr(sig)))
        return rsl, zb, Cf, sig[0::2] + 1j * sig[1::2]

    def rotation(self):
        """Polar motion m (complex) and (kTe, hTe, k_s fluid, k_s flattening)."""
        m, love = np.zeros(2), np.zeros(4)
        self._c(lib().orc_get_rotation(self.h, ptr(m), ptr(love)))
        return m[0] + 1j * m[1], love

    def rotation_update(self, load, dt_s):
        self._c(lib().orc_rotation_update(self.h, ptr(np.ascontiguousarray(load, dtype=np.float64)), dt_s))

    def rotation_inertia(self, load):
        out = np.zeros(2)
        self._c(lib().orc_rotation_inertia(self.h, ptr(np.ascontiguousarray(load, dtype=np.float64)), ptr(out)))
        return out[0] + 1j * out[1]

    def state(self):
        n = 4 * self.ne * self.nk
        arrs = [np.zeros(n) for _ in range(6)]
        t = C.c_double(0)
        self._c(lib().orc_get_state(self.h, *[ptr(a) for a in arrs], C.byref(t)))
        return arrs, t.value

    def set_state(self, arrs, t):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
        self._c(lib().orc_set_state(self.h, *[ptr(a) for a in arrs], t))

    def set_dt(self, dt_s):
        self._c(lib().orc_response_set_dt(self.h, dt_s))

    def begin_step(self):
        self._c(lib().orc_response_begin_step(self.h))

    def apply(self, sigma):
        s = np.zeros(2 * self.nlm)
        s[0::2], s[1::2] = sigma.real, sigma.imag
        u, n = np.zeros(2 * self.nlm), np.zeros(2 * self.nlm)
        self._c(lib().orc_response_apply(self.h, ptr(s), ptr(u), ptr(n)))
        return u[0::2] + 1j * u[1::2], n[0::2] + 1j * n[1::2]

    def advance(self, sigma):
        s = np.zeros(2 * self.nlm)
        s[0::2], s[1::2] = sigma.real, sigma.imag
        self._c(lib().orc_response_advance(self.h, ptr(s)))

    def gains(self):
        L = self.p.lmax + 1
        gu, gn, gv = np.zeros(L), np.zeros(L), np.zeros(L)
        self._c(lib().orc_get_gains(self.h, ptr(gu), ptr(gn), ptr(gv)))
        return gu, gn, gv

    def drift(self):
        a = [np.zeros(2 * self.nk) for _ in range(3)]
        self._c(lib().orc_get_drift(self.h, *[ptr(x) for x in a]))
        return [x[0::2] + 1j * x[1::2] for x in a]

    def analysis(self, f):
        q = np.zeros(2 * self.nlm)
        self._c(lib().orc_sht_analysis(self.h, ptr(np.ascontiguousarray(f, dtype=np.float64)), ptr(q)))
        return q[0::2] + 1j * q[1::2]

    def synthesis(self, q):
        s = np.zeros(2 * self.nlm)
        s[0::2], s[1::2] = q.real, q.imag
        f = np.zeros(self.ng)
        self._c(lib().orc_sht_synthesis(self.h, ptr(s), ptr(f)))
        return f

    def tensor_synth(self, c):
        """c: (4 or 6, nlm) complex -> dyad (6, ng) (rr, rt, rp, tt, tp, pp)"""
        nch = c.shape[0]
        s = np.zeros(2 * nch * self.nlm)
        cf = np.ascontiguousarray(c).reshape(-1)
        s[0::2], s[1::2] = cf.real, cf.imag
        d = np.zeros(6 * self.ng)
        self._c(lib().orc_tensor_synth(self.h, ptr(s), ptr(d), nch))
        return d.reshape(6, self.ng)

    def tensor_analysis(self, dyad, nch=4):
        c = np.zeros(2 * nch * self.nlm)
        d = np.ascontiguousarray(dyad, dtype=np.float64).reshape(-1)
        self._c(lib().orc_tensor_analysis(self.h, ptr(d), ptr(c), nch))
        return (c[0::2] + 1j * c[1::2]).reshape(nch, self.nlm)

    def toroidal(self):
        """Surface toroidal drift W(a) as t_lm (lm order); zero while not carried."""
        t = np.zeros(2 * self.nlm)
        self._c(lib().orc_get_toroidal(self.h, ptr(t)))
        return t[0::2] + 1j * t[1::2]

    def state_tor(self):
        """Toroidal memory (NLAM_TOR, ne, nk) x 6, or None while not carried."""
        n = 2 * self.ne * self.nk
        arrs = [np.zeros(n) for _ in range(6)]
        c = C.c_int(0)
        self._c(lib().orc_get_state_tor(self.h, *[ptr(a) for a in arrs], C.byref(c)))
        return arrs if c.value else None

    def grid(self):
        colat, w = np.zeros(self.p.nlat), np.zeros(self.p.nlat)
        self._c(lib().orc_grid(self.h, ptr(colat), ptr(w)))
        return colat, w

    def surface_integral(self, f):
        return lib().orc_surface_integral(self.h, ptr(np.ascontiguousarray(f, dtype=np.float64)))

    def mesh(self):
        r = np.zeros(self.nr)
        lay = (C.c_int * self.ne)()
        self._c(lib().orc_mesh(self.h, ptr(r), lay))
        return r, np.array(lay[:])
