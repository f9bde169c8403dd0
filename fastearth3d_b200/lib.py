"""ctypes binding of the CUDA library (libvilma_gpu.so) through its C-ABI.

This is the same binding a Python host would write against include/vilma_gpu.h
(the Fortran host binds the same symbols through iso_c_binding). There is no
CPU path: loading fails loudly if the library is missing.
"""
import ctypes as C
import os

import numpy as np

from .abi import VG_NPHASE, VgInfo, VgParams

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvilma_gpu.so")
_lib = None
_P = C.POINTER(C.c_double)
_VP = C.c_void_p

_SIGS = [
    ("vg_params_default", [C.POINTER(VgParams)]),
    ("vg_create", [C.POINTER(VgParams), C.POINTER(_VP)]),
    ("vg_destroy", [_VP]),
    ("vg_set_reference", [_VP, _P, _P, _P]),
    ("vg_enable_visc3d", [_VP, _P]),
    ("vg_update", [_VP, _P, C.c_double]),
    ("vg_update_device", [_VP, C.c_void_p, C.c_double]),
    ("vg_get_fields", [_VP, _P, _P, _P, _P]),
    ("vg_rsl_device", [_VP, C.POINTER(C.c_void_p)]),
    ("vg_get_info", [_VP, C.POINTER(VgInfo)]),
    ("vg_get_rotation", [_VP, _P, _P]),
    ("vg_response_set_dt", [_VP, C.c_double]),
    ("vg_response_begin_step", [_VP]),
    ("vg_response_apply", [_VP, _P, _P, _P]),
    ("vg_response_advance", [_VP, _P]),
    ("vg_get_gains", [_VP, _P, _P, _P]),
    ("vg_get_drift", [_VP, _P, _P, _P]),
    ("vg_get_state", [_VP, _P, _P, _P, _P, _P, _P, _P]),
    ("vg_set_state", [_VP, _P, _P, _P, _P, _P, _P, C.c_double]),
    ("vg_set_fields", [_VP, _P, _P, _P, _P]),
    ("vg_get_rotation_state", [_VP, _P, _P, _P]),
    ("vg_get_step_state", [_VP, _P, _P, C.POINTER(C.c_int)]),
    ("vg_get_toroidal", [_VP, _P]),
    ("vg_enable_visc3d_from_nodes", [_VP, _P, C.c_double, C.c_double, C.c_double]),
    ("vg_advance", [_VP, _P, _P, C.c_double, C.c_double, _P, _P, _P, _P]),
    ("vg_remap_create", [_VP, _P, C.c_int, _P, C.c_int, C.POINTER(_VP)]),
    ("vg_remap_to_gauss", [_VP, _P, _P, C.c_int]),
    ("vg_remap_to_ll", [_VP, _P, _P]),
    ("vg_set_reference_ll", [_VP, _P, _P, _P]),
    ("vg_update_ll", [_VP, _P, C.c_double, _P, _P]),
    ("vg_remap_destroy", [_VP]),
    ("vg_update_batch", [C.POINTER(_VP), C.c_int, C.POINTER(_P), C.c_int, C.c_double, C.c_int,
                         C.POINTER(C.c_int)]),
    ("vg_get_state_tor", [_VP, _P, _P, _P, _P, _P, _P, C.POINTER(C.c_int)]),
    ("vg_set_state_tor", [_VP, _P, _P, _P, _P, _P, _P]),
    ("vg_set_step_state", [_VP, C.c_double, _P, C.c_int]),
    ("vg_set_rotation_state", [_VP, _P, _P, _P]),
    ("vg_spinup", [_VP, _P, C.c_double, C.c_double, C.c_int, _P, C.POINTER(C.c_int), C.POINTER(C.c_int),
                   C.POINTER(C.c_int)]),
    ("vg_misfit", [_VP, C.c_int, C.c_double, _P, C.c_int, C.POINTER(C.c_int), _P, _P]),
    ("vg_misfit_grad", [_VP, C.c_int, C.c_double, _P, C.c_int, C.POINTER(C.c_int), _P, C.c_int, _P, _P, _P]),
    ("vg_sle_misfit", [_VP, C.c_int, C.c_double, _P, C.c_int, C.POINTER(C.c_int), _P, _P]),
    ("vg_autotune", [_VP, C.c_double, C.c_int, C.c_char_p, C.POINTER(C.c_int)]),
    ("vg_get_tuning", [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("vg_sle_misfit_grad", [_VP, C.c_int, C.c_double, _P, C.c_int, C.POINTER(C.c_int), _P, C.c_int, _P, _P, _P,
                            _P]),
    ("vg_sht_analysis", [_VP, _P, _P]),
    ("vg_sht_synthesis", [_VP, _P, _P]),
    ("vg_sht_analysis_noalloc", [_VP, C.c_void_p, C.c_void_p, C.c_int]),
    ("vg_stream", [_VP, C.POINTER(C.c_void_p)]),
    ("vg_profile_enable", [_VP, C.c_int]),
    ("vg_set_wait_limit", [_VP, C.c_double]),
    ("vg_profile_read", [_VP, _P, C.POINTER(C.c_longlong)]),
]
EXPORTS = [n for n, _ in _SIGS] + ["vg_last_error"]


def lib():
    """Load libvilma_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m fastearth3d_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.vg_last_error.argtypes = [_VP]
        L.vg_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_P)


def default_params():
    p = VgParams()
    lib().vg_params_default(C.byref(p))
    return p


class VilmaError(RuntimeError):
    pass


def _pack(z):
    out = np.zeros(2 * z.size)
    out[0::2], out[1::2] = z.real, z.imag
    return out


def _unpack(a):
    return a[0::2] + 1j * a[1::2]


class Model:
    """One model instance on the current CUDA device (vg_create ... vg_destroy)."""

    def __init__(self, p):
        self.p = p
        self._L = lib()  # held by the instance, so that close() at interpreter exit needs no module global
        h = _VP()
        rc = self._L.vg_create(C.byref(p), C.byref(h))
        if rc != 0:
            raise VilmaError(lib().vg_last_error(None).decode())
        self.h = h
        info = self.info()
        self.nlm, self.nk, self.ne, self.nr = info.nlm, info.nk, info.ne, info.nr
        self.ng = p.nphi * p.nlat

    def close(self):
        L = getattr(self, "_L", None)
        if getattr(self, "h", None) and L is not None:
            L.vg_destroy(self.h)
            self.h = None

    __del__ = close

    def _c(self, rc):
        if rc != 0:
            raise VilmaError(lib().vg_last_error(self.h).decode())

    def info(self):
        i = VgInfo()
        self._c(lib().vg_get_info(self.h, C.byref(i)))
        return i

    def set_reference(self, z_bed_eq, h_ice_eq, h_ice_init=None):
        f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        self._c(lib().vg_set_reference(self.h, ptr(f(z_bed_eq)), ptr(f(h_ice_eq)), ptr(f(h_ice_init))))

    def enable_visc3d(self, pert):
        self._c(lib().vg_enable_visc3d(self.h, ptr(np.ascontiguousarray(pert, dtype=np.float64))))

    def update(self, h_ice, dt_yr):
        self._c(lib().vg_update(self.h, ptr(np.ascontiguousarray(h_ice, dtype=np.float64)), dt_yr))

    def spinup(self, h_ice_lgm, t_max_yr, rate_tol, pre_1d=False, with_1d=False):
        """solid_earth_spinup (vg_spinup): returns (model years spent, passes,
        converged) of the full phase, and with with_1d the 1-D phase's passes."""
        t = C.c_double(0.0)
        n, ok, n1 = C.c_int(0), C.c_int(0), C.c_int(0)
        ice = np.ascontiguousarray(h_ice_lgm, dtype=np.float64)
        self._c(lib().vg_spinup(self.h, ptr(ice), t_max_yr, rate_tol, 1 if pre_1d else 0, C.byref(t), C.byref(n),
                                C.byref(ok), C.byref(n1)))
        out = (t.value, n.value, bool(ok.value))
        return out + (n1.value,) if with_1d else out

    def update_device(self, d_h_ice_ptr, dt_yr):
        self._c(lib().vg_update_device(self.h, C.c_void_p(d_h_ice_ptr), dt_yr))

    def rsl_device_ptr(self):
        p = C.c_void_p()
        self._c(lib().vg_rsl_device(self.h, C.byref(p)))
        return p.value

    def fields(self):
        rsl, zb, Cf = np.zeros(self.ng), np.zeros(self.ng), np.zeros(self.ng)
        sig = np.zeros(2 * self.nlm)
        self._c(lib().vg_get_fields(self.h, ptr(rsl), ptr(zb), ptr(Cf), ptr(sig)))
        return rsl, zb, Cf, _unpack(sig)

    def set_fields(self, h_ice=None, rsl=None, z_bed=None, C_ocean=None):
        self._c(lib().vg_set_fields(self.h, *[ptr(None if a is None else np.ascontiguousarray(a, dtype=np.float64))
                                              for a in (h_ice, rsl, z_bed, C_ocean)]))

    def advance_interval(self, ice0, ice1, t0_yr, t1_yr, s_rot=None):
        """vg_advance (stepper_advance): (rsl, C, sigma_lm) at t1."""
        rsl, Cf, sig = np.zeros(self.ng), np.zeros(self.ng), np.zeros(2 * self.nlm)
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (ice0, ice1)]
        sr = None if s_rot is None else np.ascontiguousarray(s_rot, dtype=np.float64)
        self._c(lib().vg_advance(self.h, ptr(a[0]), ptr(a[1]), t0_yr, t1_yr, ptr(sr), ptr(rsl), ptr(Cf), ptr(sig)))
        return rsl, Cf, _unpack(sig)

    def enable_visc3d_from_nodes(self, visc_node, lid_depth=0.0, lid_log10max=0.0, log10_cap=0.0):
        """Lateral viscosity from absolute nodal log10(eta), (nr, nlat*nphi) bottom-up."""
        v = np.ascontiguousarray(visc_node, dtype=np.float64)
        self._c(lib().vg_enable_visc3d_from_nodes(self.h, ptr(v), lid_depth, lid_log10max, log10_cap))

    def toroidal(self):
        """Surface toroidal drift W(a) as t_lm (lm order); zero while not carried."""
        t = np.zeros(2 * self.nlm)
        self._c(lib().vg_get_toroidal(self.h, ptr(t)))
        return t[0::2] + 1j * t[1::2]

    def state_tor(self):
        """Toroidal memory (NLAM_TOR, ne, nk) x 6, or None while not carried."""
        n = 2 * self.ne * self.nk
        arrs = [np.zeros(n) for _ in range(6)]
        c = C.c_int(0)
        self._c(lib().vg_get_state_tor(self.h, *[ptr(a) for a in arrs], C.byref(c)))
        return arrs if c.value else None

    def set_state_tor(self, arrs):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
        self._c(lib().vg_set_state_tor(self.h, *[ptr(a) for a in arrs]))

    def step_state(self):
        """(dt_try [yr], sigma_n as nlm complex, primed) of the time stepper."""
        dt = C.c_double(0.0)
        pr = C.c_int(0)
        q = np.zeros(2 * self.nlm)
        self._c(lib().vg_get_step_state(self.h, C.byref(dt), ptr(q), C.byref(pr)))
        return dt.value, q[0::2] + 1j * q[1::2], bool(pr.value)

    def set_step_state(self, dt_try_yr, sigma_n, primed):
        q = np.zeros(2 * self.nlm)
        q[0::2], q[1::2] = np.real(sigma_n), np.imag(sigma_n)
        self._c(lib().vg_set_step_state(self.h, dt_try_yr, ptr(q), 1 if primed else 0))

    def rotation_state(self):
        n = 6 * self.ne * 4
        m, lm, tm = np.zeros(2), np.zeros(n), np.zeros(n)
        self._c(lib().vg_get_rotation_state(self.h, ptr(m), ptr(lm), ptr(tm)))
        return m, lm, tm

    def set_rotation_state(self, m, load_mem, tidal_mem):
        self._c(lib().vg_set_rotation_state(self.h, ptr(np.ascontiguousarray(m, dtype=np.float64)),
                                            ptr(np.ascontiguousarray(load_mem, dtype=np.float64)),
                                            ptr(np.ascontiguousarray(tidal_mem, dtype=np.float64))))

    def _misfit_args(self, sigma, sites, obs):
        sig = np.ascontiguousarray(np.stack([np.asarray(sigma).real, np.asarray(sigma).imag], axis=-1).reshape(-1),
                                   dtype=np.float64)
        st = np.ascontiguousarray(sites, dtype=np.int32)
        ob = np.ascontiguousarray(obs, dtype=np.float64).reshape(-1)
        return sig, st, ob

    def misfit(self, sigma, dt_s, sites, obs):
        """J of the response-level run (sigma: (nsteps, nlm) complex; obs: (nsteps, nsite))."""
        sig, st, ob = self._misfit_args(sigma, sites, obs)
        J = C.c_double(0)
        self._c(lib().vg_misfit(self.h, len(sigma), dt_s, ptr(sig), len(st),
                                st.ctypes.data_as(C.POINTER(C.c_int)), ptr(ob), C.byref(J)))
        return J.value

    def misfit_grad(self, sigma, dt_s, sites, obs, ckpt_every=50, want_pert=False):
        """(J, dJ/dsigma[, dJ/dpert]): dJ/dsigma shaped like sigma (d/dRe + 1j d/dIm),
        dJ/dpert shaped (ne, nlat, nphi) like the vg_enable_visc3d input."""
        sig, st, ob = self._misfit_args(sigma, sites, obs)
        J = C.c_double(0)
        g = np.zeros_like(sig)
        gp = np.zeros(self.ne * self.ng) if want_pert else None
        self._c(lib().vg_misfit_grad(self.h, len(sigma), dt_s, ptr(sig), len(st),
                                     st.ctypes.data_as(C.POINTER(C.c_int)), ptr(ob), ckpt_every, C.byref(J), ptr(g),
                                     ptr(gp)))
        g = g.reshape(len(sigma), -1, 2)
        out = (J.value, g[..., 0] + 1j * g[..., 1])
        if want_pert:
            out = out + (gp.reshape(self.ne, self.p.nlat, self.p.nphi),)
        return out

    def _sle_args(self, ice, sites, obs):
        ice = np.ascontiguousarray(np.asarray(ice, dtype=np.float64).reshape(-1, self.ng))
        st = np.ascontiguousarray(np.asarray(sites, dtype=np.int32))
        ob = np.ascontiguousarray(np.asarray(obs, dtype=np.float64).reshape(len(ice), len(st)))
        return ice, st, ob

    def sle_misfit(self, ice, dt_yr, sites, obs):
        """J of the coupled run over len(ice) intervals (ice: interval-end thickness per interval)."""
        ice, st, ob = self._sle_args(ice, sites, obs)
        J = C.c_double(0)
        self._c(lib().vg_sle_misfit(self.h, len(ice), dt_yr, ptr(ice), len(st),
                                    st.ctypes.data_as(C.POINTER(C.c_int)), ptr(ob), C.byref(J)))
        return J.value

    def sle_misfit_grad(self, ice, dt_yr, sites, obs, ckpt_every=50, want_pert=False):
        """(J, dJ/dice[, dJ/dpert, dJ/dq]): dJ/dice shaped (nsteps, nlat, nphi); with want_pert
        dJ/dpert shaped (ne, nlat, nphi) and dJ/dq of the shared lateral field's spectrum
        (nlm complex, d/dRe + 1j d/dIm)."""
        ice, st, ob = self._sle_args(ice, sites, obs)
        J = C.c_double(0)
        gi = np.zeros_like(ice)
        gp = np.zeros(self.ne * self.ng) if want_pert else None
        gq = np.zeros(2 * self.nlm) if want_pert else None
        self._c(lib().vg_sle_misfit_grad(self.h, len(ice), dt_yr, ptr(ice), len(st),
                                         st.ctypes.data_as(C.POINTER(C.c_int)), ptr(ob), ckpt_every, C.byref(J),
                                         ptr(gi), ptr(gp), ptr(gq)))
        out = (J.value, gi.reshape(len(ice), self.p.nlat, self.p.nphi))
        if want_pert:
            out = out + (gp.reshape(self.ne, self.p.nlat, self.p.nphi), gq[0::2] + 1j * gq[1::2])
        return out

    def autotune(self, dt_yr, cache_path=None, knobs=3):
        """vg_autotune (knobs: 1 the exact stages' warp splits, 2 the sea-level loop's CTAs);
        returns True when the choices came from the cache file."""
        fc = C.c_int(0)
        path = None if cache_path is None else str(cache_path).encode()
        self._c(lib().vg_autotune(self.h, dt_yr, knobs, path, C.byref(fc)))
        return bool(fc.value)

    def tuning(self):
        """(converter warps of the four exact stages, sea-level loop CTAs)."""
        ncw = (C.c_int * 4)()
        ctas = C.c_int(0)
        self._c(lib().vg_get_tuning(self.h, ncw, C.byref(ctas)))
        return list(ncw), ctas.value

    def rotation(self):
        """Polar motion m (complex, rad) and (kTe, hTe, k_s fluid, k_s flattening)."""
        m, love = np.zeros(2), np.zeros(4)
        self._c(lib().vg_get_rotation(self.h, ptr(m), ptr(love)))
        return m[0] + 1j * m[1], love

    def state(self):
        n = 4 * self.ne * self.nk
        arrs = [np.zeros(n) for _ in range(6)]
        t = C.c_double(0)
        self._c(lib().vg_get_state(self.h, *[ptr(a) for a in arrs], C.byref(t)))
        return arrs, t.value

    def set_state(self, arrs, t):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
        self._c(lib().vg_set_state(self.h, *[ptr(a) for a in arrs], t))

    def set_dt(self, dt_s):
        self._c(lib().vg_response_set_dt(self.h, dt_s))

    def begin_step(self):
        self._c(lib().vg_response_begin_step(self.h))

    def apply(self, sigma):
        s = _pack(np.asarray(sigma, dtype=complex))
        u, n = np.zeros(2 * self.nlm), np.zeros(2 * self.nlm)
        self._c(lib().vg_response_apply(self.h, ptr(s), ptr(u), ptr(n)))
        return _unpack(u), _unpack(n)

    def advance(self, sigma):
        s = _pack(np.asarray(sigma, dtype=complex))
        self._c(lib().vg_response_advance(self.h, ptr(s)))

    def gains(self):
        L = self.p.lmax + 1
        gu, gn, gv = np.zeros(L), np.zeros(L), np.zeros(L)
        self._c(lib().vg_get_gains(self.h, ptr(gu), ptr(gn), ptr(gv)))
        return gu, gn, gv

    def drift(self):
        a = [np.zeros(2 * self.nk) for _ in range(3)]
        self._c(lib().vg_get_drift(self.h, *[ptr(x) for x in a]))
        return [_unpack(x) for x in a]

    def stream_ptr(self):
        s = C.c_void_p()
        self._c(lib().vg_stream(self.h, C.byref(s)))
        return s.value

    def profile_enable(self, on=True):
        self._c(lib().vg_profile_enable(self.h, int(on)))

    def profile_read(self):
        """Per-phase (milliseconds, calls) since the last read (and reset)."""
        ms = np.zeros(VG_NPHASE)
        calls = (C.c_longlong * VG_NPHASE)()
        self._c(lib().vg_profile_read(self.h, ptr(ms), calls))
        return ms, np.array(calls[:])

    def analysis(self, f):
        q = np.zeros(2 * self.nlm)
        self._c(lib().vg_sht_analysis(self.h, ptr(np.ascontiguousarray(f, dtype=np.float64)), ptr(q)))
        return _unpack(q)

    def synthesis(self, q):
        s = _pack(np.asarray(q, dtype=complex))
        f = np.zeros(self.ng)
        self._c(lib().vg_sht_synthesis(self.h, ptr(s), ptr(f)))
        return f


def update_batch(models, ices, dt_yr, on_device=False, nthreads=0):
    """Advance independent models together (vg_update_batch): ices[i] is model
    i's ice, a host array (or, on_device, a device pointer as an int)."""
    n = len(models)
    hs = (_VP * n)(*[m.h for m in models])
    if on_device:
        arr = (_P * n)(*[C.cast(int(p), _P) for p in ices])
    else:
        keep = [np.ascontiguousarray(x, dtype=np.float64) for x in ices]
        arr = (_P * n)(*[ptr(x) for x in keep])
    failed = C.c_int(-1)
    rc = lib().vg_update_batch(hs, n, arr, 1 if on_device else 0, dt_yr, nthreads, C.byref(failed))
    if rc != 0:
        i = failed.value
        msg = lib().vg_last_error(models[i].h if i >= 0 else None).decode()
        raise VilmaError(f"vg_update_batch: instance {i}: {msg}")


class Remap:
    """Host lon-lat <-> Gauss-grid remap of a model (vg_remap_*); fields are
    (nlat_src, nlon) arrays, latitude ascending."""

    def __init__(self, model, lon_src, lat_src):
        self.m = model
        self.lon = np.ascontiguousarray(lon_src, dtype=np.float64)
        self.lat = np.ascontiguousarray(lat_src, dtype=np.float64)
        r = _VP()
        self._L = lib()
        model._c(self._L.vg_remap_create(model.h, ptr(self.lon), len(self.lon), ptr(self.lat), len(self.lat),
                                       C.byref(r)))
        self.r = r
        self.shape = (len(self.lat), len(self.lon))

    def __del__(self):
        L = getattr(self, "_L", None)
        if getattr(self, "r", None) and L is not None:
            L.vg_remap_destroy(self.r)
            self.r = None

    def _c(self, rc):
        if rc != 0:
            raise VilmaError(lib().vg_last_error(self.m.h).decode())

    def to_gauss(self, f_ll, conserve_mass=False):
        g = np.zeros(self.m.ng)
        self._c(lib().vg_remap_to_gauss(self.r, ptr(np.ascontiguousarray(f_ll, dtype=np.float64)), ptr(g),
                                        1 if conserve_mass else 0))
        return g.reshape(self.m.p.nlat, self.m.p.nphi)

    def to_ll(self, f_gauss):
        out = np.zeros(self.shape)
        self._c(lib().vg_remap_to_ll(self.r, ptr(np.ascontiguousarray(f_gauss, dtype=np.float64)), ptr(out)))
        return out

    def set_reference(self, z_bed_eq, h_ice_eq, h_ice_init=None):
        a = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (z_bed_eq, h_ice_eq, h_ice_init)]
        self._c(lib().vg_set_reference_ll(self.r, ptr(a[0]), ptr(a[1]), ptr(a[2])))

    def update(self, h_ice, dt_yr):
        """(rsl, z_bed) on the host grid after the interval."""
        rsl, zb = np.zeros(self.shape), np.zeros(self.shape)
        self._c(lib().vg_update_ll(self.r, ptr(np.ascontiguousarray(h_ice, dtype=np.float64)), dt_yr, ptr(rsl),
                                   ptr(zb)))
        return rsl, zb
