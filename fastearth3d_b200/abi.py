"""ctypes mirror of the C-ABI structs declared in include/vilma_gpu.h.

`VgParams` is the &vilma namelist record restricted to what the time step
reads (src/vilma_params.f90:26-205); `VgInfo` carries the diagnostics of the
coupling record and the stepper counters (src/vilma_coupling.f90:71-140,
src/vilma_timestep.f90:64-68).
"""
import ctypes as C

VG_MAX_LAYER = 16
VG_RHEOL_ELASTIC, VG_RHEOL_MAXWELL, VG_RHEOL_FLUID = 0, 1, 2
VG_VISC3D_FP64, VG_VISC3D_SPLIT_TC, VG_VISC3D_EXACT_TC = 0, 1, 2

_D16 = C.c_double * VG_MAX_LAYER
_I16 = C.c_int * VG_MAX_LAYER


class VgParams(C.Structure):
    _fields_ = [
        ("lmax", C.c_int), ("nlat", C.c_int), ("nphi", C.c_int),
        ("n_layer", C.c_int),
        ("r_earth", C.c_double),
        ("r_bot", _D16), ("r_top", _D16),
        ("rho", _D16), ("mu", _D16), ("eta", _D16),
        ("rheology", _I16),
        ("ne_layer", _I16),
        ("scheme", C.c_int),
        ("deg1_cm", C.c_int),
        ("skip_tol", C.c_double),
        ("visc3d_tol", C.c_double),
        ("dt_init", C.c_double),
        ("cfl", C.c_double), ("guard_growth", C.c_double),
        ("dt_min", C.c_double), ("dt_max", C.c_double),
        ("sle_n_outer", C.c_int), ("sle_n_inner", C.c_int),
        ("sle_tol", C.c_double),
        ("sle_fixed_ocean", C.c_int), ("sle_subgrid", C.c_int), ("sle_warm_start", C.c_int),
        ("rotation", C.c_int),
        ("visc3d_precision", C.c_int),
        ("rtol", C.c_double), ("atol", C.c_double), ("safety", C.c_double),
        ("grow_max", C.c_double), ("shrink_min", C.c_double),
        ("sle_max_mem_iter", C.c_int),
        ("couple_tol", C.c_double),
        ("toroidal", C.c_int),
        ("sle_ctas", C.c_int),
    ]


class VgInfo(C.Structure):
    _fields_ = [
        ("lmax", C.c_int), ("nlat", C.c_int), ("nphi", C.c_int), ("nlm", C.c_int),
        ("nr", C.c_int), ("ne", C.c_int), ("ndof", C.c_int), ("nk", C.c_int), ("ne3d", C.c_int),
        ("n_sub_last", C.c_int),
        ("n_accept", C.c_longlong), ("n_reject", C.c_longlong), ("n_solve", C.c_longlong),
        ("n_drift_solved", C.c_longlong),
        ("time_yr", C.c_double),
        ("worst_mass_resid", C.c_double),
        ("bsl", C.c_double),
        ("n_outer_last", C.c_int), ("n_inner_last", C.c_int), ("n_coast_flip_last", C.c_int),
        ("n_launch", C.c_longlong),
    ]


VG_PH_DRIFT, VG_PH_ADVANCE_1D, VG_PH_VISC3D, VG_PH_SLE, VG_NPHASE = 0, 1, 2, 3, 4
PHASE_NAMES = ["drift", "advance_1d", "visc3d", "sle", "v3_gather", "v3_synth", "v3_lon_inv", "v3_lon_fwd",
               "v3_analysis", "v3_scatter"]
VG_NPHASE = len(PHASE_NAMES)


def set_layers(p, layers):
    """Fill the layered-earth fields of `p` from a surface-first list of
    (r_bot, r_top, rho, mu, eta, rheology) tuples."""
    p.n_layer = len(layers)
    for i, (rb, rt, rho, mu, eta, rh) in enumerate(layers):
        p.r_bot[i], p.r_top[i], p.rho[i], p.mu[i], p.eta[i], p.rheology[i] = rb, rt, rho, mu, eta, rh


# M3-L70-V01 (src/vilma_earth_structure.f90 build_M3L70V01), the GIA benchmark earth
M3L70V01 = [
    (6301.0e3, 6371.0e3, 3037.0, 5.0605e10, 1e300, VG_RHEOL_ELASTIC),
    (5951.0e3, 6301.0e3, 3438.0, 7.0363e10, 1.0e21, VG_RHEOL_MAXWELL),
    (5701.0e3, 5951.0e3, 3871.0, 1.0549e11, 1.0e21, VG_RHEOL_MAXWELL),
    (3480.0e3, 5701.0e3, 4978.0, 2.2834e11, 2.0e21, VG_RHEOL_MAXWELL),
    (0.0, 3480.0e3, 10750.0, 0.0, 0.0, VG_RHEOL_FLUID),
]
