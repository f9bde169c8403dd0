/*
 * vilma_gpu.h — C-ABI of the B200 backend for VILMA v2's viscoelastic time step.
 *
 * Plain C: opaque handle, plain pointers and sizes, int status (0 = ok), no
 * exit or abort inside the library. A nonzero status leaves a message in
 * vg_last_error(handle) (or vg_last_error(NULL) for failures before a handle
 * exists); the Fortran shim turns it into `error stop '<msg>'`, the reference's
 * own error convention (e.g. src/vilma_radial_fe.f90:177-187,
 * src/vilma_timestep.f90:221-222).
 *
 * Array conventions (all host arrays are contiguous, Fortran-compatible):
 *   grid fields   (nphi, nlat), phi fastest, colatitude north first
 *                 (src/vilma_sht.f90:11-15; src/vilma_coupling.f90:678-682)
 *   spectra       complex(c_double) of length nlm = (lmax+1)(lmax+2)/2,
 *                 interleaved (re, im), m-major lm order with l ascending
 *                 inside each m (the SHTns order of sht_grid_lmidx,
 *                 src/vilma_sht.f90:349-354), orthonormal, no Condon-Shortley
 *                 phase, m > 0 counted twice for a real field
 *   memory state  six arrays A/B/C re/im of shape (NLAM=4, ne, nk) in the
 *                 reference's degree-grouped slot order k (src/vilma_response.f90:
 *                 629-648, the restart layout of src/vilma_io.f90:12-18)
 * Times are seconds inside the library; vg_update takes years like
 * solid_earth_update (src/vilma_coupling.f90:336-345).
 *
 * Threading: one host thread per handle; a handle owns one CUDA stream and all
 * device state (the reference forbids calls from a host parallel region,
 * src/vilma_tensor_sh.f90:153-163).
 */
#ifndef VILMA_GPU_H
#define VILMA_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VG_MAX_LAYER 16

enum { VG_RHEOL_ELASTIC = 0, VG_RHEOL_MAXWELL = 1, VG_RHEOL_FLUID = 2 };
enum { VG_SCHEME_FE = 0, VG_SCHEME_TRAP = 2 };  /* "fe" | "trap" (SCHEME_* of src/vilma_viscoelastic.f90:60-64) */
enum { VG_VISC3D_FP64 = 0, VG_VISC3D_SPLIT_TC = 1, VG_VISC3D_EXACT_TC = 2 };

/* The &vilma namelist record restricted to what the time step reads
 * (src/vilma_params.f90:26-205). Defaults: vg_params_default. */
typedef struct vg_params {
  /* Gauss grid (src/vilma_params.f90:45-48): nlat/nphi must be given. */
  int lmax, nlat, nphi;
  /* layered earth, surface-first (earth = "custom", src/vilma_earth_structure.f90:82-116) */
  int n_layer;
  double r_earth;
  double r_bot[VG_MAX_LAYER], r_top[VG_MAX_LAYER];
  double rho[VG_MAX_LAYER], mu[VG_MAX_LAYER], eta[VG_MAX_LAYER];
  int rheology[VG_MAX_LAYER];
  /* radial elements per layer; all zero => the reference depth-target rule
   * (src/vilma_radial_fe.f90:43-50, 140-224). No reference counterpart. */
  int ne_layer[VG_MAX_LAYER];
  /* response (src/vilma_params.f90:65-70, 135-158) */
  int scheme;        /* VG_SCHEME_FE ("fe") or VG_SCHEME_TRAP ("trap") */
  int deg1_cm;       /* 1: deg1_frame = "cm", 0: "cf" */
  double skip_tol;   /* drift-solve skip gate, src/vilma_response.f90:88-93 */
  double visc3d_tol; /* 1-D/3-D element split [dex] */
  double dt_init;    /* [s]; 0 => 1 kyr (src/vilma_coupling.f90:258) */
  /* explicit stepper (src/vilma_timestep.f90:51-61) */
  double cfl, guard_growth, dt_min, dt_max;
  /* sea-level equation (src/vilma_params.f90:73-78; src/vilma_sle.f90:57-98) */
  int sle_n_outer, sle_n_inner;
  double sle_tol;
  int sle_fixed_ocean, sle_subgrid, sle_warm_start;
  /* rotational feedback / polar wander (src/vilma_params.f90:96,
   * src/vilma_rotation.f90), coupled per interval like
   * src/vilma_coupling.f90:399-424 */
  int rotation;
  /* arithmetic of the 3-D stress products (no reference counterpart):
   * VG_VISC3D_FP64 (default) on the CUDA cores; VG_VISC3D_EXACT_TC, the
   * Legendre and longitude contractions on the tensor cores as 8-bit digit
   * slices of 38-bit fixed-point operands with exact int32 accumulation
   * (~36 significant bits per product, FP64 between the stages);
   * VG_VISC3D_SPLIT_TC, the same contractions with two-term TF32 operands and
   * FP32 accumulation (rsl within ~2e-6 of the FP64 path on the lmax-128
   * workload) */
  int visc3d_precision;
  /* trapezoidal scheme (scheme = VG_SCHEME_TRAP): the step-doubling controller
   * (src/vilma_timestep.f90:40-53, 229-307; rtol, atol, safety, grow_max,
   * shrink_min of src/vilma_params.f90:86-92), the sea-level <-> memory
   * co-convergence cap (sle_max_mem_iter, src/vilma_params.f90:76) and its
   * tolerance on the surface drift (couple_tol, src/vilma_response.f90:177) */
  double rtol, atol, safety, grow_max, shrink_min;
  int sle_max_mem_iter;
  double couple_tol;
  /* l_toroidal (src/vilma_params.f90:156, default 0): carry the toroidal
   * degree of freedom (W and the lambda 3, 4 memory) once a genuinely 3-D
   * element exists (src/vilma_response.f90:1048-1118) */
  int toroidal;
  /* CTAs of the fused sea-level loop (no reference counterpart): 0 = one per
   * SM; fewer leave room for other instances' kernels when several handles
   * share the GPU (vg_update_batch). Results do not depend on it. */
  int sle_ctas;
} vg_params;

/* Phase timers (the reference's [PROFILE] buckets: drift solve, memory
 * advance, 3-D advance, sea-level transforms + grid work; src/vilma_drive.f90:
 * 219-305). */
enum {
  VG_PH_DRIFT = 0,
  VG_PH_ADVANCE_1D = 1,
  VG_PH_VISC3D = 2,
  VG_PH_SLE = 3,
  /* stages inside VG_PH_VISC3D (FP64 path: the whole longitude pass is V3_LON_INV) */
  VG_PH_V3_GATHER = 4,
  VG_PH_V3_SYNTH = 5,
  VG_PH_V3_LON_INV = 6,
  VG_PH_V3_LON_FWD = 7,
  VG_PH_V3_ANALYSIS = 8,
  VG_PH_V3_SCATTER = 9,
  VG_NPHASE = 10
};

typedef struct vg_info {
  int lmax, nlat, nphi, nlm, nr, ne, ndof, nk, ne3d;
  int n_sub_last;         /* sub-steps taken by the last vg_update */
  long long n_accept, n_reject, n_solve, n_drift_solved;
  double time_yr;         /* model time [yr] */
  double worst_mass_resid;
  double bsl;             /* barystatic sea level diagnostic [m] */
  int n_outer_last, n_inner_last, n_coast_flip_last;
  long long n_launch;     /* kernels launched by the time step so far */
} vg_info;

typedef struct vg_handle vg_handle;

/* Fill p with the reference defaults (src/vilma_params.f90:26-205) and the
 * 4-layer synthetic earth used by the benchmarks of this backend. */
int vg_params_default(vg_params* p);

/* solid_earth_init, build part (src/vilma_coupling.f90:144-156, 252-318):
 * Gauss grid, radial mesh, per-degree operators assembled and factored on the
 * device, unit-load gains, zero memory. Replaces build_sht + build_solver. */
int vg_create(const vg_params* p, vg_handle** out);

/* solid_earth_init, data part: reference bed z_bed_eq and reference ice
 * h_ice_eq on the Gauss grid (the `grid` argument absent: data already on
 * Gauss, src/vilma_coupling.f90:166-170), optional current ice h_ice_init
 * (NULL => h_ice_eq). Sets rsl = 0, z_bed = z_bed_eq, C = C0. */
int vg_set_reference(vg_handle* h, const double* z_bed_eq, const double* h_ice_eq,
                     const double* h_ice_init);

/* Laterally varying viscosity: log10 viscosity perturbation per element on
 * the Gauss grid, (nphi, nlat, ne) (response_enable_lateral_visc,
 * src/vilma_response.f90:994-1053). */
int vg_enable_visc3d(vg_handle* h, const double* pert);
/* The same from absolute nodal log10 viscosities (response_enable_lateral_visc_
 * from_nodes, src/vilma_response.f90:1120-1169): visc_node is (nphi*nlat, nr),
 * Gauss grid point fastest, radial nodes bottom-up. An element takes the mean
 * of its two nodes; elements wholly above the lid base r_earth - lid_depth
 * (lid_depth > 0; <= 0 turns the rule off) with a value above lid_log10max take
 * log10_cap; the perturbation is that minus log10 of the element's radial
 * viscosity. Elastic and fluid elements stay as they are. */
int vg_enable_visc3d_from_nodes(vg_handle* h, const double* visc_node, double lid_depth, double lid_log10max,
                                double log10_cap);

/* solid_earth_update (src/vilma_coupling.f90:336-437):
 * advance by dt_yr years with the ice linearly interpolated from the carried
 * ice to h_ice (stepper_advance, src/vilma_timestep.f90:79-227). h_ice is a
 * host array. */
int vg_update(vg_handle* h, const double* h_ice, double dt_yr);
/* Same, with h_ice a device pointer (nphi*nlat doubles) on the handle's GPU. */
int vg_update_device(vg_handle* h, const double* d_h_ice, double dt_yr);
/* stepper_advance (src/vilma_timestep.f90:79-105) for hosts that run their own
 * interval driver: advance from t0_yr (which becomes the model time) to t1_yr
 * with the ice interpolated linearly from ice0 to ice1 (host arrays, nphi*nlat);
 * s_rot (may be NULL) is the rotational-feedback term of rsl held across the
 * interval, as the reference's caller passes it (not with rotation = 1, where
 * the library integrates the rotation itself). Outputs (any may be NULL): rsl
 * and C on the Gauss grid and the converged surface load sigma_lm at t1
 * (sigma_out). */
int vg_advance(vg_handle* h, const double* ice0, const double* ice1, double t0_yr, double t1_yr, const double* s_rot,
               double* rsl, double* C, double* sigma_lm);

/* Host-grid coupling (src/vilma_remap.f90:56-166; src/vilma_coupling.f90:
 * 144-176, 336-447, 625-641): when the host's lon-lat grid is not the model's
 * Gauss grid, ice (and the reference fields) come in by first-order
 * conservative remapping and rsl goes back by bilinear interpolation, on the
 * device. Host fields are (nlon, nlat) with longitude fastest and latitude
 * ascending (south first), as the reference's grid_class axes; lon_src and
 * lat_src are the cell-centre axes in degrees, ascending (longitudes in any
 * 360-degree window). A remap belongs to its handle, which must outlive it.
 *   vg_remap_create      remap_init: cell boundaries at the axis midpoints
 *   vg_remap_to_gauss    remap_to_gauss (stat "mean"; conserve_mass rescales so
 *                        the Gauss quadrature integral equals the source area
 *                        integral)
 *   vg_remap_to_ll       remap_to_ll (bilinear)
 *   vg_set_reference_ll  solid_earth_init with a host grid: z_bed_eq remapped as
 *                        geometry, h_ice_eq / h_ice_init with the mass rescale
 *   vg_update_ll         solid_earth_update with a host grid: the ice remapped
 *                        in, the interval, rsl remapped out and z_bed =
 *                        z_bed_eq - rsl on the host's own bed (either output may
 *                        be NULL) */
typedef struct vg_remap vg_remap;
int vg_remap_create(vg_handle* h, const double* lon_src, int nlon, const double* lat_src, int nlat,
                    vg_remap** out);
int vg_remap_to_gauss(vg_remap* r, const double* f_ll, double* f_gauss, int conserve_mass);
int vg_remap_to_ll(vg_remap* r, const double* f_gauss, double* f_ll);
int vg_set_reference_ll(vg_remap* r, const double* z_bed_eq_ll, const double* h_ice_eq_ll,
                        const double* h_ice_init_ll);
int vg_update_ll(vg_remap* r, const double* h_ice_ll, double dt_yr, double* rsl_ll, double* z_bed_ll);
int vg_remap_destroy(vg_remap* r);

/* Ensemble batching (no reference counterpart: the reference advances one
 * model per process): advance n independent handles -- instances with their
 * own lmax, earth, lateral viscosity and ice -- by dt_yr each, as vg_update
 * (ice_on_device = 0: ice[i] is a host array) or vg_update_device (1: a device
 * pointer) would, concurrently: every handle keeps its own stream, and up to
 * nthreads host threads (<= 0: one per handle) drive them, the costliest
 * first, so that their kernels overlap on the GPU. Results are identical to n
 * sequential calls. The handles must be distinct. Returns 0 when every update
 * succeeded, else the status of the first failing handle (its message in
 * vg_last_error(hs[i])) with *failed_index = i (failed_index may be NULL);
 * argument errors return nonzero with *failed_index = -1 and the message in
 * vg_last_error(NULL). */
int vg_update_batch(vg_handle* const* hs, int n, const double* const* ice, int ice_on_device, double dt_yr,
                    int nthreads, int* failed_index);

/* Outputs of the coupling record (se%rsl, se%z_bed, se%gg%C, se%sigma_lm,
 * src/vilma_coupling.f90:71-140). Any pointer may be NULL. */
int vg_get_fields(vg_handle* h, double* rsl, double* z_bed, double* C, double* sigma_lm);
/* Device pointer of the rsl field (read-only, valid until vg_destroy). */
int vg_rsl_device(vg_handle* h, const double** d_rsl);
int vg_get_info(vg_handle* h, vg_info* info);
/* Rotational feedback (rotation = 1; src/vilma_rotation.f90): polar motion
 * m = m1 + i m2 [rad] as (re, im), and the degree-2 constants (k^T_e, h^T_e,
 * k^T_f the secular k_s used, k_s from the observed flattening). Either
 * pointer may be NULL. Fails when rotation is off. */
int vg_get_rotation(vg_handle* h, double* m, double* love);

/* Response-level operators (src/vilma_response.f90:43-52, 266-319) for a run
 * without the sea-level equation (bench_visc3d style): begin_step freezes the
 * drift from the current memory; apply returns u_lm, n_lm for a load sigma_lm;
 * advance commits the forward-Euler memory update with sigma_lm and adds dt. */
int vg_response_set_dt(vg_handle* h, double dt_s);
int vg_response_begin_step(vg_handle* h);
int vg_response_apply(vg_handle* h, const double* sigma_lm, double* u_lm, double* n_lm);
int vg_response_advance(vg_handle* h, const double* sigma_lm);
/* elastic per-degree gains gu, gn, gv (0..lmax) (src/vilma_response.f90:603-627) */
int vg_get_gains(vg_handle* h, double* gu, double* gn, double* gv);
/* surface drift dUa, dFa, dVa (complex, nk each, interleaved) of the last begin_step */
int vg_get_drift(vg_handle* h, double* dUa, double* dFa, double* dVa);

/* Prognostic state in the restart layout (src/vilma_io.f90:12-18, 414-569):
 * six arrays of NLAM*ne*nk doubles (A re, A im, B re, B im, C re, C im) and the
 * model time [s]. */
int vg_get_state(vg_handle* h, double* Are, double* Aim, double* Bre, double* Bim,
                 double* Cre, double* Cim, double* time_s);
int vg_set_state(vg_handle* h, const double* Are, const double* Aim, const double* Bre,
                 const double* Bim, const double* Cre, const double* Cim, double time_s);
/* The restart's diagnostic fields, restored when present (vilma_restart_read,
 * src/vilma_io.f90:414-468, 587-597): carried ice h_ice, rsl (the sea-level
 * warm start), z_bed, ocean function C, all (nphi, nlat). NULL skips a field.
 * After vg_set_reference. */
int vg_set_fields(vg_handle* h, const double* h_ice, const double* rsl, const double* z_bed,
                  const double* C);
/* The toroidal part of the surface horizontal displacement, t_lm of
 * u_h = e_r x grad_1(sum t_lm Y_lm): the surface W(a) of the last drift solve
 * (response_horizontal_toroidal, src/vilma_response.f90:884-900), nlm complex
 * interleaved in lm order; zero while no toroidal field is carried. */
int vg_get_toroidal(vg_handle* h, double* t_lm);
/* Toroidal memory (lambda 3, 4) in the reference's restart order (NLAM_TOR = 2,
 * ne, nk): the channels 5, 6 of its (6, ne, nk) restart arrays
 * (src/vilma_io.f90:505-530). *carried = 0 (and nothing written) while the
 * toroidal channels are not carried; set requires them carried (vg_enable_visc3d
 * with toroidal = 1 and a genuinely 3-D element) and follows vg_set_state. */
int vg_get_state_tor(vg_handle* h, double* Are, double* Aim, double* Bre, double* Bim, double* Cre, double* Cim,
                     int* carried);
int vg_set_state_tor(vg_handle* h, const double* Are, const double* Aim, const double* Bre, const double* Bim,
                     const double* Cre, const double* Cim);
/* Time-stepping restart state (the restart variables "dt_try", "sigma_n_re",
 * "sigma_n_im", "sigma_primed" of src/vilma_io.f90:38-46, 329-334, 457-458,
 * 599-615): the adaptive controller's next-step suggestion dt_try [yr] (used by
 * the trapezoidal scheme, carried by every scheme) and the trapezoidal
 * scheme's start-of-step load sigma_n (nlm complex, interleaved) with its
 * primed flag (0: not tracked; the next update seeds it with a report-only
 * solve). vg_set_state clears the flag, so restore with vg_set_step_state
 * after it. sigma_n may be NULL (get: not returned; set: only with primed = 0). */
int vg_get_step_state(vg_handle* h, double* dt_try_yr, double* sigma_n, int* sigma_primed);
int vg_set_step_state(vg_handle* h, double dt_try_yr, const double* sigma_n, int sigma_primed);
/* Rotation restart state (rotation_get_memory / rotation_set_memory,
 * src/vilma_rotation.f90:275-295): polar motion m as (re, im) and the load and
 * tidal channels' memory stress, each (NLAM=4, ne, 6) Fortran order with the
 * last axis [A re, A im, B re, B im, C re, C im]. */
int vg_get_rotation_state(vg_handle* h, double* m, double* load_mem, double* tidal_mem);
int vg_set_rotation_state(vg_handle* h, const double* m, const double* load_mem, const double* tidal_mem);

/* LGM-memory spin-up, solid_earth_spinup (src/vilma_coupling.f90:453-570):
 * a zero-length update seeds the entering ice with h_ice_lgm (nphi, nlat);
 * with pre_1d (pre_spinup_1d) and lateral viscosity enabled, the 3-D elements
 * first take the lateral mean of their log10-viscosity perturbation and the
 * held load relaxes to rest with no time cap (relax_hold's internal pass cap
 * only), after which the real 3-D field is restored; then, if t_max_yr > 0
 * (equil_time_max), the full model relaxes (relax_hold): h_ice_lgm held over
 * passes of 200 yr growing by 1.6 per pass (at most 60, at most t_max_yr in
 * total) until the mean bed velocity int |z_bed - z_prev| dOmega / (4 pi) /
 * pass falls below rate_tol [m/yr] (equil_rate_tol). Neither phase (pre_1d = 0
 * and t_max_yr <= 0) does nothing. Outputs (any may be NULL), of the full
 * phase: the model time spent [yr], the passes, 1 if the bed came to rest
 * before the cap; passes_1d: the passes of the 1-D phase. */
int vg_spinup(vg_handle* h, const double* h_ice_lgm, double t_max_yr, double rate_tol, int pre_1d,
              double* t_done_yr, int* passes, int* converged, int* passes_1d);

/* Relative-sea-level misfit of a response-level run and its gradient
 * (hand-written discrete adjoint; the reference has no counterpart). From the
 * handle's current memory, nsteps steps of length dt_s: begin_step, apply and
 * advance (src/vilma_response.f90:228-319) with the load sigma_lm[n] (nlm
 * complex per step, interleaved) held over step n, no sea-level equation:
 *   J = sum_n sum_s (rsl_n(site[s]) - obs[n * nsite + s])^2,  rsl = N - u
 * at the Gauss-grid points site[s] (land sites, no ocean). vg_misfit_grad also
 * returns dJ/dsigma (same layout as sigma_lm; NULL skips it) and, with
 * lateral viscosity (FP64 path), dJ/dpert with respect to the log10-viscosity
 * perturbation of vg_enable_visc3d ((nphi, nlat, ne); zero on elements that
 * are not 3-D; NULL skips it), from a reverse sweep that keeps the memory every
 * ckpt_every steps and recomputes each segment from it. With 3-D elements a
 * segment's longitude grids are held on the device: min(ckpt_every, nsteps) x
 * nlat x 18 ne3d x nphi doubles (about 0.26 GB a step at lmax 128 with 54
 * 3-D elements). The handle's memory is left as it was. The drift skip gate
 * is off inside these calls. */
int vg_misfit(vg_handle* h, int nsteps, double dt_s, const double* sigma_lm, int nsite, const int* site,
              const double* obs, double* J);
int vg_misfit_grad(vg_handle* h, int nsteps, double dt_s, const double* sigma_lm, int nsite, const int* site,
                   const double* obs, int ckpt_every, double* J, double* grad_sigma, double* grad_pert);

/* Relative-sea-level misfit of the coupled time step and its gradient
 * (hand-written discrete adjoint; the reference has no counterpart). From the
 * handle's current state, nsteps intervals of vg_update (solid_earth_update,
 * src/vilma_coupling.f90:336-437: forward-Euler sub-steps, the sea-level
 * equation of src/vilma_sle.f90:124-405 with its migrating coastline, the
 * guard) of dt_yr each, ice[n * ng ...] the ice thickness at the end of
 * interval n on the Gauss grid ((nphi, nlat), phi fastest):
 *   J = sum_n sum_s (rsl_n(site[s]) - obs[n * nsite + s])^2,
 * rsl_n the relative sea level after interval n at the grid points site[s].
 * vg_sle_misfit_grad also returns, with the forward's discrete decisions held
 * (its sub-steps, the ocean function of every sea-level pass, the inner
 * iterations done):
 *   grad_ice      dJ/d ice, nsteps x ng (NULL skips it); the ice of each
 *                 sub-step is interpolated in time between the interval's
 *                 ends (solve_at, src/vilma_timestep.f90:314-326), so ice[n]
 *                 collects from intervals n and n + 1;
 *   grad_pert     with lateral viscosity (FP64 path), dJ/d the log10-viscosity
 *                 perturbation of vg_enable_visc3d, (ne, nlat, nphi), zero on
 *                 elements that are not 3-D (NULL skips it);
 *   grad_pert_lm  dJ/d the spectrum q of one lateral field shared by every
 *                 3-D element (pert_e = the handle's synthesis of q), nlm
 *                 complex (interleaved re/im, d/dRe and d/dIm); a caller that
 *                 keeps degrees <= 32 reads those entries (NULL skips it).
 * The reverse sweep keeps the interval driver's state every ckpt_every
 * intervals and recomputes each segment from it; a segment's longitude grids
 * (3-D elements) are held on the device, about 0.26 GB per sub-step at lmax
 * 128 with 54 3-D elements. Forward Euler only, no rotation; the toroidal
 * channels are differentiated with the rest (FP64 path); the drift skip
 * gate is off inside these calls. The handle's state (memory, rsl, ice,
 * ocean function, z_bed, time, counters) is put back afterwards. */
int vg_sle_misfit(vg_handle* h, int nsteps, double dt_yr, const double* ice, int nsite, const int* site,
                  const double* obs, double* J);
int vg_sle_misfit_grad(vg_handle* h, int nsteps, double dt_yr, const double* ice, int nsite, const int* site,
                       const double* obs, int ckpt_every, double* J, double* grad_ice, double* grad_pert,
                       double* grad_pert_lm);

/* Gauss-grid transforms on the device (sht_grid_synthesis / _analysis,
 * src/vilma_sht.f90:204-226), host arrays in and out. */
int vg_sht_analysis(vg_handle* h, const double* f, double* q_lm);
int vg_sht_synthesis(vg_handle* h, const double* q_lm, double* f);

/* vg_sht_analysis on device buffers, allocating nothing (no counterpart in the
 * reference). d_f holds `batch` grid fields ((nphi, nlat) each, phi fastest),
 * d_q_lm receives `batch` spectra (nlm complex each, interleaved re/im). The
 * work is queued on the handle's stream and not waited for.
 * For callers that may not allocate device memory at the point of the call:
 * hosts that reserve all device memory up front (a climate coupler with its
 * own pool), code that runs while memory is exhausted, and callers that
 * cannot tolerate the implicit synchronisation an allocation brings. The
 * Fourier scratch is a file-scope device array of VG_NOALLOC_SCRATCH_DOUBLES
 * doubles per device, so 2 * (mmax + 1) * nlat * batch must not exceed it
 * (larger requests return an error); its address in the current context is
 * looked up on every call, with the handle's device current, so a
 * cudaDeviceReset between calls is safe (the first call on a device may load
 * the module: make it before any stream capture). The scratch carries
 * nothing between calls. Calls that
 * overlap in time on one device share that array and race: order them on
 * one stream. */
#define VG_NOALLOC_SCRATCH_DOUBLES (1 << 19)
int vg_sht_analysis_noalloc(vg_handle* h, const double* d_f, double* d_q_lm, int batch);

/* Autotuner of the launch shapes (no reference counterpart: the reference's
 * OpenMP loops have none). Times a few intervals of the handle's own model on
 * the ice it holds, from its current state (put back afterwards), for each
 * candidate of the knobs selected in `knobs` (VG_TUNE_STAGES | VG_TUNE_SLE;
 * an ensemble that shares the GPU keeps its own sea-level CTA count and
 * tunes the stages only), both leaving the results unchanged bit for bit: the
 * exact tensor-core stages' split of their worker warps between converters
 * and epilogue (8 : 8 or 4 : 12, per stage) and the fused sea-level loop's CTA
 * count (one per SM, one per Gauss row, two per SM). The fastest choices are
 * applied to the handle and appended to the text file cache_path (NULL: no
 * cache), keyed by lmax, grid, elements, 3-D elements, precision, toroidal
 * channels, ocean and knobs;
 * a later call for a model of the same key reads them from there instead of
 * timing (*from_cache = 1). Needs vg_set_reference first. */
#define VG_TUNE_STAGES 1 /* the exact stages' warp splits */
#define VG_TUNE_SLE 2    /* the fused sea-level loop's CTA count */
int vg_autotune(vg_handle* h, double dt_yr, int knobs, const char* cache_path, int* from_cache);
/* The current choices: converter warps of the four exact stages (zeros
 * without an exact-stage plan) and the sea-level loop's CTA count (0: one per
 * SM). */
int vg_get_tuning(vg_handle* h, int* ncw, int* sle_ctas);

/* The CUDA stream (cudaStream_t) all of the handle's work is ordered on, so a
 * caller can record events on it. */
int vg_stream(vg_handle* h, void** stream);
/* Bound, in seconds (default 2, at most 60), on every device-side wait that
 * hands work from one CTA or warp to another: the grid barriers of the fused
 * sea-level loop and the producer / consumer waits of the tensor-core stages
 * (no reference counterpart: the reference has no device code). A wait that
 * runs out ends its kernel early with a status bit, and the call that
 * launched it returns nonzero with a message; waits for the hardware's own
 * copies and matrix operations keep their fixed bound. For hosts that want
 * a hung peer reported sooner, and for tests of that error path. */
int vg_set_wait_limit(vg_handle* h, double seconds);
/* Enable (1) or disable (0) the phase timers; vg_profile_read returns the
 * accumulated milliseconds and call counts per phase (VG_NPHASE each) since
 * the last read and resets them. */
int vg_profile_enable(vg_handle* h, int on);
int vg_profile_read(vg_handle* h, double* ms, long long* calls);

int vg_destroy(vg_handle* h);
const char* vg_last_error(const vg_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* VILMA_GPU_H */
