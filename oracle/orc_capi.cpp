// CPU ORACLE — test infrastructure only (see orc.hpp).
// The coupling driver (solid_earth_init/update, src/vilma_coupling.f90) and a
// C API mirroring include/vilma_gpu.h with an `orc_` prefix, so the tests can
// drive the oracle and the CUDA library through the same calls.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>

#include <omp.h>

#include "../include/vilma_gpu.h"
#include "orc.hpp"

using namespace orc;

struct OrcHandle {
  vg_params p;
  Earth earth;
  Mesh mesh;
  Sht sht;
  Response R;
  SleSolver sle;
  Stepper st;
  std::vector<double> z_bed_eq, h_ice_eq, h_ice, rsl, z_bed, C, C0;
  std::vector<cplx> sigma_lm;
  double time_yr = 0.0, bsl = 0.0;
  SleResult last;
  Rotation rot;
  std::string err;
};

static std::string g_err;

extern "C" {

int orc_params_default(vg_params* p) {
  std::memset(p, 0, sizeof(*p));
  const double km = 1e3;
  p->lmax = 16;
  p->nlat = 17;
  p->nphi = 34;
  p->n_layer = 4;
  p->r_earth = 6371.0 * km;
  const double rb[4] = {6301.0 * km, 5701.0 * km, 3480.0 * km, 0.0};
  const double rt[4] = {6371.0 * km, 6301.0 * km, 5701.0 * km, 3480.0 * km};
  const double rho[4] = {3300.0, 3450.0, 4900.0, 10900.0};
  const double mu[4] = {0.7e11, 0.9e11, 2.0e11, 0.0};
  const double eta[4] = {1e300, 5e20, 2e21, 0.0};
  const int rh[4] = {VG_RHEOL_ELASTIC, VG_RHEOL_MAXWELL, VG_RHEOL_MAXWELL, VG_RHEOL_FLUID};
  for (int i = 0; i < 4; ++i) {
    p->r_bot[i] = rb[i];
    p->r_top[i] = rt[i];
    p->rho[i] = rho[i];
    p->mu[i] = mu[i];
    p->eta[i] = eta[i];
    p->rheology[i] = rh[i];
  }
  p->scheme = VG_SCHEME_FE;
  p->deg1_cm = 1;
  p->skip_tol = 1e-4;
  p->visc3d_tol = 1e-3;
  p->dt_init = 0.0;
  p->cfl = 1.0;
  p->guard_growth = 1e3;
  p->dt_min = 0.0;
  p->dt_max = 1.7976931348623157e308;
  p->sle_n_outer = 3;
  p->sle_n_inner = 20;
  p->sle_tol = 1e-7;
  p->sle_fixed_ocean = 0;
  p->sle_subgrid = 1;
  p->sle_warm_start = 1;
  p->rotation = 0;
  p->visc3d_precision = VG_VISC3D_FP64;
  p->rtol = 1e-4;
  p->atol = 1e-3;
  p->safety = 0.9;
  p->grow_max = 5.0;
  p->shrink_min = 0.2;
  p->sle_max_mem_iter = 20;
  p->couple_tol = 1e-6;
  p->toroidal = 0;
  p->sle_ctas = 0;
  return 0;
}

int orc_create(const vg_params* p, OrcHandle** out) {
  try {
    OrcHandle* h = new OrcHandle();
    h->p = *p;
    h->earth.r_earth = p->r_earth;
    for (int i = 0; i < p->n_layer; ++i) {
      Layer L;
      L.r_bot = p->r_bot[i];
      L.r_top = p->r_top[i];
      L.rho = p->rho[i];
      L.mu = p->mu[i];
      L.eta = p->eta[i];
      L.rheology = p->rheology[i];
      h->earth.layers.push_back(L);
    }
    h->mesh = radial_mesh_build(h->earth, p->ne_layer);
    sht_init(h->sht, p->lmax, p->nlat, p->nphi);
    double dt0 = p->dt_init > 0.0 ? p->dt_init : KYR;
    h->R.deg1_cm = p->deg1_cm != 0;
    h->R.skip_tol = p->skip_tol;
    h->R.visc3d_tol = p->visc3d_tol;
    if (p->scheme != SCHEME_FE && p->scheme != SCHEME_TRAP)
      throw std::runtime_error("vilma_params: scheme must be \"fe\" or \"trap\"");
    response_init_ve(h->R, h->earth, h->mesh, h->sht, dt0);
    h->R.scheme = p->scheme;
    h->R.couple_tol = p->couple_tol;
    h->R.toroidal = p->toroidal != 0;
    h->sle.max_mem_iter = p->sle_max_mem_iter;
    h->st.rtol = p->rtol;
    h->st.atol = p->atol;
    h->st.safety = p->safety;
    h->st.grow_max = p->grow_max;
    h->st.shrink_min = p->shrink_min;
    h->sle.n_outer = p->sle_n_outer;
    h->sle.n_inner = p->sle_n_inner;
    h->sle.tol = p->sle_tol;
    h->sle.fixed_ocean = p->sle_fixed_ocean != 0;
    h->sle.subgrid = p->sle_subgrid != 0;
    h->sle.warm_start = p->sle_warm_start != 0;
    h->st.cfl = p->cfl;
    h->st.guard_growth = p->guard_growth;
    h->st.dt_min = p->dt_min;
    h->st.dt_max = p->dt_max;
    h->sigma_lm.assign(h->sht.nlm, 0.0);
    // rotational feedback (src/vilma_coupling.f90:310-316)
    if (p->rotation) rotation_init(h->rot, h->earth, h->mesh, dt0);
    *out = h;
    return 0;
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return 1;
  }
}

int orc_destroy(OrcHandle* h) {
  delete h;
  return 0;
}

// OpenMP threads of the oracle's parallel loops (the baseline's core count)
int orc_set_threads(int n) {
  if (n < 1) return 1;
  omp_set_num_threads(n);
  return 0;
}

const char* orc_last_error(const OrcHandle* h) { return h ? h->err.c_str() : g_err.c_str(); }

int orc_set_reference(OrcHandle* h, const double* z_bed_eq, const double* h_ice_eq, const double* h_ice_init) {
  const int ng = h->sht.nphi * h->sht.nlat;
  h->z_bed_eq.assign(z_bed_eq, z_bed_eq + ng);
  h->h_ice_eq.assign(h_ice_eq, h_ice_eq + ng);
  h->h_ice.assign(h_ice_init ? h_ice_init : h_ice_eq, (h_ice_init ? h_ice_init : h_ice_eq) + ng);
  h->rsl.assign(ng, 0.0);
  h->z_bed = h->z_bed_eq;
  h->C0.assign(ng, 0.0);
  ocean_function(ng, h->z_bed_eq.data(), h->h_ice_eq.data(), h->C0.data());
  h->C = h->C0;
  return 0;
}

int orc_enable_visc3d(OrcHandle* h, const double* pert) {
  sht_calibrate_n6(h->sht);
  response_enable_lateral_visc(h->R, h->sht, pert);
  return 0;
}

// vilma_response.f90:1120-1169 response_enable_lateral_visc_from_nodes:
// visc_node (nphi*nlat, nr) absolute log10 viscosity; element = log10-mean of
// its nodes, capped in the lid, minus log10 of the radial viscosity
int orc_enable_visc3d_from_nodes(OrcHandle* h, const double* visc_node, double lid_depth, double lid_log10max,
                                 double log10_cap) {
  const Response& R = h->R;
  const size_t ng = (size_t)h->sht.nphi * h->sht.nlat;
  const double r_top = R.r[R.nr - 1];
  const double r_lid = lid_depth > 0.0 ? r_top - lid_depth : 1.7976931348623157e308;
  std::vector<double> pert((size_t)R.ne * ng, 0.0);
  for (int e = 0; e < R.ne; ++e) {
    if (R.MkPerDt[e] == 0.0) continue;
    const double logeta_ref = std::log10(R.mu[e] / R.MkPerDt[e]);
    const bool in_lid = R.r[e] >= r_lid - 1.0e-6 * r_top;
    for (size_t g = 0; g < ng; ++g) {
      double v = 0.5 * (visc_node[(size_t)e * ng + g] + visc_node[(size_t)(e + 1) * ng + g]);
      if (in_lid && v > lid_log10max) v = log10_cap;
      pert[(size_t)e * ng + g] = v - logeta_ref;
    }
  }
  return orc_enable_visc3d(h, pert.data());
}

// vilma_coupling.f90:572-597 update_bsl
static void update_bsl(OrcHandle* h) {
  const int ng = h->sht.nphi * h->sht.nlat;
  double c_int = sht_surface_integral(h->sht, h->C.data());
  if (c_int > 0.0) {
    std::vector<double> t(ng);
    for (int i = 0; i < ng; ++i) t[i] = h->h_ice[i] * (1.0 - h->C[i]) - h->h_ice_eq[i] * (1.0 - h->C0[i]);
    h->bsl = -(RHO_ICE / RHO_WATER) * sht_surface_integral(h->sht, t.data()) / c_int;
  } else {
    h->bsl = 0.0;
  }
}

// vilma_coupling.f90:336-437 solid_earth_update; with rotation the feedback is
// coupled at the interval level (:399-424): s_rot from the entering polar motion
// is held across the interval, then the polar motion is advanced under the
// interval-end load, sub-stepped to the channels' stability ceiling.
int orc_update(OrcHandle* h, const double* h_ice, double dt_yr) {
  const int ng = h->sht.nphi * h->sht.nlat;
  double dt = dt_yr * SEC_PER_YEAR;
  double t0 = h->time_yr * SEC_PER_YEAR, t1 = t0 + dt;
  std::vector<double> ice_new(h_ice, h_ice + ng);
  std::vector<double> s_rot;
  if (h->rot.enabled) {
    rotation_begin_step(h->rot, dt);
    s_rot.resize(ng);
    rotation_s_rot(h->rot, h->sht, s_rot.data());
  }
  int rc = stepper_advance(h->st, h->sht, h->R, h->sle, h->z_bed_eq.data(), h->h_ice.data(), ice_new.data(),
                           h->h_ice_eq.data(), t0, t1, h->rsl.data(), h->C.data(),
                           h->rot.enabled ? s_rot.data() : nullptr, h->sigma_lm.data());
  if (rc) {
    h->err = rc == 1   ? "vilma_timestep: explicit guard sub-step collapsed (viscosity too stiff for FE)"
             : rc == 2 ? "vilma_timestep: implicit local-error estimate went non-finite"
                       : "vilma_timestep: implicit adaptive step collapsed (tolerance unreachable)";
    return rc;
  }
  if (h->rot.enabled) {
    std::vector<double> load(ng);
    sht_synth(h->sht, h->sigma_lm.data(), load.data());
    const int n_sub = std::max(1, (int)std::ceil(dt / h->rot.dt_fe_max));
    const double dt_sub = dt / (double)n_sub;
    for (int k = 0; k < n_sub; ++k) rotation_update(h->rot, h->sht, load.data(), dt_sub);
  }
  h->h_ice = ice_new;
  for (int i = 0; i < ng; ++i) h->z_bed[i] = h->z_bed_eq[i] - h->rsl[i];
  h->time_yr += dt_yr;
  update_bsl(h);
  return 0;
}

// vilma_coupling.f90:500-545 relax_hold: hold h_ice_lgm over passes of 200 yr
// growing by 1.6 (at most 60, capped at t_cap when t_cap > 0) until the mean
// bed velocity int |dz_bed| dOmega / (4 pi) / pass falls below tol [m/yr]
static int relax_hold(OrcHandle* h, const double* h_ice_lgm, double t_cap, double tol, double* t_done, int* passes,
                      int* converged) {
  const int ng = h->sht.nphi * h->sht.nlat;
  *t_done = 0.0;
  *passes = 0;
  *converged = 0;
  std::vector<double> prev = h->z_bed, d(ng);
  double pass_dt = 200.0;
  for (int it = 1; it <= 60; ++it) {
    if (t_cap > 0.0) pass_dt = std::min(pass_dt, t_cap - *t_done);
    if (pass_dt <= 0.0) break;
    int rc = orc_update(h, h_ice_lgm, pass_dt);
    if (rc) return rc;
    *t_done += pass_dt;
    *passes = it;
    for (int i = 0; i < ng; ++i) d[i] = std::fabs(h->z_bed[i] - prev[i]);
    const double rate = sht_surface_integral(h->sht, d.data()) / (4.0 * PI) / pass_dt;
    if (rate < tol) {
      *converged = 1;
      break;
    }
    prev = h->z_bed;
    pass_dt = pass_dt * 1.6;
  }
  return 0;
}

// vilma_coupling.f90:453-498 solid_earth_spinup: seed the entering ice with a
// zero-length update; with pre_1d relax to rest under the lateral mean of the
// 3-D viscosity (every 3-D element at mu / eta * 10^-(mean perturbation),
// :484-493), then restore the real field; then relax_hold up to t_cap
int orc_spinup(OrcHandle* h, const double* h_ice_lgm, double t_cap, double tol, int pre_1d, double* t_done,
               int* passes, int* converged, int* passes_1d) {
  *t_done = 0.0;
  *passes = 0;
  *converged = 0;
  *passes_1d = 0;
  if (!pre_1d && !(t_cap > 0.0)) return 0;
  int rc = orc_update(h, h_ice_lgm, 0.0);
  if (rc) return rc;
  if (pre_1d) {
    Response& R = h->R;
    const bool mean = R.lat_visc && R.ne3d > 0;
    std::vector<double> mk = R.MkPerDt;
    std::vector<char> act = R.active1d;
    std::vector<int> e3d = R.e3d;
    const int ne3d = R.ne3d;
    if (mean) {
      for (int ei = 0; ei < ne3d; ++ei) {
        R.MkPerDt[e3d[ei]] = mk[e3d[ei]] * std::pow(10.0, -R.pert_mean3d[ei]);
        R.active1d[e3d[ei]] = 1;
      }
      R.e3d.clear();
      R.ne3d = 0;
      R.lat_visc = false;
    }
    double t1 = 0.0;
    int c1 = 0;
    rc = relax_hold(h, h_ice_lgm, -1.0, tol, &t1, passes_1d, &c1);
    if (mean) {  // the real 3-D field (solid_earth_enable_visc_3d)
      R.MkPerDt = mk;
      R.active1d = act;
      R.e3d = e3d;
      R.ne3d = ne3d;
      R.lat_visc = true;
      for (int e = 0; e < R.ne; ++e) R.Mk[e] = R.MkPerDt[e] * R.dt;
    }
    if (rc) return rc;
  }
  if (t_cap > 0.0) return relax_hold(h, h_ice_lgm, t_cap, tol, t_done, passes, converged);
  return 0;
}

// vilma_timestep.f90:79-105 stepper_advance, driven directly: t0 becomes the
// model time, ice0 the carried ice; s_rot may be null
int orc_advance(OrcHandle* h, const double* ice0, const double* ice1, double t0_yr, double t1_yr,
                const double* s_rot, double* rsl, double* C, double* sigma_lm) {
  const int ng = h->sht.nphi * h->sht.nlat;
  h->h_ice.assign(ice0, ice0 + ng);
  std::vector<double> ice_new(ice1, ice1 + ng);
  h->time_yr = t0_yr;
  h->R.time = t0_yr * SEC_PER_YEAR;
  int rc = stepper_advance(h->st, h->sht, h->R, h->sle, h->z_bed_eq.data(), h->h_ice.data(), ice_new.data(),
                           h->h_ice_eq.data(), t0_yr * SEC_PER_YEAR, t1_yr * SEC_PER_YEAR, h->rsl.data(), h->C.data(),
                           s_rot, h->sigma_lm.data());
  if (rc) {
    h->err = "vilma_timestep: the interval failed";
    return rc;
  }
  h->h_ice = ice_new;
  h->time_yr = t1_yr;
  for (int i = 0; i < ng; ++i) h->z_bed[i] = h->z_bed_eq[i] - h->rsl[i];
  update_bsl(h);
  if (rsl) std::copy(h->rsl.begin(), h->rsl.end(), rsl);
  if (C) std::copy(h->C.begin(), h->C.end(), C);
  if (sigma_lm)
    for (int lm = 0; lm < h->sht.nlm; ++lm) {
      sigma_lm[2 * lm] = h->sigma_lm[lm].real();
      sigma_lm[2 * lm + 1] = h->sigma_lm[lm].imag();
    }
  return 0;
}

// polar motion m (re, im) and the degree-2 constants kTe, hTe, k_s (fluid), k_s (flattening)
int orc_get_rotation(OrcHandle* h, double* m, double* love) {
  if (m) {
    m[0] = h->rot.m.real();
    m[1] = h->rot.m.imag();
  }
  if (love) {
    love[0] = h->rot.kTe;
    love[1] = h->rot.hTe;
    love[2] = h->rot.k_s_fluid;
    love[3] = h->rot.k_s_flat;
  }
  return h->rot.enabled ? 0 : 1;
}

// rotation_update under a held load (the standalone polar-motion step of
// tests/test_rotation.f90) and the rigid (2,1) inertia of a load
int orc_rotation_update(OrcHandle* h, const double* load, double dt_s) {
  if (!h->rot.enabled) return 1;
  rotation_update(h->rot, h->sht, load, dt_s);
  return 0;
}
int orc_rotation_inertia(OrcHandle* h, const double* load, double* I21) {
  cplx v = inertia21(h->sht, load, h->earth.r_earth);
  I21[0] = v.real();
  I21[1] = v.imag();
  return 0;
}

int orc_get_fields(OrcHandle* h, double* rsl, double* z_bed, double* C, double* sigma_lm) {
  const int ng = h->sht.nphi * h->sht.nlat;
  if (rsl) std::copy(h->rsl.begin(), h->rsl.end(), rsl);
  if (z_bed) std::copy(h->z_bed.begin(), h->z_bed.end(), z_bed);
  if (C) std::copy(h->C.begin(), h->C.begin() + ng, C);
  if (sigma_lm)
    for (int lm = 0; lm < h->sht.nlm; ++lm) {
      sigma_lm[2 * lm] = h->sigma_lm[lm].real();
      sigma_lm[2 * lm + 1] = h->sigma_lm[lm].imag();
    }
  return 0;
}

int orc_get_info(OrcHandle* h, vg_info* info) {
  std::memset(info, 0, sizeof(*info));
  info->lmax = h->sht.lmax;
  info->nlat = h->sht.nlat;
  info->nphi = h->sht.nphi;
  info->nlm = h->sht.nlm;
  info->nr = h->R.nr;
  info->ne = h->R.ne;
  info->ndof = h->R.ndof;
  info->nk = h->R.nk;
  info->ne3d = h->R.ne3d;
  info->n_sub_last = h->st.n_sub_last;
  info->n_outer_last = h->sle.last_outer;
  info->n_inner_last = h->sle.last_inner;
  info->n_coast_flip_last = h->sle.last_flips;
  info->n_accept = h->st.n_accept;
  info->n_reject = h->st.n_reject;
  info->n_solve = h->st.n_solve;
  info->n_drift_solved = h->R.n_solved;
  info->time_yr = h->time_yr;
  info->worst_mass_resid = h->st.worst_mass_resid;
  info->bsl = h->bsl;
  return 0;
}

int orc_response_set_dt(OrcHandle* h, double dt_s) {
  response_set_dt(h->R, dt_s);
  return 0;
}
int orc_response_begin_step(OrcHandle* h) {
  response_begin_step(h->R, h->sht);
  return 0;
}
int orc_response_apply(OrcHandle* h, const double* sigma_lm, double* u_lm, double* n_lm) {
  const int nlm = h->sht.nlm;
  std::vector<cplx> s(nlm), u(nlm), n(nlm);
  for (int lm = 0; lm < nlm; ++lm) s[lm] = cplx(sigma_lm[2 * lm], sigma_lm[2 * lm + 1]);
  response_apply(h->R, h->sht, s.data(), u.data(), n.data());
  for (int lm = 0; lm < nlm; ++lm) {
    u_lm[2 * lm] = u[lm].real();
    u_lm[2 * lm + 1] = u[lm].imag();
    n_lm[2 * lm] = n[lm].real();
    n_lm[2 * lm + 1] = n[lm].imag();
  }
  return 0;
}
int orc_response_advance(OrcHandle* h, const double* sigma_lm) {
  const int nlm = h->sht.nlm;
  std::vector<cplx> s(nlm);
  for (int lm = 0; lm < nlm; ++lm) s[lm] = cplx(sigma_lm[2 * lm], sigma_lm[2 * lm + 1]);
  response_advance(h->R, h->sht, s.data());
  h->R.time += h->R.dt;
  return 0;
}
int orc_get_gains(OrcHandle* h, double* gu, double* gn, double* gv) {
  for (int l = 0; l <= h->R.lmax; ++l) {
    if (gu) gu[l] = h->R.gu[l];
    if (gn) gn[l] = h->R.gn[l];
    if (gv) gv[l] = h->R.gv[l];
  }
  return 0;
}
int orc_get_drift(OrcHandle* h, double* dUa, double* dFa, double* dVa) {
  for (int k = 0; k < h->R.nk; ++k) {
    if (dUa) {
      dUa[2 * k] = h->R.dUa[k].real();
      dUa[2 * k + 1] = h->R.dUa[k].imag();
    }
    if (dFa) {
      dFa[2 * k] = h->R.dFa[k].real();
      dFa[2 * k + 1] = h->R.dFa[k].imag();
    }
    if (dVa) {
      dVa[2 * k] = h->R.dVa[k].real();
      dVa[2 * k + 1] = h->R.dVa[k].imag();
    }
  }
  return 0;
}
// state in the reference (NLAM, ne, nk) layout == the oracle's [k][e][lam]
int orc_get_state(OrcHandle* h, double* Are, double* Aim, double* Bre, double* Bim, double* Cre, double* Cim,
                  double* time_s) {
  std::copy(h->R.Are.begin(), h->R.Are.end(), Are);
  std::copy(h->R.Aim.begin(), h->R.Aim.end(), Aim);
  std::copy(h->R.Bre.begin(), h->R.Bre.end(), Bre);
  std::copy(h->R.Bim.begin(), h->R.Bim.end(), Bim);
  std::copy(h->R.Cre.begin(), h->R.Cre.end(), Cre);
  std::copy(h->R.Cim.begin(), h->R.Cim.end(), Cim);
  if (time_s) *time_s = h->R.time;
  return 0;
}
int orc_set_state(OrcHandle* h, const double* Are, const double* Aim, const double* Bre, const double* Bim,
                  const double* Cre, const double* Cim, double time_s) {
  size_t n = h->R.Are.size();
  h->R.Are.assign(Are, Are + n);
  h->R.Aim.assign(Aim, Aim + n);
  h->R.Bre.assign(Bre, Bre + n);
  h->R.Bim.assign(Bim, Bim + n);
  h->R.Cre.assign(Cre, Cre + n);
  h->R.Cim.assign(Cim, Cim + n);
  h->R.time = time_s;
  return 0;
}
// response_horizontal_toroidal (vilma_response.f90:884-900): t_lm of the
// surface W(a) of the last drift solve, in lm order; zero while no toroidal
// field is carried
int orc_get_toroidal(OrcHandle* h, double* t_lm) {
  for (int lm = 0; lm < 2 * h->sht.nlm; ++lm) t_lm[lm] = 0.0;
  if (h->R.nlam == NLAM) return 0;
  for (int k = 0; k < h->R.nk; ++k) {
    t_lm[2 * h->R.k2lm[k]] = h->R.dWa[k].real();
    t_lm[2 * h->R.k2lm[k] + 1] = h->R.dWa[k].imag();
  }
  return 0;
}
// toroidal memory in the (NLAM_TOR, ne, nk) layout; *carried = 0 (and
// nothing written) while only the spheroidal channels exist
int orc_get_state_tor(OrcHandle* h, double* Are, double* Aim, double* Bre, double* Bim, double* Cre, double* Cim,
                      int* carried) {
  *carried = h->R.nlam > NLAM ? 1 : 0;
  if (!*carried) return 0;
  std::copy(h->R.Atre.begin(), h->R.Atre.end(), Are);
  std::copy(h->R.Atim.begin(), h->R.Atim.end(), Aim);
  std::copy(h->R.Btre.begin(), h->R.Btre.end(), Bre);
  std::copy(h->R.Btim.begin(), h->R.Btim.end(), Bim);
  std::copy(h->R.Ctre.begin(), h->R.Ctre.end(), Cre);
  std::copy(h->R.Ctim.begin(), h->R.Ctim.end(), Cim);
  return 0;
}
// dense toroidal operator of degree j on the params' mesh (nr x nr, column-major)
int orc_toroidal_operator(const vg_params* p, int j, double* A, int* nr_out) {
  Earth e;
  e.r_earth = p->r_earth;
  for (int i = 0; i < p->n_layer; ++i) {
    Layer L;
    L.r_bot = p->r_bot[i];
    L.r_top = p->r_top[i];
    L.rho = p->rho[i];
    L.mu = p->mu[i];
    L.eta = p->eta[i];
    L.rheology = p->rheology[i];
    e.layers.push_back(L);
  }
  Mesh m = radial_mesh_build(e, p->ne_layer);
  *nr_out = m.nr;
  if (A) {
    std::vector<double> mu(m.ne);
    for (int k = 0; k < m.ne; ++k) mu[k] = e.layers[m.elem_layer[k]].mu;  // as response_init_ve
    std::vector<double> D = build_toroidal_operator(m.r, mu, j);
    std::copy(D.begin(), D.end(), A);
  }
  return 0;
}
int orc_sht_analysis(OrcHandle* h, const double* f, double* q) {
  std::vector<cplx> c(h->sht.nlm);
  sht_analysis(h->sht, f, c.data());
  for (int lm = 0; lm < h->sht.nlm; ++lm) {
    q[2 * lm] = c[lm].real();
    q[2 * lm + 1] = c[lm].imag();
  }
  return 0;
}
int orc_sht_synthesis(OrcHandle* h, const double* q, double* f) {
  std::vector<cplx> c(h->sht.nlm);
  for (int lm = 0; lm < h->sht.nlm; ++lm) c[lm] = cplx(q[2 * lm], q[2 * lm + 1]);
  sht_synth(h->sht, c.data(), f);
  return 0;
}

// ---- stand-alone pieces for the known-answer tests -----------------------
// Elastic loading Love numbers of a layered earth at degree j
// (test_benchmark_love.f90 path: mesh, assemble, unit-load solve, loading_love).
int orc_love_numbers(const vg_params* p, int jmin, int jmax, double* h_out, double* l_out, double* k_out) {
  try {
    Earth e;
    e.r_earth = p->r_earth;
    for (int i = 0; i < p->n_layer; ++i) {
      Layer L;
      L.r_bot = p->r_bot[i];
      L.r_top = p->r_top[i];
      L.rho = p->rho[i];
      L.mu = p->mu[i];
      L.eta = p->eta[i];
      L.rheology = p->rheology[i];
      e.layers.push_back(L);
    }
    Mesh m = radial_mesh_build(e, p->ne_layer);
#pragma omp parallel for schedule(dynamic)
    for (int j = jmin; j <= jmax; ++j) {
      RadialOp op;
      radial_operator_assemble(op, e, m, j);
      std::vector<double> b(op.ndof), x(op.ndof);
      radial_operator_load_rhs(op, 1.0, b.data());
      radial_operator_solve_vec(op, b.data(), x.data(), nullptr);
      double hh, ll, kk;
      loading_love(e, j, 1.0, x[idx_u(op.nr - 1)], x[idx_v(op.nr - 1)], x[idx_f(op.nr - 1)], hh, ll, kk);
      h_out[j - jmin] = hh;
      l_out[j - jmin] = ll;
      k_out[j - jmin] = kk;
    }
    return 0;
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return 1;
  }
}

// Band LU of a dense n x n matrix (column-major) through the band machinery,
// solved for one RHS (test_band.f90 path).
int orc_band_dense_solve(int n, const double* A, const double* b, double* x) {
  std::vector<int> rows, cols;
  std::vector<double> vals;
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i)
      if (A[(size_t)k * n + i] != 0.0) {
        rows.push_back(i + 1);
        cols.push_back(k + 1);
        vals.push_back(A[(size_t)k * n + i]);
      }
  Band B;
  if (!band_build(B, n, rows, cols, vals)) return 2;
  for (int i = 0; i < n; ++i) x[i] = b[i];
  band_solve(B, x);
  return 0;
}

// Dense per-degree operator (with the E_uniq term for j = 1), for the symmetry check.
int orc_dense_operator(const vg_params* p, int j, int with_uniq, double* A, int* nd_out) {
  Earth e;
  e.r_earth = p->r_earth;
  for (int i = 0; i < p->n_layer; ++i) {
    Layer L;
    L.r_bot = p->r_bot[i];
    L.r_top = p->r_top[i];
    L.rho = p->rho[i];
    L.mu = p->mu[i];
    L.eta = p->eta[i];
    L.rheology = p->rheology[i];
    e.layers.push_back(L);
  }
  Mesh m = radial_mesh_build(e, p->ne_layer);
  int nd = ndof_of(m.nr);
  *nd_out = nd;
  if (A) {
    std::vector<double> D = build_dense_operator(e, m, j, with_uniq != 0);
    std::copy(D.begin(), D.end(), A);
  }
  return 0;
}

// tensor synth/analysis round trip on the handle's grid (test_tensor_sh path);
// nch = 4 (spheroidal) or 6 (with the toroidal lambda 3, 4)
int orc_tensor_synth(OrcHandle* h, const double* c /* nch*nlm complex, channel-major */, double* dyad, int nch) {
  if (nch != 4 && nch != 6) return 2;
  sht_calibrate_n6(h->sht);
  std::vector<cplx> cc((size_t)nch * h->sht.nlm);
  for (size_t t = 0; t < cc.size(); ++t) cc[t] = cplx(c[2 * t], c[2 * t + 1]);
  tensor_synth(h->sht, cc.data(), dyad, nch);
  return 0;
}
int orc_tensor_analysis(OrcHandle* h, const double* dyad, double* c, int nch) {
  if (nch != 4 && nch != 6) return 2;
  sht_calibrate_n6(h->sht);
  std::vector<cplx> cc((size_t)nch * h->sht.nlm);
  tensor_analysis(h->sht, dyad, cc.data(), nch);
  for (size_t t = 0; t < cc.size(); ++t) {
    c[2 * t] = cc[t].real();
    c[2 * t + 1] = cc[t].imag();
  }
  return 0;
}
int orc_grid(OrcHandle* h, double* colat, double* wts) {
  for (int j = 0; j < h->sht.nlat; ++j) {
    if (colat) colat[j] = h->sht.colat[j];
    if (wts) wts[j] = h->sht.wts[j];
  }
  return 0;
}
double orc_surface_integral(OrcHandle* h, const double* f) { return sht_surface_integral(h->sht, f); }
int orc_mesh(OrcHandle* h, double* r, int* elem_layer) {
  for (int i = 0; i < h->mesh.nr; ++i)
    if (r) r[i] = h->mesh.r[i];
  for (int e = 0; e < h->mesh.ne; ++e)
    if (elem_layer) elem_layer[e] = h->mesh.elem_layer[e];
  return 0;
}

}  // extern "C"
