// CPU ORACLE — test infrastructure only (see orc.hpp).
// Sea-level equation (migrating coastline, subgrid term, grounded-ice masking)
// and the forward-Euler sub-stepping driver with its reactive guard.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "orc.hpp"

namespace orc {

// vilma_sle.f90:407-425 ocean_function
void ocean_function(int n, const double* topo, const double* ice, double* C) {
  for (int i = 0; i < n; ++i) C[i] = (topo[i] < 0.0 && RHO_ICE * ice[i] < -RHO_WATER * topo[i]) ? 1.0 : 0.0;
}

// vilma_sle.f90:124-405 sle_solve; the im loop is the sea-level <-> memory
// co-convergence (:218-365): one pass for forward Euler, repeated trapezoid
// endpoint passes until the surface drift settles for the trapezoidal scheme
void sle_solve(SleSolver& sle, const Sht& s, Response& R, const double* d_ice, const double* ice,
               const double* topo0, double* rsl, double* C, SleResult& res, bool report_only,
               cplx* sigma_out, const double* s_rot) {
  const int ng = s.nphi * s.nlat, nlm = s.nlm;
  sle.n_solve++;
  std::vector<double> load(ng), u(ng, 0.0), N(ng, 0.0), Sraw(ng), rsl_new(ng), C0(ng), wcorr(ng, 0.0),
      C_next(ng), d_ice_g(ng, 0.0), tmp(ng), ice_ref(ng);
  std::vector<cplx> load_lm(nlm), u_lm(nlm), N_lm(nlm);
  const double rho_ratio = RHO_ICE / RHO_WATER;
  if (!sle.warm_start)
    for (int i = 0; i < ng; ++i) rsl[i] = 0.0;
  double dphi = 0.0, ice_int = 0.0, zeta_int = 0.0, C_int = 0.0, Cs_int = 0.0;
  res.n_inner_last = 0;
  res.resid = 0.0;
  res.n_outer_done = 0;
  res.n_coast_flip = 0;
  for (int i = 0; i < ng; ++i) ice_ref[i] = ice[i] - d_ice[i];
  ocean_function(ng, topo0, ice_ref.data(), C0.data());  // the reference ocean, :212
  response_begin_step(R, s);
  if (!report_only) response_prepare_endpoint(R);
  auto assemble_load = [&]() {  // assemble_load, :386-405
    for (int i = 0; i < ng; ++i) load[i] = RHO_ICE * d_ice_g[i] + RHO_WATER * (C[i] * rsl[i]) + wcorr[i];
  };
  const int n_mem = report_only ? 1 : sle.max_mem_iter;
  res.n_couple_done = 0;
  for (int im = 1; im <= n_mem; ++im) {    // co-convergence, :230
  for (int io = 1; io <= sle.n_outer; ++io) {  // coastline passes, :231-345
    if (sle.fixed_ocean) {  // the ocean of this pass, :233-247
      if (io == 1)
        for (int i = 0; i < ng; ++i) C[i] = C0[i];
    } else if (io == 1) {
      for (int i = 0; i < ng; ++i) tmp[i] = topo0[i] - rsl[i];
      ocean_function(ng, tmp.data(), ice, C);
    } else {
      for (int i = 0; i < ng; ++i) C[i] = C_next[i];
    }
    // grounded-ice increment and the pass's integrals, :249-294
    for (int i = 0; i < ng; ++i) d_ice_g[i] = ice[i] * (1.0 - C[i]) - (ice[i] - d_ice[i]) * (1.0 - C0[i]);
    C_int = sht_surface_integral(s, C);
    if (C_int <= 0.0) break;
    ice_int = -rho_ratio * sht_surface_integral(s, d_ice_g.data());
    if (sle.subgrid) {
      for (int i = 0; i < ng; ++i) {
        wcorr[i] = -RHO_WATER * topo0[i] * (C[i] - C0[i]);
        tmp[i] = topo0[i] * (C[i] - C0[i]);
      }
      zeta_int = sht_surface_integral(s, tmp.data());
    } else {
      std::fill(wcorr.begin(), wcorr.end(), 0.0);
      zeta_int = 0.0;
    }
    for (int ii = 1; ii <= sle.n_inner; ++ii) {  // the water-load fixed point, :296-318
      assemble_load();
      sht_analysis(s, load.data(), load_lm.data());
      response_apply(R, s, load_lm.data(), u_lm.data(), N_lm.data());
      sht_synth(s, u_lm.data(), u.data());
      sht_synth(s, N_lm.data(), N.data());
      for (int i = 0; i < ng; ++i) {
        Sraw[i] = N[i] - u[i];
        if (s_rot) Sraw[i] = Sraw[i] + s_rot[i];
        tmp[i] = C[i] * Sraw[i];
      }
      Cs_int = sht_surface_integral(s, tmp.data());
      dphi = (ice_int - Cs_int + zeta_int) / C_int;  // mass-conservation offset, :310
      double dmax = 0.0, smax = 0.0;
      for (int i = 0; i < ng; ++i) {
        rsl_new[i] = Sraw[i] + dphi;
        dmax = std::max(dmax, std::fabs(C[i] * (rsl_new[i] - rsl[i])));
      }
      for (int i = 0; i < ng; ++i) {
        rsl[i] = rsl_new[i];
        smax = std::max(smax, std::fabs(C[i] * rsl[i]));
      }
      res.n_inner_last = ii;
      res.resid = dmax;
      if (dmax <= sle.tol * std::max(smax, 2.2250738585072014e-308)) break;  // :317
    }
    res.n_outer_done = io;
    sle.n_outer_tot++;
    sle.n_inner_tot += res.n_inner_last;
    if (sle.fixed_ocean) break;
    // the migrated coastline; C_next becomes C at the top of the next pass, :342-344
    for (int i = 0; i < ng; ++i) tmp[i] = topo0[i] - rsl[i];
    ocean_function(ng, tmp.data(), ice, C_next.data());
    int flips = 0;
    for (int i = 0; i < ng; ++i) flips += (C_next[i] != C[i]);
    res.n_coast_flip = flips;
    if (flips == 0) break;
  }
  // the closing load and the endpoint advance, :346-364
  assemble_load();
  sht_analysis(s, load.data(), load_lm.data());
  if (report_only) break;
  response_advance_endpoint(R, s, load_lm.data());
  res.n_couple_done = im;
  if (response_endpoint_converged(R)) break;
  }
  if (!report_only) response_finalize_step(R);
  if (sigma_out)
    for (int lm = 0; lm < nlm; ++lm) sigma_out[lm] = load_lm[lm];
  // ocean-mass conservation check and the converged offset, :372-381
  for (int i = 0; i < ng; ++i) tmp[i] = C[i] * rsl[i];
  Cs_int = sht_surface_integral(s, tmp.data()) - zeta_int;
  res.ocean_frac = C_int / (16.0 * std::atan(1.0));
  if (std::fabs(ice_int) > 0.0)
    res.mass_resid = std::fabs(Cs_int - ice_int) / std::fabs(ice_int);
  else
    res.mass_resid = std::fabs(Cs_int);
  res.esl = dphi;
  sle.last_outer = res.n_outer_done;
  sle.last_inner = res.n_inner_last;
  sle.last_flips = res.n_coast_flip;
}

// vilma_timestep.f90:79-227 stepper_advance, explicit (forward-Euler) branch.
// The rollback snapshot is held here (response_save_state/restore_state).
int stepper_advance(Stepper& st, const Sht& s, Response& R, SleSolver& sle, const double* topo0,
                    const double* ice0, const double* ice1, const double* ice_ref, double t0, double t1,
                    double* rsl, double* C, const double* s_rot, cplx* sigma_out) {
  const int ng = s.nphi * s.nlat;
  const double span = t1 - t0;
  std::vector<cplx> sig_last(s.nlm, 0.0);
  st.worst_mass_resid = 0.0;
  std::vector<double> ice_now(ng), dice_now(ng), rsl_n(ng);
  SleResult res;
  if (span <= 0.0) {
    for (int i = 0; i < ng; ++i) {
      ice_now[i] = ice0[i];
      dice_now[i] = ice0[i] - ice_ref[i];
    }
    sle_solve(sle, s, R, dice_now.data(), ice_now.data(), topo0, rsl, C, res, true, sig_last.data(), s_rot);
    st.worst_mass_resid = res.mass_resid;
    if (sigma_out) std::copy(sig_last.begin(), sig_last.end(), sigma_out);
    return 0;
  }
  if (R.scheme == SCHEME_TRAP) {
    // vilma_timestep.f90:229-307 implicit branch: step doubling around each
    // trial step, accept / reject against rtol, atol; dt_try carried across calls
    auto solve_at = [&](double t_eval) {
      const double frac = (t_eval - t0) / span;
      for (int i = 0; i < ng; ++i) {
        ice_now[i] = ice0[i] + frac * (ice1[i] - ice0[i]);
        dice_now[i] = ice_now[i] - ice_ref[i];
      }
      st.n_solve++;
      sle_solve(sle, s, R, dice_now.data(), ice_now.data(), topo0, rsl, C, res, false, sig_last.data(), s_rot);
      st.worst_mass_resid = std::max(st.worst_mass_resid, res.mass_resid);
    };
    if (!R.sigma_primed) {  // seed sigma_n with a report-only solve at t0 (:234-241)
      std::vector<cplx> sig0(s.nlm);
      for (int i = 0; i < ng; ++i) {
        ice_now[i] = ice0[i];
        dice_now[i] = ice0[i] - ice_ref[i];
      }
      sle_solve(sle, s, R, dice_now.data(), ice_now.data(), topo0, rsl, C, res, true, sig0.data(), s_rot);
      response_prime_sigma(R, sig0.data());
    }
    const double ricfac = 3.0, expo = 1.0 / 3.0;  // order p = 2: 2^p - 1, 1 / (p + 1)
    double t = t0;
    if (st.dt_try <= 0.0) st.dt_try = span;
    int n_acc = 0;
    while (true) {
      if (t >= t1 - 1.0e-9 * span) break;
      const double dt = std::min(st.dt_try, t1 - t);
      const bool at_floor = (st.dt_min > 0.0 && dt <= st.dt_min * (1.0 + 1.0e-9));
      rsl_n.assign(rsl, rsl + ng);
      response_save_state(R);
      response_set_dt(R, dt);
      solve_at(t + dt);  // coarse
      response_stash_coarse(R);
      response_restore_state(R);
      std::copy(rsl_n.begin(), rsl_n.end(), rsl);
      response_set_dt(R, 0.5 * dt);
      solve_at(t + 0.5 * dt);  // fine
      solve_at(t + dt);
      double err_inf = 0.0, tau_inf = 0.0;
      response_coarse_fine_error(R, err_inf, tau_inf);
      response_set_dt(R, dt);
      const double errsc = (err_inf / ricfac) / (st.atol + st.rtol * tau_inf);
      if (!(errsc <= 1.7976931348623157e308)) return 2;  // non-finite estimate (:268-274)
      const bool accept = (errsc <= 1.0) || at_floor;
      if (accept) {
        t = t + dt;
        st.n_accept++;
        ++n_acc;
        if (at_floor && errsc > 1.0) st.n_floor++;
      } else {
        response_restore_state(R);
        std::copy(rsl_n.begin(), rsl_n.end(), rsl);
        st.n_reject++;
      }
      double fac = (errsc <= 0.0) ? st.grow_max : st.safety * std::pow(errsc, -expo);
      fac = std::min(st.grow_max, std::max(st.shrink_min, fac));
      st.dt_try = std::min(st.dt_max, std::max(st.dt_min, dt * fac));
      if (st.dt_try <= 1.0e-12 * span) return 3;  // step collapsed (:302-303)
    }
    st.n_sub_last = n_acc;
    if (sigma_out) std::copy(sig_last.begin(), sig_last.end(), sigma_out);
    return 0;
  }
  double rate = response_max_rate(R);
  double dt_stab = rate > 0.0 ? st.cfl / rate : span;
  dt_stab = std::min(dt_stab, st.dt_max);
  if (st.dt_min > 0.0) dt_stab = std::max(dt_stab, st.dt_min);
  int n_sub = std::max(1, (int)std::ceil(span / dt_stab - 1.0e-9));
  st.n_sub_last = n_sub;
  double dt = span / (double)n_sub;
  double t = t0;
  double tau_run = response_memory_norm(R);
  std::vector<double> sAre, sAim, sBre, sBim, sCre, sCim;
  while (true) {
    if (t >= t1 - 1.0e-9 * span) break;
    dt = std::min(dt, t1 - t);
    rsl_n.assign(rsl, rsl + ng);
    double tau0 = response_memory_norm(R);
    sAre = R.Are;
    sAim = R.Aim;
    sBre = R.Bre;
    sBim = R.Bim;
    sCre = R.Cre;
    sCim = R.Cim;
    double time_s = R.time;
    response_set_dt(R, dt);
    {  // solve_at(t + dt)
      double frac = (t + dt - t0) / span;
      for (int i = 0; i < ng; ++i) {
        ice_now[i] = ice0[i] + frac * (ice1[i] - ice0[i]);
        dice_now[i] = ice_now[i] - ice_ref[i];
      }
      st.n_solve++;
      sle_solve(sle, s, R, dice_now.data(), ice_now.data(), topo0, rsl, C, res, false, sig_last.data(), s_rot);
      st.worst_mass_resid = std::max(st.worst_mass_resid, res.mass_resid);
    }
    double err_inf = response_memory_norm(R);
    bool finite = err_inf <= 1.7976931348623157e308;
    double scale = std::max(tau0, tau_run);
    bool accept = scale <= 0.0 ? finite : (finite && err_inf <= st.guard_growth * scale);
    if (accept) {
      tau_run = std::max(tau_run, err_inf);
      t = t + dt;
      st.n_accept++;
      dt = std::min(span / (double)n_sub, 2.0 * dt);
    } else {
      R.Are = sAre;
      R.Aim = sAim;
      R.Bre = sBre;
      R.Bim = sBim;
      R.Cre = sCre;
      R.Cim = sCim;
      R.time = time_s;
      std::copy(rsl_n.begin(), rsl_n.end(), rsl);
      st.n_reject++;
      dt = 0.5 * dt;
      if (dt <= 1.0e-12 * span) return 1;
    }
  }
  if (sigma_out) std::copy(sig_last.begin(), sig_last.end(), sigma_out);
  return 0;
}

}  // namespace orc
