// CPU ORACLE — test infrastructure only (see orc.hpp).
// Viscoelastic field driver: per-degree operators and unit-load response,
// Maxwell memory kernel, drift solve with the skip gate, affine apply, the
// forward-Euler memory advance, and the pseudo-spectral 3-D advance.
#include <string>
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "orc.hpp"

namespace orc {

// vilma_viscoelastic.f90:329-359 strain_coeffs
static inline void strain_coeffs(double u1, double u2, double v1, double v2, double Jr, double a[4],
                                 double b[4], double c[4]) {
  a[0] = -u1 + u2;
  b[0] = 0.0;
  c[0] = 0.0;
  a[1] = -v1 + v2;
  b[1] = u1 - v1;
  c[1] = u2 - v2;
  a[2] = 0.0;
  b[2] = -u1 / Jr + 0.5 * v1;
  c[2] = -u2 / Jr + 0.5 * v2;
  a[3] = 0.0;
  b[3] = 0.5 * v1;
  c[3] = 0.5 * v2;
  if (Jr <= 2.0) {
    b[3] = 0.0;
    c[3] = 0.0;
  }
}

// vilma_viscoelastic.f90:361-371 ve_strain_constants
static void ve_strain_constants(double Jr, double norm[4], double sa[16], double sb[16], double sc[16]) {
  norm[0] = 1.0;
  norm[1] = 0.5 * Jr;
  norm[2] = 2.0 * Jr * Jr;
  norm[3] = 2.0 * Jr * (Jr - 2.0);
  const double unit[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
  for (int t = 0; t < 4; ++t)
    strain_coeffs(unit[t][0], unit[t][1], unit[t][2], unit[t][3], Jr, &sa[t * 4], &sb[t * 4], &sc[t * 4]);
}

// vilma_viscoelastic.f90:441-480 dissipative_rhs; A/B/C are (4, ne) [e][lam]
static void dissipative_rhs(int ne, const double* r, const double* sa, const double* sb, const double* sc,
                            const double* norm, const double* Am, const double* Bm, const double* Cm,
                            double* f) {
  const double xg = 0.5773502691896257;
  const double gp[2] = {-xg, xg};
  for (int e = 0; e < ne; ++e) {
    double rk = r[e], rk1 = r[e + 1], h = rk1 - rk;
    double floc[4] = {0, 0, 0, 0};
    for (int ig = 0; ig < 2; ++ig) {
      double ra = 0.5 * (h * gp[ig] + rk + rk1);
      double psik = (rk1 - ra) / h, psik1 = (ra - rk) / h;
      double tauV[4];
      for (int m = 0; m < 4; ++m)
        tauV[m] = Am[e * 4 + m] / h + Bm[e * 4 + m] * psik / ra + Cm[e * 4 + m] * psik1 / ra;
      for (int t = 0; t < 4; ++t) {
        double D = 0.0;
        for (int m = 0; m < 4; ++m) {
          double deps = sa[t * 4 + m] / h + sb[t * 4 + m] * psik / ra + sc[t * 4 + m] * psik1 / ra;
          D = D + norm[m] * tauV[m] * deps;
        }
        floc[t] = floc[t] - D * ra * ra * h * 0.5;
      }
    }
    f[idx_u(e)] += floc[0];
    f[idx_u(e + 1)] += floc[1];
    f[idx_v(e)] += floc[2];
    f[idx_v(e + 1)] += floc[3];
  }
}

// vilma_viscoelastic.f90:482-589 advance_memory, forward-Euler branch (:577-584)
static void advance_memory_fe(int ne, const double* mu, const double* Mk, const double* Un, const double* Vn,
                              double Jr, double* Am, double* Bm, double* Cm, const char* active) {
  for (int e = 0; e < ne; ++e) {
    if (active && !active[e]) continue;
    double a[4], b[4], c[4];
    strain_coeffs(Un[e], Un[e + 1], Vn[e], Vn[e + 1], Jr, a, b, c);
    double Me = Mk[e];
    double om = 1.0 - Me, two_muM = 2.0 * mu[e] * Me;
    for (int m = 0; m < 4; ++m) {
      Am[e * 4 + m] = om * Am[e * 4 + m] - two_muM * a[m];
      Bm[e * 4 + m] = om * Bm[e * 4 + m] - two_muM * b[m];
      Cm[e * 4 + m] = om * Cm[e * 4 + m] - two_muM * c[m];
    }
  }
}

// vilma_viscoelastic.f90:482-589 advance_memory, trapezoidal branch (:556-569):
// tau_{n+1} = [(1 - M/2) tau_n - mu M (eps_n + eps_{n+1})] / (1 + M/2) with
// eps_{n+1} from (Un, Vn) and eps_n from (Un_prev, Vn_prev)
static void advance_memory_trap(int ne, const double* mu, const double* Mk, const double* Un, const double* Vn,
                                const double* Un_prev, const double* Vn_prev, double Jr, double* A, double* B,
                                double* C, const char* active) {
  for (int e = 0; e < ne; ++e) {
    if (!active[e]) continue;
    double a[4], b[4], c[4], ap[4], bp[4], cp[4];
    strain_coeffs(Un[e], Un[e + 1], Vn[e], Vn[e + 1], Jr, a, b, c);
    strain_coeffs(Un_prev[e], Un_prev[e + 1], Vn_prev[e], Vn_prev[e + 1], Jr, ap, bp, cp);
    const double Me = Mk[e], denom = 1.0 + 0.5 * Me;
    const double c_old = (1.0 - 0.5 * Me) / denom, w_eps = mu[e] * Me / denom;
    for (int m = 0; m < 4; ++m) {
      A[e * 4 + m] = c_old * A[e * 4 + m] - w_eps * (a[m] + ap[m]);
      B[e * 4 + m] = c_old * B[e * 4 + m] - w_eps * (b[m] + bp[m]);
      C[e * 4 + m] = c_old * C[e * 4 + m] - w_eps * (c[m] + cp[m]);
    }
  }
}

// ------------------------------------------------------------- toroidal kernels
// vilma_viscoelastic.f90:373-390 strain_coeffs_tor: lam 0 = lambda 3, 1 = lambda 4
static inline void strain_coeffs_tor(double w1, double w2, double Jr, double a[2], double b[2], double c[2]) {
  a[0] = -w1 + w2;
  b[0] = -w1;
  c[0] = -w2;
  a[1] = 0.0;
  b[1] = w1;
  c[1] = w2;
  if (Jr <= 2.0) {
    b[1] = 0.0;
    c[1] = 0.0;
  }
}

// vilma_viscoelastic.f90:392-401 ve_strain_constants_tor
static void ve_strain_constants_tor(double Jr, double norm[2], double sa[4], double sb[4], double sc[4]) {
  norm[0] = 0.5 * Jr;
  norm[1] = 0.5 * Jr * (Jr - 2.0);
  strain_coeffs_tor(1.0, 0.0, Jr, &sa[0], &sb[0], &sc[0]);
  strain_coeffs_tor(0.0, 1.0, Jr, &sa[2], &sb[2], &sc[2]);
}

// vilma_viscoelastic.f90:403-439 dissipative_rhs_tor; A/B/C are (2, ne) [e][lam],
// f per node
static void dissipative_rhs_tor(int ne, const double* r, const double* sa, const double* sb, const double* sc,
                                const double* norm, const double* Am, const double* Bm, const double* Cm,
                                double* f) {
  const double xg = 0.5773502691896257;
  const double gp[2] = {-xg, xg};
  for (int e = 0; e < ne; ++e) {
    double rk = r[e], rk1 = r[e + 1], h = rk1 - rk;
    double floc[2] = {0, 0};
    for (int ig = 0; ig < 2; ++ig) {
      double ra = 0.5 * (h * gp[ig] + rk + rk1);
      double psik = (rk1 - ra) / h, psik1 = (ra - rk) / h;
      double tauV[2];
      for (int m = 0; m < 2; ++m)
        tauV[m] = Am[e * 2 + m] / h + Bm[e * 2 + m] * psik / ra + Cm[e * 2 + m] * psik1 / ra;
      for (int t = 0; t < 2; ++t) {
        double D = 0.0;
        for (int m = 0; m < 2; ++m) {
          double deps = sa[t * 2 + m] / h + sb[t * 2 + m] * psik / ra + sc[t * 2 + m] * psik1 / ra;
          D = D + norm[m] * tauV[m] * deps;
        }
        floc[t] = floc[t] - D * ra * ra * h * 0.5;
      }
    }
    f[e] += floc[0];
    f[e + 1] += floc[1];
  }
}

// vilma_viscoelastic.f90:591-629 advance_memory_tor with maxwell_fe (:640-654)
// or, given Wn_prev, maxwell_trap (:683-700)
static void advance_memory_tor(int ne, const double* mu, const double* Mk, const double* Wn, const double* Wn_prev,
                               double Jr, double* A, double* B, double* C, const char* active) {
  for (int e = 0; e < ne; ++e) {
    if (active && !active[e]) continue;
    double a[2], b[2], c[2];
    strain_coeffs_tor(Wn[e], Wn[e + 1], Jr, a, b, c);
    const double Me = Mk[e];
    if (Wn_prev) {
      double ap[2], bp[2], cp[2];
      strain_coeffs_tor(Wn_prev[e], Wn_prev[e + 1], Jr, ap, bp, cp);
      const double denom = 1.0 + 0.5 * Me;
      const double c_old = (1.0 - 0.5 * Me) / denom, w_eps = mu[e] * Me / denom;
      for (int m = 0; m < 2; ++m) {
        A[e * 2 + m] = c_old * A[e * 2 + m] - w_eps * (a[m] + ap[m]);
        B[e * 2 + m] = c_old * B[e * 2 + m] - w_eps * (b[m] + bp[m]);
        C[e * 2 + m] = c_old * C[e * 2 + m] - w_eps * (c[m] + cp[m]);
      }
    } else {
      const double om = 1.0 - Me, two_muM = 2.0 * mu[e] * Me;
      for (int m = 0; m < 2; ++m) {
        A[e * 2 + m] = om * A[e * 2 + m] - two_muM * a[m];
        B[e * 2 + m] = om * B[e * 2 + m] - two_muM * b[m];
        C[e * 2 + m] = om * C[e * 2 + m] - two_muM * c[m];
      }
    }
  }
}

// vilma_response.f90:386-420 response_deg1_to_cm
static void deg1_to_cm(const RadialOp& op, double* x) {
  if (op.nullmode.empty()) return;
  double fa_n = op.nullmode[idx_f(op.nr - 1)];
  if (fa_n == 0.0) return;
  double c = -x[idx_f(op.nr - 1)] / fa_n;
  for (int i = 0; i < op.ndof; ++i) x[i] = x[i] + c * op.nullmode[i];
}

// vilma_response.f90:542-677 response_init_ve
void response_init_ve(Response& R, const Earth& e, const Mesh& m, const Sht& s, double dt) {
  R.lmax = s.lmax;
  R.nlm = s.nlm;
  R.nr = m.nr;
  R.ne = m.ne;
  R.ndof = ndof_of(m.nr);
  R.dt = dt;
  R.time = 0.0;
  R.a = e.r_earth;
  R.g = earth_gravity_at(e, e.r_earth);
  R.r = m.r;
  R.mu.assign(R.ne, 0.0);
  R.Mk.assign(R.ne, 0.0);
  R.MkPerDt.assign(R.ne, 0.0);
  R.active1d.assign(R.ne, 1);
  for (int el = 0; el < R.ne; ++el) {
    const Layer& L = e.layers[m.elem_layer[el]];
    R.mu[el] = L.mu;
    if (L.rheology == RHEOL_MAXWELL) {
      R.Mk[el] = R.mu[el] * dt / L.eta;
      R.MkPerDt[el] = R.mu[el] / L.eta;
    }
  }
  const int L = R.lmax, nr = R.nr;
  R.Jr.assign(L + 1, 0.0);
  R.nrmc.assign((size_t)(L + 1) * 4, 0.0);
  R.sa.assign((size_t)(L + 1) * 16, 0.0);
  R.sb = R.sa;
  R.sc = R.sa;
  R.gu.assign(L + 1, 0.0);
  R.gn.assign(L + 1, 0.0);
  R.gv.assign(L + 1, 0.0);
  R.xUn.assign((size_t)(L + 1) * nr, 0.0);
  R.xVn.assign((size_t)(L + 1) * nr, 0.0);
  R.ops.assign(L + 1, RadialOp());
  R.gn[0] = 4.0 * PI * GRAV_G * R.a / R.g;
  std::vector<double> b(R.ndof), x(R.ndof);
  for (int l = 1; l <= L; ++l) {
    R.Jr[l] = (double)l * (double)(l + 1);
    ve_strain_constants(R.Jr[l], &R.nrmc[l * 4], &R.sa[l * 16], &R.sb[l * 16], &R.sc[l * 16]);
  }
  // an exception may not leave an OpenMP region: the first failing degree's
  // message is kept and rethrown after the loop (the reference stops there)
  std::string first_error;
  int first_error_l = L + 1;
#pragma omp parallel for schedule(dynamic)
  for (int l = 1; l <= L; ++l) {
    try {
      std::vector<double> bb(R.ndof), xx(R.ndof);
      radial_operator_assemble(R.ops[l], e, m, l);
      radial_operator_load_rhs(R.ops[l], 1.0, bb.data());
      radial_operator_solve_vec(R.ops[l], bb.data(), xx.data(), nullptr);
      if (l == 1 && R.deg1_cm) deg1_to_cm(R.ops[l], xx.data());
      R.gu[l] = xx[idx_u(nr - 1)];
      R.gn[l] = -xx[idx_f(nr - 1)] / R.g;
      R.gv[l] = xx[idx_v(nr - 1)];
      for (int node = 0; node < nr; ++node) {
        R.xUn[(size_t)l * nr + node] = xx[idx_u(node)];
        R.xVn[(size_t)l * nr + node] = xx[idx_v(node)];
      }
    } catch (const std::exception& ex) {
#pragma omp critical(orc_operator_error)
      if (l < first_error_l) {
        first_error_l = l;
        first_error = ex.what();
      }
    }
  }
  if (!first_error.empty()) throw std::runtime_error(first_error);
  if (L >= 1 && !R.deg1_cm) R.gn[1] = 0.0;
  // degree-grouped slot map
  R.nk = 0;
  for (int l = 1; l <= L; ++l) R.nk += std::min(l, s.mmax) + 1;
  R.k2lm.assign(R.nk, 0);
  R.kdeg.assign(R.nk, 0);
  R.kbeg.assign(L + 2, 0);
  int k = 0;
  for (int l = 1; l <= L; ++l) {
    R.kbeg[l] = k;
    for (int mm = 0; mm <= std::min(l, s.mmax); ++mm) {
      R.k2lm[k] = s.lmidx(l, mm);
      R.kdeg[k] = l;
      ++k;
    }
  }
  R.kbeg[L + 1] = k;
  const size_t nmem = (size_t)R.nk * R.ne * 4;
  R.Are.assign(nmem, 0.0);
  R.Aim = R.Are;
  R.Bre = R.Are;
  R.Bim = R.Are;
  R.Cre = R.Are;
  R.Cim = R.Are;
  R.dUa.assign(R.nk, 0.0);
  R.dFa = R.dUa;
  R.dVa = R.dUa;
  R.dUn_re.assign((size_t)R.nk * nr, 0.0);
  R.dUn_im = R.dUn_re;
  R.dVn_re = R.dUn_re;
  R.dVn_im = R.dUn_re;
  R.mnorm.assign(R.nk, 0.0);
}

// vilma_response.f90:811-826 absmax6
static double absmax6(int n, const double* x1, const double* x2, const double* x3, const double* x4,
                      const double* x5, const double* x6) {
  double amax = 0.0;
  for (int i = 0; i < n; ++i) {
    amax = std::max(amax, std::fabs(x1[i]));
    amax = std::max(amax, std::fabs(x2[i]));
    amax = std::max(amax, std::fabs(x3[i]));
    amax = std::max(amax, std::fabs(x4[i]));
    amax = std::max(amax, std::fabs(x5[i]));
    amax = std::max(amax, std::fabs(x6[i]));
  }
  return amax;
}

// vilma_response.f90:679-809 solve_drift: the nodal drift into the given
// targets (begin_step: dUn, the endpoint pass: edUn) and the surface drift
// dUa, dFa, dVa (the report drift the sea-level iteration applies)
static void solve_drift(Response& R, std::vector<double>& dUn_re, std::vector<double>& dUn_im,
                        std::vector<double>& dVn_re, std::vector<double>& dVn_im, std::vector<double>* dWn_re,
                        std::vector<double>* dWn_im) {
  const int nb = 4 * R.ne, nr = R.nr, nbt = 2 * R.ne;
  const bool tor = R.nlam > NLAM;
  if (tor && !(dWn_re && dWn_im))
    throw std::runtime_error("solve_drift: the toroidal channels are carried, so W targets are required");
#pragma omp parallel for schedule(static)
  for (int k = 0; k < R.nk; ++k) {
    size_t o = (size_t)k * nb;
    R.mnorm[k] = absmax6(nb, &R.Are[o], &R.Bre[o], &R.Cre[o], &R.Aim[o], &R.Bim[o], &R.Cim[o]);
    if (tor) {  // the (nlam, ne) slot block scanned flat includes lambda 3, 4
      size_t ot = (size_t)k * nbt;
      R.mnorm[k] = std::max(R.mnorm[k], absmax6(nbt, &R.Atre[ot], &R.Btre[ot], &R.Ctre[ot], &R.Atim[ot],
                                                &R.Btim[ot], &R.Ctim[ot]));
    }
  }
  double mx = 0.0;
  for (int k = 0; k < R.nk; ++k) mx = std::max(mx, R.mnorm[k]);
  const double thr = R.skip_tol * mx;
  long solved = 0;
#pragma omp parallel reduction(+ : solved)
  {
    std::vector<double> fre(R.ndof), fim(R.ndof), xre(R.ndof), xim(R.ndof);
    std::vector<double> gre(nr), gim(nr), wre(nr), wim(nr);
#pragma omp for schedule(dynamic)
    for (int l = 1; l <= R.lmax; ++l) {
      for (int k = R.kbeg[l]; k < R.kbeg[l + 1]; ++k) {
        if (R.mnorm[k] <= thr) {
          R.dUa[k] = 0.0;
          R.dFa[k] = 0.0;
          R.dVa[k] = 0.0;
          for (int node = 0; node < nr; ++node) {
            dUn_re[(size_t)k * nr + node] = 0.0;
            dUn_im[(size_t)k * nr + node] = 0.0;
            dVn_re[(size_t)k * nr + node] = 0.0;
            dVn_im[(size_t)k * nr + node] = 0.0;
          }
          if (tor) {
            R.dWa[k] = 0.0;
            for (int node = 0; node < nr; ++node) {
              (*dWn_re)[(size_t)k * nr + node] = 0.0;
              (*dWn_im)[(size_t)k * nr + node] = 0.0;
            }
          }
          continue;
        }
        ++solved;
        std::fill(fre.begin(), fre.end(), 0.0);
        std::fill(fim.begin(), fim.end(), 0.0);
        size_t o = (size_t)k * nb;
        dissipative_rhs(R.ne, R.r.data(), &R.sa[l * 16], &R.sb[l * 16], &R.sc[l * 16], &R.nrmc[l * 4],
                        &R.Are[o], &R.Bre[o], &R.Cre[o], fre.data());
        dissipative_rhs(R.ne, R.r.data(), &R.sa[l * 16], &R.sb[l * 16], &R.sc[l * 16], &R.nrmc[l * 4],
                        &R.Aim[o], &R.Bim[o], &R.Cim[o], fim.data());
        radial_operator_solve_vec(R.ops[l], fre.data(), xre.data(), nullptr);
        radial_operator_solve_vec(R.ops[l], fim.data(), xim.data(), nullptr);
        if (l == 1 && R.deg1_cm) {
          deg1_to_cm(R.ops[l], xre.data());
          deg1_to_cm(R.ops[l], xim.data());
        }
        R.dUa[k] = cplx(xre[idx_u(nr - 1)], xim[idx_u(nr - 1)]);
        R.dFa[k] = cplx(xre[idx_f(nr - 1)], xim[idx_f(nr - 1)]);
        R.dVa[k] = cplx(xre[idx_v(nr - 1)], xim[idx_v(nr - 1)]);
        if (l == 1 && !R.deg1_cm) R.dFa[k] = 0.0;
        for (int node = 0; node < nr; ++node) {
          dUn_re[(size_t)k * nr + node] = xre[idx_u(node)];
          dUn_im[(size_t)k * nr + node] = xim[idx_u(node)];
          dVn_re[(size_t)k * nr + node] = xre[idx_v(node)];
          dVn_im[(size_t)k * nr + node] = xim[idx_v(node)];
        }
        if (tor) {  // its own forcing, its own operator; no frame projection at l = 1
          std::fill(gre.begin(), gre.end(), 0.0);
          std::fill(gim.begin(), gim.end(), 0.0);
          size_t ot = (size_t)k * nbt;
          dissipative_rhs_tor(R.ne, R.r.data(), &R.sat[l * 4], &R.sbt[l * 4], &R.sct[l * 4], &R.nrmt[l * 2],
                              &R.Atre[ot], &R.Btre[ot], &R.Ctre[ot], gre.data());
          dissipative_rhs_tor(R.ne, R.r.data(), &R.sat[l * 4], &R.sbt[l * 4], &R.sct[l * 4], &R.nrmt[l * 2],
                              &R.Atim[ot], &R.Btim[ot], &R.Ctim[ot], gim.data());
          toroidal_operator_solve_vec(R.tops[l], gre.data(), wre.data());
          toroidal_operator_solve_vec(R.tops[l], gim.data(), wim.data());
          for (int node = 0; node < nr; ++node) {
            (*dWn_re)[(size_t)k * nr + node] = wre[node];
            (*dWn_im)[(size_t)k * nr + node] = wim[node];
          }
          R.dWa[k] = cplx(wre[nr - 1], wim[nr - 1]);
        }
      }
    }
  }
  R.n_solved += solved;
  R.n_drift++;
}

// vilma_response.f90:679-809 ve_response_begin: the drift of the entering memory
void response_begin_step(Response& R, const Sht& s) {
  (void)s;
  if (R.nlam > NLAM)
    solve_drift(R, R.dUn_re, R.dUn_im, R.dVn_re, R.dVn_im, &R.dWn_re, &R.dWn_im);
  else
    solve_drift(R, R.dUn_re, R.dUn_im, R.dVn_re, R.dVn_im, nullptr, nullptr);
}

// vilma_response.f90:842-864 ve_response_apply
void response_apply(const Response& R, const Sht& s, const cplx* sigma, cplx* u, cplx* n) {
  for (int lm = 0; lm < s.nlm; ++lm) {
    u[lm] = 0.0;
    n[lm] = 0.0;
  }
  int lm0 = s.lmidx(0, 0);
  u[lm0] = R.gu[0] * sigma[lm0];
  n[lm0] = R.gn[0] * sigma[lm0];
  for (int k = 0; k < R.nk; ++k) {
    int l = R.kdeg[k], lm = R.k2lm[k];
    u[lm] = R.gu[l] * sigma[lm] + R.dUa[k];
    n[lm] = R.gn[l] * sigma[lm] - R.dFa[k] / R.g;
  }
}

// ------------------------------------------------------------- 3-D advance
// vilma_response.f90:1227-1272 gather_tensor_coeffs (spheroidal channels);
// blocks are (4, nlm) channel-major here: c[lam*nlm + lm].
static void gather_tensor_coeffs(const Response& R, const Sht& s, const cplx* sigma, int e, cplx* cma,
                                 cplx* cmb, cplx* cmc, cplx* cea, cplx* ceb, cplx* cec) {
  const int nlm = s.nlm, nr = R.nr;
  for (int t = 0; t < R.nlam * nlm; ++t) cma[t] = cmb[t] = cmc[t] = cea[t] = ceb[t] = cec[t] = 0.0;
  for (int k = 0; k < R.nk; ++k) {
    int l = R.kdeg[k], lm = R.k2lm[k];
    double sre = sigma[lm].real(), sim = sigma[lm].imag();
    const double* xu = &R.xUn[(size_t)l * nr];
    const double* xv = &R.xVn[(size_t)l * nr];
    size_t kn = (size_t)k * nr;
    double Ur = sre * xu[e] + R.dUn_re[kn + e], Ui = sim * xu[e] + R.dUn_im[kn + e];
    double Ur1 = sre * xu[e + 1] + R.dUn_re[kn + e + 1], Ui1 = sim * xu[e + 1] + R.dUn_im[kn + e + 1];
    double Vr = sre * xv[e] + R.dVn_re[kn + e], Vi = sim * xv[e] + R.dVn_im[kn + e];
    double Vr1 = sre * xv[e + 1] + R.dVn_re[kn + e + 1], Vi1 = sim * xv[e + 1] + R.dVn_im[kn + e + 1];
    double ar[4], br[4], cr[4], ai[4], bi[4], ci[4];
    strain_coeffs(Ur, Ur1, Vr, Vr1, R.Jr[l], ar, br, cr);
    strain_coeffs(Ui, Ui1, Vi, Vi1, R.Jr[l], ai, bi, ci);
    size_t o = ((size_t)k * R.ne + e) * 4;
    for (int lam = 0; lam < 4; ++lam) {
      cea[lam * nlm + lm] = cplx(ar[lam], ai[lam]);
      ceb[lam * nlm + lm] = cplx(br[lam], bi[lam]);
      cec[lam * nlm + lm] = cplx(cr[lam], ci[lam]);
      cma[lam * nlm + lm] = cplx(R.Are[o + lam], R.Aim[o + lam]);
      cmb[lam * nlm + lm] = cplx(R.Bre[o + lam], R.Bim[o + lam]);
      cmc[lam * nlm + lm] = cplx(R.Cre[o + lam], R.Cim[o + lam]);
    }
    if (R.nlam == NLAM) continue;
    // channels 4, 5: the lambda 3, 4 memory and the strain of the nodal W drift
    // (no load term: eq 84 does not force W)
    double at[2], bt[2], ct[2], ati[2], bti[2], cti[2];
    strain_coeffs_tor(R.dWn_re[kn + e], R.dWn_re[kn + e + 1], R.Jr[l], at, bt, ct);
    strain_coeffs_tor(R.dWn_im[kn + e], R.dWn_im[kn + e + 1], R.Jr[l], ati, bti, cti);
    size_t ot = ((size_t)k * R.ne + e) * 2;
    for (int lam = 0; lam < 2; ++lam) {
      const size_t c = (size_t)(NLAM + lam) * nlm + lm;
      cea[c] = cplx(at[lam], ati[lam]);
      ceb[c] = cplx(bt[lam], bti[lam]);
      cec[c] = cplx(ct[lam], cti[lam]);
      cma[c] = cplx(R.Atre[ot + lam], R.Atim[ot + lam]);
      cmb[c] = cplx(R.Btre[ot + lam], R.Btim[ot + lam]);
      cmc[c] = cplx(R.Ctre[ot + lam], R.Ctim[ot + lam]);
    }
  }
}

// vilma_response.f90:1274-1319 advance_shape_tensor (increment form)
static void advance_shape_tensor(const Response& R, const Sht& s, int e, cplx* c, const cplx* eps,
                                 double* dtau, double* deps, cplx* cdel) {
  const size_t ng = (size_t)s.nphi * s.nlat;
  double twoMu = 2.0 * R.mu[e];
  tensor_synth(s, c, dtau, R.nlam);
  tensor_synth(s, eps, deps, R.nlam);
  const double* M = &R.Mk3[(size_t)e * ng];
  for (int p = 0; p < 6; ++p)
    for (size_t g = 0; g < ng; ++g) dtau[p * ng + g] = -M[g] * (dtau[p * ng + g] + twoMu * deps[p * ng + g]);
  tensor_analysis(s, dtau, cdel, R.nlam);
  for (int t = 0; t < R.nlam * s.nlm; ++t) c[t] = c[t] + cdel[t];
}

// vilma_response.f90:1171-1225 advance_memory_3d
static void advance_memory_3d(Response& R, const Sht& s, const cplx* sigma) {
  if (R.ne3d == 0) return;
  const int nlm = s.nlm;
  const size_t ng = (size_t)s.nphi * s.nlat;
#pragma omp parallel
  {
    const int nc = R.nlam * nlm;
    std::vector<cplx> cma(nc), cmb(nc), cmc(nc), cea(nc), ceb(nc), cec(nc), cdel(nc);
    std::vector<double> dtau(6 * ng), deps(6 * ng);
#pragma omp for schedule(dynamic)
    for (int ei = 0; ei < R.ne3d; ++ei) {
      int e = R.e3d[ei];
      gather_tensor_coeffs(R, s, sigma, e, cma.data(), cmb.data(), cmc.data(), cea.data(), ceb.data(),
                           cec.data());
      advance_shape_tensor(R, s, e, cma.data(), cea.data(), dtau.data(), deps.data(), cdel.data());
      advance_shape_tensor(R, s, e, cmb.data(), ceb.data(), dtau.data(), deps.data(), cdel.data());
      advance_shape_tensor(R, s, e, cmc.data(), cec.data(), dtau.data(), deps.data(), cdel.data());
      for (int k = 0; k < R.nk; ++k) {
        int lm = R.k2lm[k];
        size_t o = ((size_t)k * R.ne + e) * 4;
        for (int lam = 0; lam < 4; ++lam) {
          R.Are[o + lam] = cma[lam * nlm + lm].real();
          R.Aim[o + lam] = cma[lam * nlm + lm].imag();
          R.Bre[o + lam] = cmb[lam * nlm + lm].real();
          R.Bim[o + lam] = cmb[lam * nlm + lm].imag();
          R.Cre[o + lam] = cmc[lam * nlm + lm].real();
          R.Cim[o + lam] = cmc[lam * nlm + lm].imag();
        }
        if (R.nlam == NLAM) continue;
        size_t ot = ((size_t)k * R.ne + e) * 2;
        for (int lam = 0; lam < 2; ++lam) {
          const size_t c = (size_t)(NLAM + lam) * nlm + lm;
          R.Atre[ot + lam] = cma[c].real();
          R.Atim[ot + lam] = cma[c].imag();
          R.Btre[ot + lam] = cmb[c].real();
          R.Btim[ot + lam] = cmb[c].imag();
          R.Ctre[ot + lam] = cmc[c].real();
          R.Ctim[ot + lam] = cmc[c].imag();
        }
      }
    }
  }
}

// vilma_response.f90:944-992 vilma_advance
void response_advance(Response& R, const Sht& s, const cplx* sigma) {
  if (R.lat_visc) advance_memory_3d(R, s, sigma);
  const int nr = R.nr;
#pragma omp parallel
  {
    std::vector<double> Ure(nr), Uim(nr), Vre(nr), Vim(nr);
#pragma omp for schedule(static)
    for (int k = 0; k < R.nk; ++k) {
      int l = R.kdeg[k], lm = R.k2lm[k];
      double sre = sigma[lm].real(), sim = sigma[lm].imag();
      const double* xu = &R.xUn[(size_t)l * nr];
      const double* xv = &R.xVn[(size_t)l * nr];
      size_t kn = (size_t)k * nr;
      for (int node = 0; node < nr; ++node) {
        Ure[node] = sre * xu[node] + R.dUn_re[kn + node];
        Uim[node] = sim * xu[node] + R.dUn_im[kn + node];
        Vre[node] = sre * xv[node] + R.dVn_re[kn + node];
        Vim[node] = sim * xv[node] + R.dVn_im[kn + node];
      }
      size_t o = (size_t)k * R.ne * 4;
      advance_memory_fe(R.ne, R.mu.data(), R.Mk.data(), Ure.data(), Vre.data(), R.Jr[l], &R.Are[o], &R.Bre[o],
                        &R.Cre[o], R.active1d.data());
      advance_memory_fe(R.ne, R.mu.data(), R.Mk.data(), Uim.data(), Vim.data(), R.Jr[l], &R.Aim[o], &R.Bim[o],
                        &R.Cim[o], R.active1d.data());
      if (R.nlam > NLAM) {  // W is pure drift: no sigma x_Wn term
        size_t ot = (size_t)k * R.ne * 2;
        advance_memory_tor(R.ne, R.mu.data(), R.Mk.data(), &R.dWn_re[kn], nullptr, R.Jr[l], &R.Atre[ot],
                           &R.Btre[ot], &R.Ctre[ot], R.active1d.data());
        advance_memory_tor(R.ne, R.mu.data(), R.Mk.data(), &R.dWn_im[kn], nullptr, R.Jr[l], &R.Atim[ot],
                           &R.Btim[ot], &R.Ctim[ot], R.active1d.data());
      }
    }
  }
  R.n_mem++;
}

// ------------------------------------------------------------- trapezoidal scheme
// vilma_response.f90:1371-1445 gather_tensor_coeffs_trap: tau_n (the *0
// snapshot), eps_n (sigma_n x_Un + dUn) and eps_{n+1} (sigma_{n+1} x_Un + edUn)
// of element e as (4, nlm) channel-major blocks
static void gather_strain_block(const Response& R, const cplx* sigma, const std::vector<double>& dUr,
                                const std::vector<double>& dUi, const std::vector<double>& dVr,
                                const std::vector<double>& dVi, const std::vector<double>& dWr,
                                const std::vector<double>& dWi, int e, cplx* ca, cplx* cb, cplx* cc, int nlm) {
  const int nr = R.nr;
  for (int t = 0; t < R.nlam * nlm; ++t) ca[t] = cb[t] = cc[t] = 0.0;
  for (int k = 0; k < R.nk; ++k) {
    int l = R.kdeg[k], lm = R.k2lm[k];
    double sre = sigma[lm].real(), sim = sigma[lm].imag();
    const double* xu = &R.xUn[(size_t)l * nr];
    const double* xv = &R.xVn[(size_t)l * nr];
    size_t kn = (size_t)k * nr;
    double Ur = sre * xu[e] + dUr[kn + e], Ui = sim * xu[e] + dUi[kn + e];
    double Ur1 = sre * xu[e + 1] + dUr[kn + e + 1], Ui1 = sim * xu[e + 1] + dUi[kn + e + 1];
    double Vr = sre * xv[e] + dVr[kn + e], Vi = sim * xv[e] + dVi[kn + e];
    double Vr1 = sre * xv[e + 1] + dVr[kn + e + 1], Vi1 = sim * xv[e + 1] + dVi[kn + e + 1];
    double ar[4], br[4], cr[4], ai[4], bi[4], ci[4];
    strain_coeffs(Ur, Ur1, Vr, Vr1, R.Jr[l], ar, br, cr);
    strain_coeffs(Ui, Ui1, Vi, Vi1, R.Jr[l], ai, bi, ci);
    for (int lam = 0; lam < 4; ++lam) {
      ca[lam * nlm + lm] = cplx(ar[lam], ai[lam]);
      cb[lam * nlm + lm] = cplx(br[lam], bi[lam]);
      cc[lam * nlm + lm] = cplx(cr[lam], ci[lam]);
    }
    if (R.nlam == NLAM) continue;
    double at[2], bt[2], ct[2], ati[2], bti[2], cti[2];
    strain_coeffs_tor(dWr[kn + e], dWr[kn + e + 1], R.Jr[l], at, bt, ct);
    strain_coeffs_tor(dWi[kn + e], dWi[kn + e + 1], R.Jr[l], ati, bti, cti);
    for (int lam = 0; lam < 2; ++lam) {
      const size_t c = (size_t)(NLAM + lam) * nlm + lm;
      ca[c] = cplx(at[lam], ati[lam]);
      cb[c] = cplx(bt[lam], bti[lam]);
      cc[c] = cplx(ct[lam], cti[lam]);
    }
  }
}

// vilma_response.f90:1447-1478 advance_shape_tensor_trap (increment form):
// tau+ - tau_n = -M [tau_n + mu (eps_n + eps_{n+1})] / (1 + M/2) on the grid
static void advance_shape_tensor_trap(const Response& R, const Sht& s, int e, cplx* c0, const cplx* eps_n,
                                      const cplx* eps_1, double* dt0, double* den, double* de1, cplx* cdel) {
  const size_t ng = (size_t)s.nphi * s.nlat;
  tensor_synth(s, c0, dt0, R.nlam);
  tensor_synth(s, eps_n, den, R.nlam);
  tensor_synth(s, eps_1, de1, R.nlam);
  const double* M = &R.Mk3[(size_t)e * ng];
  for (size_t g = 0; g < ng; ++g) {
    const double wtau = M[g] / (1.0 + 0.5 * M[g]), weps = R.mu[e] * M[g] / (1.0 + 0.5 * M[g]);
    for (int p = 0; p < 6; ++p)
      dt0[p * ng + g] = -wtau * dt0[p * ng + g] - weps * (den[p * ng + g] + de1[p * ng + g]);
  }
  tensor_analysis(s, dt0, cdel, R.nlam);
  for (int t = 0; t < R.nlam * s.nlm; ++t) c0[t] = c0[t] + cdel[t];
}

// vilma_response.f90:1321-1369 advance_memory_3d_trap
static void advance_memory_3d_trap(Response& R, const Sht& s, const cplx* sigma) {
  if (R.ne3d == 0) return;
  const int nlm = s.nlm;
  const size_t ng = (size_t)s.nphi * s.nlat;
  const cplx* sig_n = R.sigma_primed ? R.sigma_n.data() : sigma;  // first step: sigma_{n+1} (:1398-1403)
#pragma omp parallel
  {
    const int nc = R.nlam * nlm;
    std::vector<cplx> c0[3], cn[3], c1[3];
    for (int q = 0; q < 3; ++q) {
      c0[q].assign(nc, 0.0);
      cn[q].assign(nc, 0.0);
      c1[q].assign(nc, 0.0);
    }
    std::vector<cplx> cdel(nc);
    std::vector<double> dt0(6 * ng), den(6 * ng), de1(6 * ng);
#pragma omp for schedule(dynamic)
    for (int ei = 0; ei < R.ne3d; ++ei) {
      const int e = R.e3d[ei];
      for (int q = 0; q < 3; ++q) std::fill(c0[q].begin(), c0[q].end(), cplx(0.0));
      for (int k = 0; k < R.nk; ++k) {
        const int lm = R.k2lm[k];
        const size_t o = ((size_t)k * R.ne + e) * 4;
        for (int lam = 0; lam < 4; ++lam) {
          c0[0][lam * nlm + lm] = cplx(R.Are0[o + lam], R.Aim0[o + lam]);
          c0[1][lam * nlm + lm] = cplx(R.Bre0[o + lam], R.Bim0[o + lam]);
          c0[2][lam * nlm + lm] = cplx(R.Cre0[o + lam], R.Cim0[o + lam]);
        }
        if (R.nlam == NLAM) continue;
        const size_t ot = ((size_t)k * R.ne + e) * 2;
        for (int lam = 0; lam < 2; ++lam) {
          const size_t c = (size_t)(NLAM + lam) * nlm + lm;
          c0[0][c] = cplx(R.Atre0[ot + lam], R.Atim0[ot + lam]);
          c0[1][c] = cplx(R.Btre0[ot + lam], R.Btim0[ot + lam]);
          c0[2][c] = cplx(R.Ctre0[ot + lam], R.Ctim0[ot + lam]);
        }
      }
      gather_strain_block(R, sig_n, R.dUn_re, R.dUn_im, R.dVn_re, R.dVn_im, R.dWn_re, R.dWn_im, e, cn[0].data(),
                          cn[1].data(), cn[2].data(), nlm);
      gather_strain_block(R, sigma, R.edUn_re, R.edUn_im, R.edVn_re, R.edVn_im, R.edWn_re, R.edWn_im, e,
                          c1[0].data(), c1[1].data(), c1[2].data(), nlm);
      for (int q = 0; q < 3; ++q)
        advance_shape_tensor_trap(R, s, e, c0[q].data(), cn[q].data(), c1[q].data(), dt0.data(), den.data(),
                                  de1.data(), cdel.data());
      for (int k = 0; k < R.nk; ++k) {
        const int lm = R.k2lm[k];
        const size_t o = ((size_t)k * R.ne + e) * 4;
        for (int lam = 0; lam < 4; ++lam) {
          R.Are[o + lam] = c0[0][lam * nlm + lm].real();
          R.Aim[o + lam] = c0[0][lam * nlm + lm].imag();
          R.Bre[o + lam] = c0[1][lam * nlm + lm].real();
          R.Bim[o + lam] = c0[1][lam * nlm + lm].imag();
          R.Cre[o + lam] = c0[2][lam * nlm + lm].real();
          R.Cim[o + lam] = c0[2][lam * nlm + lm].imag();
        }
        if (R.nlam == NLAM) continue;
        const size_t ot = ((size_t)k * R.ne + e) * 2;
        for (int lam = 0; lam < 2; ++lam) {
          const size_t c = (size_t)(NLAM + lam) * nlm + lm;
          R.Atre[ot + lam] = c0[0][c].real();
          R.Atim[ot + lam] = c0[0][c].imag();
          R.Btre[ot + lam] = c0[1][c].real();
          R.Btim[ot + lam] = c0[1][c].imag();
          R.Ctre[ot + lam] = c0[2][c].real();
          R.Ctim[ot + lam] = c0[2][c].imag();
        }
      }
    }
  }
}

// vilma_response.f90:1524-1596 trapezoid_advance_all: reset to tau_n, advance
// the 1-D-effective elements with (eps_n, eps_{n+1}), then the 3-D ones
static void trapezoid_advance_all(Response& R, const Sht& s, const cplx* sigma) {
  const int nr = R.nr;
#pragma omp parallel
  {
    std::vector<double> Ure(nr), Uim(nr), Vre(nr), Vim(nr), Urn(nr), Uin(nr), Vrn(nr), Vin(nr);
#pragma omp for schedule(static)
    for (int k = 0; k < R.nk; ++k) {
      const int l = R.kdeg[k], lm = R.k2lm[k];
      const double sre = sigma[lm].real(), sim = sigma[lm].imag();
      const double srn = R.sigma_primed ? R.sigma_n[lm].real() : sre;
      const double sin_ = R.sigma_primed ? R.sigma_n[lm].imag() : sim;
      const double* xu = &R.xUn[(size_t)l * nr];
      const double* xv = &R.xVn[(size_t)l * nr];
      const size_t kn = (size_t)k * nr;
      for (int node = 0; node < nr; ++node) {
        Urn[node] = srn * xu[node] + R.dUn_re[kn + node];
        Vrn[node] = srn * xv[node] + R.dVn_re[kn + node];
        Uin[node] = sin_ * xu[node] + R.dUn_im[kn + node];
        Vin[node] = sin_ * xv[node] + R.dVn_im[kn + node];
        Ure[node] = sre * xu[node] + R.edUn_re[kn + node];
        Vre[node] = sre * xv[node] + R.edVn_re[kn + node];
        Uim[node] = sim * xu[node] + R.edUn_im[kn + node];
        Vim[node] = sim * xv[node] + R.edVn_im[kn + node];
      }
      const size_t o = (size_t)k * R.ne * 4, n4 = (size_t)R.ne * 4;
      std::copy(&R.Are0[o], &R.Are0[o] + n4, &R.Are[o]);
      std::copy(&R.Bre0[o], &R.Bre0[o] + n4, &R.Bre[o]);
      std::copy(&R.Cre0[o], &R.Cre0[o] + n4, &R.Cre[o]);
      std::copy(&R.Aim0[o], &R.Aim0[o] + n4, &R.Aim[o]);
      std::copy(&R.Bim0[o], &R.Bim0[o] + n4, &R.Bim[o]);
      std::copy(&R.Cim0[o], &R.Cim0[o] + n4, &R.Cim[o]);
      advance_memory_trap(R.ne, R.mu.data(), R.Mk.data(), Ure.data(), Vre.data(), Urn.data(), Vrn.data(), R.Jr[l],
                          &R.Are[o], &R.Bre[o], &R.Cre[o], R.active1d.data());
      advance_memory_trap(R.ne, R.mu.data(), R.Mk.data(), Uim.data(), Vim.data(), Uin.data(), Vin.data(), R.Jr[l],
                          &R.Aim[o], &R.Bim[o], &R.Cim[o], R.active1d.data());
      if (R.nlam > NLAM) {  // W: eps_n from tau_n's drift, eps_{n+1} from the endpoint's
        const size_t ot = (size_t)k * R.ne * 2, n2 = (size_t)R.ne * 2;
        std::copy(&R.Atre0[ot], &R.Atre0[ot] + n2, &R.Atre[ot]);
        std::copy(&R.Btre0[ot], &R.Btre0[ot] + n2, &R.Btre[ot]);
        std::copy(&R.Ctre0[ot], &R.Ctre0[ot] + n2, &R.Ctre[ot]);
        std::copy(&R.Atim0[ot], &R.Atim0[ot] + n2, &R.Atim[ot]);
        std::copy(&R.Btim0[ot], &R.Btim0[ot] + n2, &R.Btim[ot]);
        std::copy(&R.Ctim0[ot], &R.Ctim0[ot] + n2, &R.Ctim[ot]);
        advance_memory_tor(R.ne, R.mu.data(), R.Mk.data(), &R.edWn_re[kn], &R.dWn_re[kn], R.Jr[l], &R.Atre[ot],
                           &R.Btre[ot], &R.Ctre[ot], R.active1d.data());
        advance_memory_tor(R.ne, R.mu.data(), R.Mk.data(), &R.edWn_im[kn], &R.dWn_im[kn], R.Jr[l], &R.Atim[ot],
                           &R.Btim[ot], &R.Ctim[ot], R.active1d.data());
      }
    }
  }
  if (R.lat_visc) advance_memory_3d_trap(R, s, sigma);
  R.n_mem++;
}

// vilma_response.f90:1598-1616 ve_response_prepare_endpoint
void response_prepare_endpoint(Response& R) {
  R.couple_pass = 0;
  R.couple_done = false;
  if (R.scheme != SCHEME_TRAP) return;
  R.Are0 = R.Are;  // snapshot_taun (:1514-1522)
  R.Aim0 = R.Aim;
  R.Bre0 = R.Bre;
  R.Bim0 = R.Bim;
  R.Cre0 = R.Cre;
  R.Cim0 = R.Cim;
  R.edUn_re = R.dUn_re;
  R.edUn_im = R.dUn_im;
  R.edVn_re = R.dVn_re;
  R.edVn_im = R.dVn_im;
  R.dUa_prev = R.dUa;  // keep_drift (:1492-1497)
  if (R.nlam > NLAM) {
    R.Atre0 = R.Atre;
    R.Atim0 = R.Atim;
    R.Btre0 = R.Btre;
    R.Btim0 = R.Btim;
    R.Ctre0 = R.Ctre;
    R.Ctim0 = R.Ctim;
    R.edWn_re = R.dWn_re;
    R.edWn_im = R.dWn_im;
    R.dWa_prev = R.dWa;
  }
}

// vilma_response.f90:1618-1646 ve_response_advance_endpoint
void response_advance_endpoint(Response& R, const Sht& s, const cplx* sigma) {
  if (R.scheme != SCHEME_TRAP) {
    response_advance(R, s, sigma);
    R.couple_pass = 1;
    R.couple_done = true;
    return;
  }
  trapezoid_advance_all(R, s, sigma);
  R.sigma_next.assign(sigma, sigma + R.nlm);
  const bool tor = R.nlam > NLAM;
  solve_drift(R, R.edUn_re, R.edUn_im, R.edVn_re, R.edVn_im, tor ? &R.edWn_re : nullptr,
              tor ? &R.edWn_im : nullptr);  // solve_endpoint_drift (:1480-1490)
  R.couple_pass++;
  double cnorm = 0.0, snorm = 0.0;  // drift_change (:1499-1512)
  for (int k = 0; k < R.nk; ++k) {
    cnorm = std::max(cnorm, std::abs(R.dUa[k] - R.dUa_prev[k]));
    snorm = std::max(snorm, std::abs(R.dUa[k]));
  }
  if (tor)
    for (int k = 0; k < R.nk; ++k) {
      cnorm = std::max(cnorm, std::abs(R.dWa[k] - R.dWa_prev[k]));
      snorm = std::max(snorm, std::abs(R.dWa[k]));
    }
  R.dUa_prev = R.dUa;
  if (tor) R.dWa_prev = R.dWa;
  R.couple_done = (R.couple_pass >= 2 && cnorm <= R.couple_tol * std::max(snorm, 2.2250738585072014e-308));
}

// vilma_response.f90:1648-1651
bool response_endpoint_converged(const Response& R) { return R.couple_done; }

// vilma_response.f90:1653-1663 ve_response_finalize_step
void response_finalize_step(Response& R) {
  R.couple_iters_last = R.couple_pass;
  if (!R.sigma_next.empty()) {
    R.sigma_n = R.sigma_next;
    R.sigma_primed = true;
  }
  R.time += R.dt;
}

// response_prime_sigma: the start-of-step load sigma_n
void response_prime_sigma(Response& R, const cplx* sig0) {
  R.sigma_n.assign(sig0, sig0 + R.nlm);
  R.sigma_primed = true;
}

// vilma_response.f90:1695-1740 response_save_state / response_restore_state
void response_save_state(Response& R) {
  R.Are_s = R.Are;
  R.Aim_s = R.Aim;
  R.Bre_s = R.Bre;
  R.Bim_s = R.Bim;
  R.Cre_s = R.Cre;
  R.Cim_s = R.Cim;
  R.time_s = R.time;
  R.sigma_n_s = R.sigma_n;
  R.sigma_primed_s = R.sigma_primed;
  if (R.nlam > NLAM) {
    R.Atre_s = R.Atre;
    R.Atim_s = R.Atim;
    R.Btre_s = R.Btre;
    R.Btim_s = R.Btim;
    R.Ctre_s = R.Ctre;
    R.Ctim_s = R.Ctim;
  }
}
void response_restore_state(Response& R) {
  R.Are = R.Are_s;
  R.Aim = R.Aim_s;
  R.Bre = R.Bre_s;
  R.Bim = R.Bim_s;
  R.Cre = R.Cre_s;
  R.Cim = R.Cim_s;
  R.time = R.time_s;
  R.sigma_n = R.sigma_n_s;
  R.sigma_primed = R.sigma_primed_s;
  if (R.nlam > NLAM) {
    R.Atre = R.Atre_s;
    R.Atim = R.Atim_s;
    R.Btre = R.Btre_s;
    R.Btim = R.Btim_s;
    R.Ctre = R.Ctre_s;
    R.Ctim = R.Ctim_s;
  }
}

// vilma_response.f90:1742-1758 response_stash_coarse
void response_stash_coarse(Response& R) {
  R.Are_c = R.Are;
  R.Aim_c = R.Aim;
  R.Bre_c = R.Bre;
  R.Bim_c = R.Bim;
  R.Cre_c = R.Cre;
  R.Cim_c = R.Cim;
  if (R.nlam > NLAM) {
    R.Atre_c = R.Atre;
    R.Atim_c = R.Atim;
    R.Btre_c = R.Btre;
    R.Btim_c = R.Btim;
    R.Ctre_c = R.Ctre;
    R.Ctim_c = R.Ctim;
  }
}

// vilma_response.f90:1760-1781 response_coarse_fine_error: max |tau_fine - tau_coarse|, max |tau_fine|
void response_coarse_fine_error(const Response& R, double& err_inf, double& tau_inf) {
  err_inf = 0.0;
  tau_inf = 0.0;
  const std::vector<double>* f[6] = {&R.Are, &R.Aim, &R.Bre, &R.Bim, &R.Cre, &R.Cim};
  const std::vector<double>* c[6] = {&R.Are_c, &R.Aim_c, &R.Bre_c, &R.Bim_c, &R.Cre_c, &R.Cim_c};
  for (int q = 0; q < 6; ++q)
    for (size_t i = 0; i < f[q]->size(); ++i) {
      err_inf = std::max(err_inf, std::fabs((*f[q])[i] - (*c[q])[i]));
      tau_inf = std::max(tau_inf, std::fabs((*f[q])[i]));
    }
  if (R.nlam == NLAM) return;
  const std::vector<double>* ft[6] = {&R.Atre, &R.Atim, &R.Btre, &R.Btim, &R.Ctre, &R.Ctim};
  const std::vector<double>* ct[6] = {&R.Atre_c, &R.Atim_c, &R.Btre_c, &R.Btim_c, &R.Ctre_c, &R.Ctim_c};
  for (int q = 0; q < 6; ++q)
    for (size_t i = 0; i < ft[q]->size(); ++i) {
      err_inf = std::max(err_inf, std::fabs((*ft[q])[i] - (*ct[q])[i]));
      tau_inf = std::max(tau_inf, std::fabs((*ft[q])[i]));
    }
}

// vilma_response.f90:1665-1680 response_set_dt
void response_set_dt(Response& R, double dt) {
  R.dt = dt;
  for (int e = 0; e < R.ne; ++e) R.Mk[e] = R.MkPerDt[e] * dt;
  if (R.lat_visc)
    for (size_t g = 0; g < R.Mk3.size(); ++g) R.Mk3[g] = R.MkPerDt3[g] * dt;
}

// vilma_response.f90:1783-1793
double response_max_rate(const Response& R) {
  double rate = 0.0;
  for (double v : R.MkPerDt) rate = std::max(rate, v);
  if (R.lat_visc)
    for (double v : R.MkPerDt3) rate = std::max(rate, v);
  return rate;
}

// vilma_response.f90:1795-1811. The guard that reads this norm treats it as
// non-finite for a NaN memory (vilma_timestep.f90:204, "finite = (err_inf <=
// huge(1.0_wp)) ! .false. for NaN / +Inf"); Fortran leaves MAX with a NaN
// argument to the processor, so the scan propagates NaN explicitly to keep
// that stated meaning (finite values: the same maximum as absmax6).
static inline double nan_max(double a, double b) { return (a != a || b != b) ? a + b : std::max(a, b); }

static double absmax6_nan(int n, const double* x1, const double* x2, const double* x3, const double* x4,
                          const double* x5, const double* x6) {
  double amax = 0.0;
  for (int i = 0; i < n; ++i) {
    amax = nan_max(amax, std::fabs(x1[i]));
    amax = nan_max(amax, std::fabs(x2[i]));
    amax = nan_max(amax, std::fabs(x3[i]));
    amax = nan_max(amax, std::fabs(x4[i]));
    amax = nan_max(amax, std::fabs(x5[i]));
    amax = nan_max(amax, std::fabs(x6[i]));
  }
  return amax;
}

double response_memory_norm(const Response& R) {
  const int nb = 4 * R.ne;
  std::vector<double> part((size_t)R.nk, 0.0);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < R.nk; ++k) {
    size_t o = (size_t)k * nb;
    part[k] = absmax6_nan(nb, &R.Are[o], &R.Aim[o], &R.Bre[o], &R.Bim[o], &R.Cre[o], &R.Cim[o]);
  }
  double nrm = 0.0;
  for (int k = 0; k < R.nk; ++k) nrm = nan_max(nrm, part[k]);
  if (R.nlam > NLAM) {
    const int nbt = 2 * R.ne;
    for (int k = 0; k < R.nk; ++k) {
      size_t o = (size_t)k * nbt;
      nrm = nan_max(nrm, absmax6_nan(nbt, &R.Atre[o], &R.Atim[o], &R.Btre[o], &R.Btim[o], &R.Ctre[o], &R.Ctim[o]));
    }
  }
  return nrm;
}

// vilma_response.f90:994-1053 response_enable_lateral_visc (spheroidal channels)
void response_enable_lateral_visc(Response& R, const Sht& s, const double* pert) {
  const size_t ng = (size_t)s.nphi * s.nlat;
  R.MkPerDt3.assign(ng * R.ne, 0.0);
  R.Mk3.assign(ng * R.ne, 0.0);
  R.pert_mean3d.clear();
  for (int e = 0; e < R.ne; ++e)
    for (size_t g = 0; g < ng; ++g) R.MkPerDt3[e * ng + g] = R.MkPerDt[e] * std::pow(10.0, -pert[e * ng + g]);
  std::fill(R.active1d.begin(), R.active1d.end(), 1);
  R.ne3d = 0;
  for (int e = 0; e < R.ne; ++e) {
    if (R.MkPerDt[e] == 0.0) continue;
    double mx = -1e300, mn = 1e300, sum = 0.0;
    for (size_t g = 0; g < ng; ++g) {
      mx = std::max(mx, pert[e * ng + g]);
      mn = std::min(mn, pert[e * ng + g]);
    }
    if (mx - mn > R.visc3d_tol) {
      R.active1d[e] = 0;
      R.ne3d++;
      for (size_t g = 0; g < ng; ++g) sum += pert[e * ng + g];
      R.pert_mean3d.push_back(sum / (double)ng);
    } else {
      for (size_t g = 0; g < ng; ++g) sum += pert[e * ng + g];
      double mean_pert = sum / (double)ng;
      R.MkPerDt[e] = R.MkPerDt[e] * std::pow(10.0, -mean_pert);
    }
  }
  for (int e = 0; e < R.ne; ++e) R.Mk[e] = R.MkPerDt[e] * R.dt;
  for (size_t g = 0; g < R.Mk3.size(); ++g) R.Mk3[g] = R.MkPerDt3[g] * R.dt;
  R.e3d.clear();
  for (int e = 0; e < R.ne; ++e)
    if (!R.active1d[e]) R.e3d.push_back(e);
  R.ne3d = (int)R.e3d.size();
  R.lat_visc = true;
  // a genuinely 3-D element couples spheroidal and toroidal (:1048-1052)
  if (R.toroidal && R.ne3d > 0 && R.nlam == NLAM) response_enable_toroidal(R);
}

// vilma_response.f90:1055-1118 enable_toroidal: per-degree W operators and
// constants, the W drift arrays and the toroidal memory, zero
void response_enable_toroidal(Response& R) {
  R.tops.assign(R.lmax + 1, TorOp());
  R.nrmt.assign((size_t)(R.lmax + 1) * 2, 0.0);
  R.sat.assign((size_t)(R.lmax + 1) * 4, 0.0);
  R.sbt = R.sat;
  R.sct = R.sat;
  for (int l = 1; l <= R.lmax; ++l) {
    toroidal_operator_assemble(R.tops[l], R.r, R.mu, l);
    ve_strain_constants_tor(R.Jr[l], &R.nrmt[l * 2], &R.sat[l * 4], &R.sbt[l * 4], &R.sct[l * 4]);
  }
  R.dWa.assign(R.nk, 0.0);
  R.dWa_prev = R.dWa;
  R.dWn_re.assign((size_t)R.nk * R.nr, 0.0);
  R.dWn_im = R.dWn_re;
  R.edWn_re = R.dWn_re;
  R.edWn_im = R.dWn_re;
  R.Atre.assign((size_t)R.nk * R.ne * 2, 0.0);
  R.Atim = R.Atre;
  R.Btre = R.Atre;
  R.Btim = R.Atre;
  R.Ctre = R.Atre;
  R.Ctim = R.Atre;
  R.nlam = NLAM + NLAM_TOR;
}

}  // namespace orc

// ================================================================ rotation
// vilma_rotation.f90 (CPU restatement). JROT = 2 throughout.

namespace orc {

// vilma_rotation.f90:375-433 channel_init
static void channel_init(Deg2Channel& c, const Earth& e, const Mesh& m, double dt, bool tidal) {
  c = Deg2Channel();
  c.tidal = tidal;
  c.nr = m.nr;
  c.ne = m.ne;
  c.ndof = ndof_of(m.nr);
  c.Jr = 6.0;
  c.dt = dt;
  c.r = m.r;
  c.mu.assign(c.ne, 0.0);
  c.MkPerDt.assign(c.ne, 0.0);
  c.Mk.assign(c.ne, 0.0);
  for (int k = 0; k < c.ne; ++k) {
    const Layer& L = e.layers[m.elem_layer[k]];
    c.mu[k] = L.mu;
    c.MkPerDt[k] = L.eta > 0.0 ? c.mu[k] / L.eta : 0.0;
    c.Mk[k] = c.MkPerDt[k] * dt;
  }
  ve_strain_constants(c.Jr, c.norm, c.sa, c.sb, c.sc);
  radial_operator_assemble(c.op, e, m, 2);
  std::vector<double> b(c.ndof), x(c.ndof);
  if (tidal)
    radial_operator_tidal_rhs(c.op, 1.0, b.data());
  else
    radial_operator_load_rhs(c.op, 1.0, b.data());
  radial_operator_solve_vec(c.op, b.data(), x.data(), nullptr);
  c.Fe = x[idx_f(c.nr - 1)];
  c.Ue = x[idx_u(c.nr - 1)];
  c.xUn.resize(c.nr);
  c.xVn.resize(c.nr);
  for (int k = 0; k < c.nr; ++k) {
    c.xUn[k] = x[idx_u(k)];
    c.xVn[k] = x[idx_v(k)];
  }
  for (auto* v : {&c.Are, &c.Aim, &c.Bre, &c.Bim, &c.Cre, &c.Cim}) v->assign((size_t)NLAM * c.ne, 0.0);
  for (auto* v : {&c.dUn_re, &c.dUn_im, &c.dVn_re, &c.dVn_im}) v->assign(c.nr, 0.0);
  c.dF = 0.0;
  c.dU = 0.0;
}

// vilma_rotation.f90:435-440
static void channel_set_dt(Deg2Channel& c, double dt) {
  c.dt = dt;
  for (int k = 0; k < c.ne; ++k) c.Mk[k] = c.MkPerDt[k] * dt;
}

// vilma_rotation.f90:442-463 channel_begin: drift frozen from the entering memory
static void channel_begin(Deg2Channel& c) {
  std::vector<double> fre(c.ndof, 0.0), fim(c.ndof, 0.0), xre(c.ndof), xim(c.ndof);
  dissipative_rhs(c.ne, c.r.data(), c.sa, c.sb, c.sc, c.norm, c.Are.data(), c.Bre.data(), c.Cre.data(), fre.data());
  dissipative_rhs(c.ne, c.r.data(), c.sa, c.sb, c.sc, c.norm, c.Aim.data(), c.Bim.data(), c.Cim.data(), fim.data());
  radial_operator_solve_vec(c.op, fre.data(), xre.data(), nullptr);
  radial_operator_solve_vec(c.op, fim.data(), xim.data(), nullptr);
  c.dF = cplx(xre[idx_f(c.nr - 1)], xim[idx_f(c.nr - 1)]);
  c.dU = cplx(xre[idx_u(c.nr - 1)], xim[idx_u(c.nr - 1)]);
  for (int k = 0; k < c.nr; ++k) {
    c.dUn_re[k] = xre[idx_u(k)];
    c.dUn_im[k] = xim[idx_u(k)];
    c.dVn_re[k] = xre[idx_v(k)];
    c.dVn_im[k] = xim[idx_v(k)];
  }
}

// vilma_rotation.f90:465-485 channel_commit: forward-Euler memory with the converged forcing
static void channel_commit(Deg2Channel& c, cplx coeff) {
  std::vector<double> Ure(c.nr), Uim(c.nr), Vre(c.nr), Vim(c.nr);
  const double cr = coeff.real(), ci = coeff.imag();
  for (int k = 0; k < c.nr; ++k) {
    Ure[k] = cr * c.xUn[k] + c.dUn_re[k];
    Uim[k] = ci * c.xUn[k] + c.dUn_im[k];
    Vre[k] = cr * c.xVn[k] + c.dVn_re[k];
    Vim[k] = ci * c.xVn[k] + c.dVn_im[k];
  }
  advance_memory_fe(c.ne, c.mu.data(), c.Mk.data(), Ure.data(), Vre.data(), c.Jr, c.Are.data(), c.Bre.data(),
                    c.Cre.data(), nullptr);
  advance_memory_fe(c.ne, c.mu.data(), c.Mk.data(), Uim.data(), Vim.data(), c.Jr, c.Aim.data(), c.Bim.data(),
                    c.Cim.data(), nullptr);
}

// vilma_rotation.f90:342-371 fluid_tidal_k: elastic tidal solve with every Maxwell
// layer fluidised (elastic lithosphere and fluid core unchanged)
static double fluid_tidal_k(const Earth& e, const Mesh& m) {
  Earth ef = e;
  for (auto& L : ef.layers)
    if (L.rheology == RHEOL_MAXWELL) {
      L.mu = 0.0;
      L.rheology = RHEOL_FLUID;
    }
  RadialOp op;
  radial_operator_assemble(op, ef, m, 2);
  std::vector<double> b(op.ndof), x(op.ndof);
  radial_operator_tidal_rhs(op, 1.0, b.data());
  radial_operator_solve_vec(op, b.data(), x.data(), nullptr);
  return -x[idx_f(m.nr - 1)] / 1.0 - 1.0;  // tidal_love, vilma_radial_fe.f90:868-893
}

// vilma_rotation.f90:114-152 rotation_init
void rotation_init(Rotation& rt, const Earth& e, const Mesh& m, double dt) {
  rt = Rotation();
  rt.a = e.r_earth;
  rt.g = earth_gravity_at(e, e.r_earth);
  channel_init(rt.load_ch, e, m, dt, false);
  channel_init(rt.tidal_ch, e, m, dt, true);
  rt.kTe = -rt.tidal_ch.Fe - 1.0;
  rt.hTe = earth_gravity_at(e, e.r_earth) * rt.tidal_ch.Ue;
  rt.k_s_fluid = fluid_tidal_k(e, m);
  rt.k_s_flat = 3.0 * GRAV_G * rt.CminusA / (std::pow(rt.a, 5) * rt.Omega * rt.Omega);
  double mx = 0.0;
  for (double v : rt.load_ch.MkPerDt) mx = std::max(mx, v);
  if (mx > 0.0) rt.dt_fe_max = 1.0 / mx;
  rt.k_s = rt.k_s_fluid;
  rt.m = 0.0;
  rt.time = 0.0;
  rt.enabled = true;
}

// vilma_rotation.f90:154-168
void rotation_begin_step(Rotation& rt, double dt) {
  if (!rt.enabled) return;
  if (dt != rt.load_ch.dt) {
    channel_set_dt(rt.load_ch, dt);
    channel_set_dt(rt.tidal_ch, dt);
  }
  channel_begin(rt.load_ch);
  channel_begin(rt.tidal_ch);
}

// vilma_rotation.f90:315-338 inertia21: I13 + i I23 of a surface load by Gauss-grid quadrature
cplx inertia21(const Sht& s, const double* load, double a) {
  const int np = s.nphi, nl = s.nlat;
  std::vector<double> w13((size_t)np * nl), w23((size_t)np * nl);
  for (int j = 0; j < nl; ++j) {
    const double st = std::sin(s.colat[j]), ct = std::cos(s.colat[j]), sc2 = st * ct;
    for (int i = 0; i < np; ++i) {
      const double lon = 2.0 * PI * (double)i / (double)np;
      w13[(size_t)j * np + i] = load[(size_t)j * np + i] * sc2 * std::cos(lon);
      w23[(size_t)j * np + i] = load[(size_t)j * np + i] * sc2 * std::sin(lon);
    }
  }
  const double a4 = std::pow(a, 4);
  return cplx(-a4 * sht_surface_integral(s, w13.data()), -a4 * sht_surface_integral(s, w23.data()));
}

// vilma_rotation.f90:170-190 rotation_solve_m
void rotation_solve_m(Rotation& rt, const Sht& s, const double* load) {
  if (!rt.enabled) return;
  const cplx Irig = inertia21(s, load, rt.a);
  const double scl = 5.0 / (4.0 * PI * GRAV_G * rt.a);
  rt.cload = Irig * scl;
  const cplx Itot = -(rt.load_ch.Fe * rt.cload + rt.load_ch.dF);
  const cplx psiL = Itot / rt.CminusA;
  rt.m = (psiL - rt.tidal_ch.dF / rt.k_s) / (1.0 - rt.kTe / rt.k_s);
}

// vilma_rotation.f90:192-222 rotation_s_rot: s_rot = N_rot - u_rot on the Gauss grid
void rotation_s_rot(const Rotation& rt, const Sht& s, double* srot) {
  const int np = s.nphi, nl = s.nlat;
  if (!rt.enabled) {
    for (size_t i = 0; i < (size_t)np * nl; ++i) srot[i] = 0.0;
    return;
  }
  const cplx cN = rt.m + (rt.kTe * rt.m - rt.tidal_ch.dF);
  const cplx cU = rt.tidal_ch.Ue * rt.m + rt.tidal_ch.dU;
  const double kN = rt.Omega * rt.Omega * rt.a * rt.a / rt.g;
  const double ku = rt.Omega * rt.Omega * rt.a * rt.a;
  for (int j = 0; j < nl; ++j) {
    const double gam = std::sin(s.colat[j]) * std::cos(s.colat[j]);
    for (int i = 0; i < np; ++i) {
      const double lon = 2.0 * PI * (double)i / (double)np;
      const double cphi = std::cos(lon), sphi = std::sin(lon);
      srot[(size_t)j * np + i] = gam * (kN * (cN.real() * cphi + cN.imag() * sphi) -
                                        ku * (cU.real() * cphi + cU.imag() * sphi));
    }
  }
}

// vilma_rotation.f90:224-233
void rotation_commit(Rotation& rt) {
  if (!rt.enabled) return;
  channel_commit(rt.load_ch, rt.cload);
  channel_commit(rt.tidal_ch, rt.m);
  rt.time += rt.load_ch.dt;
}

// vilma_rotation.f90:235-249
void rotation_update(Rotation& rt, const Sht& s, const double* load, double dt) {
  if (!rt.enabled) return;
  rotation_begin_step(rt, dt);
  rotation_solve_m(rt, s, load);
  rotation_commit(rt);
}

}  // namespace orc
