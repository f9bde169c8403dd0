// CPU ORACLE — test infrastructure only (see orc.hpp).
// Earth structure, radial P1/P0 mesh, closed-form element integrals, per-degree
// saddle-point assembly, geometric-mean equilibration with an optional KKT
// border, and the LAPACK-dgbtf2/dgbtrs-order banded LU.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "orc.hpp"

namespace orc {

// vilma_earth_structure.f90 earth_mass_below / earth_gravity_at / earth_moi
double earth_mass_below(const Earth& e, double r) {
  double m = 0.0;
  for (const Layer& L : e.layers) {
    double lo = L.r_bot, hi = std::min(L.r_top, r);
    if (hi > lo) m += (4.0 / 3.0) * PI * L.rho * (hi * hi * hi - lo * lo * lo);
  }
  return m;
}
double earth_gravity_at(const Earth& e, double r) {
  if (r > 0.0) return GRAV_G * earth_mass_below(e, r) / (r * r);
  return 0.0;
}
double earth_moi(const Earth& e) {
  double I = 0.0;
  for (const Layer& L : e.layers)
    I += (8.0 * PI / 15.0) * L.rho * (std::pow(L.r_top, 5) - std::pow(L.r_bot, 5));
  return I;
}

// src/vilma_earth_structure.f90:220-238 build_M3L70V01 (Spada et al. 2011, Table 3)
Earth build_M3L70V01() {
  const double km = 1e3;
  Earth e;
  e.r_earth = 6371.0 * km;
  e.layers = {
      {6301.0 * km, 6371.0 * km, 3037.0, 5.0605e10, 1e300, RHEOL_ELASTIC},
      {5951.0 * km, 6301.0 * km, 3438.0, 7.0363e10, 1.0e21, RHEOL_MAXWELL},
      {5701.0 * km, 5951.0 * km, 3871.0, 1.0549e11, 1.0e21, RHEOL_MAXWELL},
      {3480.0 * km, 5701.0 * km, 4978.0, 2.2834e11, 2.0e21, RHEOL_MAXWELL},
      {0.0, 3480.0 * km, 10750.0, 0.0, 0.0, RHEOL_FLUID},
  };
  return e;
}

// vilma_radial_fe.f90:140-151 dr_target (VEGA spacing)
static double dr_target(double depth) {
  if (depth <= 70.0e3) return 5.0e3;
  if (depth <= 670.0e3) return 10.0e3;
  return 40.0e3;
}

// vilma_radial_fe.f90:153-224 radial_mesh_build. The optional per-layer count
// replaces the depth rule (the reference has no such knob).
Mesh radial_mesh_build(const Earth& e, const int* ne_layer) {
  const int nl = (int)e.layers.size();
  if (std::fabs(e.layers[0].r_top - e.r_earth) > 1.0)
    throw std::runtime_error("radial_mesh_build: r_top(1) must equal r_earth");
  if (e.layers[nl - 1].r_bot != 0.0)
    throw std::runtime_error("radial_mesh_build: the innermost layer must reach r = 0");
  for (int i = 0; i < nl; ++i) {
    if (e.layers[i].r_top <= e.layers[i].r_bot)
      throw std::runtime_error("radial_mesh_build: every layer needs r_top > r_bot");
    if (i < nl - 1 && std::fabs(e.layers[i].r_bot - e.layers[i + 1].r_top) > 1.0)
      throw std::runtime_error("radial_mesh_build: layers must be contiguous");
  }
  bool explicit_counts = false;
  if (ne_layer)
    for (int i = 0; i < nl; ++i) explicit_counts |= ne_layer[i] > 0;
  auto count = [&](int i) {
    if (explicit_counts) return std::max(1, ne_layer[i]);
    double r0 = e.layers[i].r_bot, r1 = e.layers[i].r_top;
    double depth_mid = e.r_earth - 0.5 * (r0 + r1);
    return std::max(1, (int)std::ceil((r1 - r0) / dr_target(depth_mid)));
  };
  int ntot = 0;
  for (int i = 0; i < nl; ++i) ntot += count(i);
  Mesh m;
  m.ne = ntot;
  m.nr = ntot + 1;
  m.r.assign(m.nr, 0.0);
  m.elem_layer.assign(m.ne, 0);
  int off = 0;  // index of last node placed (0-based)
  for (int i = nl - 1; i >= 0; --i) {
    double r0 = e.layers[i].r_bot, r1 = e.layers[i].r_top;
    int nel = count(i);
    double h = (r1 - r0) / (double)nel;
    for (int k = 1; k <= nel; ++k) {
      m.r[off + k] = r0 + (double)k * h;
      m.elem_layer[off + k - 1] = i;
    }
    off += nel;
  }
  m.r[m.nr - 1] = e.r_earth;
  return m;
}

// vilma_radial_integrals.f90:28-126 (Martinec 2000 App. C). m[a][b], a,b in {0,1}.
struct M2 {
  double v[2][2];
};
static M2 I1(double rk, double rk1) {
  double h = rk1 - rk, d = (rk1 * rk1 + rk1 * rk + rk * rk) / (3.0 * h);
  return {{{d, -d}, {-d, d}}};
}
static M2 I2(double rk, double rk1) {
  M2 m;
  m.v[0][0] = -(rk1 * rk1 + 2.0 * rk1 * rk + 3.0 * rk * rk) / 12.0;
  m.v[0][1] = -m.v[0][0];
  m.v[1][1] = (3.0 * rk1 * rk1 + 2.0 * rk1 * rk + rk * rk) / 12.0;
  m.v[1][0] = -m.v[1][1];
  return m;
}
static M2 I3(double rk, double rk1) {
  M2 m;
  m.v[0][0] = -(rk1 + 2.0 * rk) / 6.0;
  m.v[0][1] = -m.v[0][0];
  m.v[1][1] = (2.0 * rk1 + rk) / 6.0;
  m.v[1][0] = -m.v[1][1];
  return m;
}
static M2 I4(double rk, double rk1) {
  double h = rk1 - rk;
  M2 m;
  m.v[0][0] = h / 30.0 * (rk1 * rk1 + 3.0 * rk1 * rk + 6.0 * rk * rk);
  m.v[0][1] = h / 60.0 * (3.0 * rk1 * rk1 + 4.0 * rk1 * rk + 3.0 * rk * rk);
  m.v[1][0] = m.v[0][1];
  m.v[1][1] = h / 30.0 * (6.0 * rk1 * rk1 + 3.0 * rk1 * rk + rk * rk);
  return m;
}
static M2 I5(double rk, double rk1) {
  double h = rk1 - rk;
  M2 m;
  m.v[0][0] = h / 12.0 * (rk1 + 3.0 * rk);
  m.v[0][1] = h / 12.0 * (rk1 + rk);
  m.v[1][0] = m.v[0][1];
  m.v[1][1] = h / 12.0 * (3.0 * rk1 + rk);
  return m;
}
static M2 I6(double rk, double rk1) {
  double h = rk1 - rk;
  return {{{h / 3.0, h / 6.0}, {h / 6.0, h / 3.0}}};
}
static M2 I7(double rk, double rk1) {
  double h = rk1 - rk, lg = std::log(rk1 / rk);
  M2 m;
  m.v[0][0] = (rk1 * rk1 / h * lg - 2.0 * rk1 + 0.5 * (rk1 + rk)) / h;
  m.v[0][1] = (-rk1 * rk / h * lg + 0.5 * (rk1 + rk)) / h;
  m.v[1][0] = m.v[0][1];
  m.v[1][1] = (rk * rk / h * lg - 2.0 * rk + 0.5 * (rk1 + rk)) / h;
  return m;
}
static void K1(double rk, double rk1, double v[2]) {
  v[0] = -(rk1 * rk1 + rk1 * rk + rk * rk) / 3.0;
  v[1] = -v[0];
}
static void K2(double rk, double rk1, double v[2]) {
  double h = rk1 - rk;
  v[0] = h / 6.0 * (rk1 + 2.0 * rk);
  v[1] = h / 6.0 * (2.0 * rk1 + rk);
}
static void K3(double rk, double rk1, double v[2]) {
  double h = rk1 - rk;
  v[0] = h / 12.0 * (rk1 * rk1 + 2.0 * rk1 * rk + 3.0 * rk * rk);
  v[1] = h / 12.0 * (3.0 * rk1 * rk1 + 2.0 * rk1 * rk + rk * rk);
}

// vilma_radial_fe.f90:252-270 shell_Rk
static std::vector<double> shell_Rk(const Earth& e, const Mesh& m) {
  std::vector<double> Rk(m.ne, 0.0);
  for (int k = 1; k < m.ne; ++k) {
    double rho_k = e.layers[m.elem_layer[k]].rho, rho_km1 = e.layers[m.elem_layer[k - 1]].rho;
    Rk[k] = Rk[k - 1] + (rho_km1 - rho_k) * std::pow(m.r[k], 3);
  }
  return Rk;
}

// vilma_radial_fe.f90:425-443 uniq_weight
std::vector<double> uniq_weight(const Mesh& m) {
  std::vector<double> w(ndof_of(m.nr), 0.0);
  for (int e = 0; e < m.ne; ++e) {
    double k3[2];
    K3(m.r[e], m.r[e + 1], k3);
    w[idx_u(e)] += k3[0];
    w[idx_u(e + 1)] += k3[1];
    w[idx_v(e)] += 2.0 * k3[0];
    w[idx_v(e + 1)] += 2.0 * k3[1];
  }
  return w;
}

// vilma_radial_fe.f90:274-423 build_dense_operator. Column-major A[k*nd + i].
std::vector<double> build_dense_operator(const Earth& e, const Mesh& m, int j, bool with_uniq) {
  const int nr = m.nr, ne = m.ne, nd = ndof_of(nr);
  const double Jr = (double)j * (double)(j + 1);
  const double fourpiG = 4.0 * PI * GRAV_G;
  std::vector<double> A((size_t)nd * nd, 0.0);
  auto Aat = [&](int i, int k) -> double& { return A[(size_t)k * nd + i]; };
  std::vector<double> Rk = shell_Rk(e, m);
  const int lU[2] = {0, 3}, lV[2] = {1, 4}, lF[2] = {2, 5}, lP = 6;
  for (int el = 0; el < ne; ++el) {
    double rlo = m.r[el], rhi = m.r[el + 1];
    const Layer& L = e.layers[m.elem_layer[el]];
    double mu_k = L.mu, rho_k = L.rho;
    M2 i1 = I1(rlo, rhi), i2 = I2(rlo, rhi), i3 = I3(rlo, rhi), i4 = I4(rlo, rhi), i5 = I5(rlo, rhi),
       i6 = I6(rlo, rhi);
    M2 i7 = {{{0, 0}, {0, 0}}};
    if (Rk[el] != 0.0) i7 = I7(rlo, rhi);
    double k1[2], k2[2];
    K1(rlo, rhi, k1);
    K2(rlo, rhi, k2);
    double Al[7][7] = {};
    for (int ia = 0; ia < 2; ++ia) {
      for (int ib = 0; ib < 2; ++ib) {
        // shear (eq 80), W dropped
        Al[lU[ib]][lU[ia]] += mu_k * (2.0 * i1.v[ia][ib]);
        Al[lV[ib]][lV[ia]] += mu_k * (Jr * i1.v[ia][ib]);
        Al[lV[ib]][lU[ia]] += mu_k * (Jr * i3.v[ia][ib]);
        Al[lV[ib]][lV[ia]] -= mu_k * (Jr * i3.v[ia][ib]);
        Al[lV[ib]][lV[ia]] -= mu_k * (Jr * i3.v[ib][ia]);
        Al[lU[ib]][lV[ia]] += mu_k * (Jr * i3.v[ib][ia]);
        Al[lU[ib]][lU[ia]] += mu_k * (Jr * i6.v[ia][ib]);
        Al[lU[ib]][lV[ia]] -= mu_k * (Jr * i6.v[ia][ib]);
        Al[lV[ib]][lU[ia]] -= mu_k * (Jr * i6.v[ia][ib]);
        Al[lV[ib]][lV[ia]] += mu_k * (Jr * i6.v[ia][ib]);
        Al[lU[ib]][lU[ia]] += mu_k * (4.0 * i6.v[ia][ib]);
        Al[lV[ib]][lU[ia]] -= mu_k * (2.0 * Jr * i6.v[ia][ib]);
        Al[lU[ib]][lV[ia]] -= mu_k * (2.0 * Jr * i6.v[ia][ib]);
        Al[lV[ib]][lV[ia]] += mu_k * (Jr * Jr * i6.v[ia][ib]);
        Al[lV[ib]][lV[ia]] += mu_k * (Jr * (Jr - 2.0) * i6.v[ia][ib]);
        // self-gravity (eq 81)
        double gg = (fourpiG / 3.0) * (rho_k * i4.v[ia][ib] + Rk[el] * i7.v[ia][ib]);
        Al[lU[ib]][lU[ia]] += rho_k * (-4.0 * gg + fourpiG * rho_k * i4.v[ia][ib]);
        Al[lU[ib]][lV[ia]] += rho_k * (Jr * gg);
        Al[lU[ib]][lF[ia]] += rho_k * (i2.v[ib][ia]);
        Al[lV[ib]][lU[ia]] += rho_k * (Jr * gg);
        Al[lV[ib]][lF[ia]] += rho_k * (Jr * i5.v[ia][ib]);
        Al[lF[ib]][lF[ia]] += (i1.v[ia][ib] + Jr * i6.v[ia][ib]) / fourpiG;
        Al[lF[ib]][lU[ia]] += rho_k * (i2.v[ia][ib]);
        Al[lF[ib]][lV[ia]] += rho_k * (Jr * i5.v[ia][ib]);
      }
    }
    // incompressibility (eq 82)
    for (int ia = 0; ia < 2; ++ia) {
      Al[lP][lU[ia]] += (k1[ia] + 2.0 * k2[ia]);
      Al[lU[ia]][lP] += (k1[ia] + 2.0 * k2[ia]);
      Al[lP][lV[ia]] -= (Jr * k2[ia]);
      Al[lV[ia]][lP] -= (Jr * k2[ia]);
    }
    int gmap[7] = {idx_u(el), idx_v(el), idx_f(el), idx_u(el + 1), idx_v(el + 1), idx_f(el + 1), idx_p(el)};
    for (int b = 0; b < 7; ++b)
      for (int a = 0; a < 7; ++a) Aat(gmap[b], gmap[a]) += Al[b][a];
  }
  // surface term (eq 84)
  Aat(idx_f(nr - 1), idx_f(nr - 1)) += e.r_earth / fourpiG * (double)(j + 1);
  if (j == 1 && with_uniq) {
    std::vector<double> w = uniq_weight(m);
    const double UNIQ = 4.0 * PI / 3.0;
    for (int ib = 0; ib < nd; ++ib) {
      if (w[ib] == 0.0) continue;
      for (int ia = 0; ia < nd; ++ia) {
        if (w[ia] == 0.0) continue;
        Aat(ib, ia) += UNIQ * w[ib] * w[ia];
      }
    }
  }
  return A;
}

// vilma_band.f90:28-59 band_build + :61-109 band_factor (dgbtf2 order)
static bool band_factor(Band& B) {
  const int n = B.n, kl = B.kl, ku = B.ku, kv = B.kv;
  int ju = 1;
  for (int j = 1; j <= n; ++j) {
    if (j + kv <= n)
      for (int i = 1; i <= kl; ++i) B.at(i, j + kv) = 0.0;
    int km = std::min(kl, n - j);
    int jp = 0;
    double piv = std::fabs(B.at(kv + 1, j));
    for (int p = 1; p <= km; ++p) {
      if (std::fabs(B.at(kv + 1 + p, j)) > piv) {
        piv = std::fabs(B.at(kv + 1 + p, j));
        jp = p;
      }
    }
    B.ipiv[j - 1] = j + jp - 1;
    if (B.at(kv + 1 + jp, j) == 0.0) return false;
    ju = std::max(ju, std::min(j + ku + jp, n));
    if (jp != 0) {
      for (int jj = j; jj <= ju; ++jj) {
        double tmp = B.at(kv + 1 + j - jj, jj);
        B.at(kv + 1 + j - jj, jj) = B.at(kv + 1 + (j + jp) - jj, jj);
        B.at(kv + 1 + (j + jp) - jj, jj) = tmp;
      }
    }
    if (km > 0) {
      double rp = 1.0 / B.at(kv + 1, j);
      for (int p = 1; p <= km; ++p) B.at(kv + 1 + p, j) *= rp;
      for (int jj = j + 1; jj <= ju; ++jj) {
        double tmp = B.at(kv + 1 + j - jj, jj);
        if (tmp != 0.0) {
          for (int p = 1; p <= km; ++p) {
            int i = j + p;
            B.at(kv + 1 + i - jj, jj) -= B.at(kv + 1 + p, j) * tmp;
          }
        }
      }
    }
  }
  return true;
}

bool band_build(Band& B, int n, const std::vector<int>& rows, const std::vector<int>& cols,
                const std::vector<double>& vals) {
  int kl = 0, ku = 0;
  for (size_t t = 0; t < vals.size(); ++t) {
    if (vals[t] == 0.0) continue;
    kl = std::max(kl, rows[t] - cols[t]);
    ku = std::max(ku, cols[t] - rows[t]);
  }
  B.n = n;
  B.kl = kl;
  B.ku = ku;
  B.kv = kl + ku;
  B.ldab = 2 * kl + ku + 1;
  B.ab.assign((size_t)B.ldab * n, 0.0);
  B.ipiv.assign(n, 0);
  for (size_t t = 0; t < vals.size(); ++t) {
    if (vals[t] == 0.0) continue;
    B.at(B.kv + 1 + rows[t] - cols[t], cols[t]) += vals[t];
  }
  return band_factor(B);
}

// vilma_band.f90:111-142 band_solve (dgbtrs, no transpose), in place
void band_solve(const Band& B, double* x) {
  const int n = B.n, kl = B.kl, kv = B.kv;
  for (int j = 1; j <= n - 1; ++j) {
    int lm = std::min(kl, n - j);
    int l = B.ipiv[j - 1] + 1;
    if (l != j) std::swap(x[l - 1], x[j - 1]);
    double tmp = x[j - 1];
    for (int i = 1; i <= lm; ++i) x[j + i - 1] -= B.at(kv + 1 + i, j) * tmp;
  }
  for (int j = n; j >= 1; --j) {
    x[j - 1] = x[j - 1] / B.at(kv + 1, j);
    double tmp = x[j - 1];
    int lm = std::min(kv, j - 1);
    for (int i = 1; i <= lm; ++i) x[j - i - 1] -= B.at(kv + 1 - i, j) * tmp;
  }
}

// vilma_radial_fe.f90:819-833 colnorm / rownorm
static double colnorm_of(const double* col, int n, int stride) {
  double m = 0.0;
  for (int i = 0; i < n; ++i) m = std::max(m, std::fabs(col[(size_t)i * stride]));
  return m > 0.0 ? 1.0 / std::sqrt(m) : 1.0;
}

// vilma_radial_fe.f90:497-576 bordered_band_factor
void bordered_band_factor(BorderedBand& sys, const std::vector<double>& A, int nd, const std::vector<double>& w,
                          int nb) {
  sys.nd = nd;
  sys.nb = nb;
  sys.ns = nd + nb;
  sys.w.assign((size_t)nd * nb, 0.0);
  if (nb) sys.w.assign(w.begin(), w.begin() + (size_t)nd * nb);
  sys.dc.assign(nd, 1.0);
  sys.dr.assign(nd, 1.0);
  std::vector<double> dc_b(nb), dr_b(nb);
  for (int k = 0; k < nd; ++k) {
    sys.dc[k] = colnorm_of(&A[(size_t)k * nd], nd, 1);
    for (int b = 0; b < nb; ++b)
      if (std::fabs(sys.w[(size_t)b * nd + k]) > 1.0 / (sys.dc[k] * sys.dc[k]))
        sys.dc[k] = 1.0 / std::sqrt(std::fabs(sys.w[(size_t)b * nd + k]));
  }
  for (int b = 0; b < nb; ++b) dc_b[b] = colnorm_of(&sys.w[(size_t)b * nd], nd, 1);
  for (int i = 0; i < nd; ++i) {
    double m = 0.0;
    for (int k = 0; k < nd; ++k) m = std::max(m, std::fabs(A[(size_t)k * nd + i] * sys.dc[k]));
    sys.dr[i] = m > 0.0 ? 1.0 / std::sqrt(m) : 1.0;
    for (int b = 0; b < nb; ++b)
      if (std::fabs(sys.w[(size_t)b * nd + i]) * dc_b[b] > 1.0 / (sys.dr[i] * sys.dr[i]))
        sys.dr[i] = 1.0 / std::sqrt(std::fabs(sys.w[(size_t)b * nd + i]) * dc_b[b]);
  }
  for (int b = 0; b < nb; ++b) {
    double m = 0.0;
    for (int k = 0; k < nd; ++k) m = std::max(m, std::fabs(sys.w[(size_t)b * nd + k] * sys.dc[k]));
    dr_b[b] = m > 0.0 ? 1.0 / std::sqrt(m) : 1.0;
  }
  std::vector<int> rows, cols;
  std::vector<double> vals;
  for (int k = 0; k < nd; ++k)
    for (int i = 0; i < nd; ++i) {
      double a = A[(size_t)k * nd + i];
      if (a == 0.0) continue;
      rows.push_back(i + 1);
      cols.push_back(k + 1);
      vals.push_back(sys.dr[i] * a * sys.dc[k]);
    }
  for (int b = 0; b < nb; ++b) {
    const double* wb = &sys.w[(size_t)b * nd];
    for (int i = 0; i < nd; ++i) {
      if (wb[i] == 0.0) continue;
      rows.push_back(i + 1);
      cols.push_back(nd + b + 1);
      vals.push_back(sys.dr[i] * wb[i] * dc_b[b]);
    }
    for (int k = 0; k < nd; ++k) {
      if (wb[k] == 0.0) continue;
      rows.push_back(nd + b + 1);
      cols.push_back(k + 1);
      vals.push_back(dr_b[b] * wb[k] * sys.dc[k]);
    }
  }
  if (!band_build(sys.band, sys.ns, rows, cols, vals))
    throw std::runtime_error("bordered_band_factor: band LU factorization failed");
}

// vilma_radial_fe.f90:578-605 bordered_band_solve
void bordered_band_solve(const BorderedBand& sys, const double* b, double* x, const double* border) {
  std::vector<double> bs(sys.ns, 0.0);
  for (int i = 0; i < sys.nd; ++i) bs[i] = sys.dr[i] * b[i];
  if (border)
    for (int i = 0; i < sys.nb; ++i) bs[sys.nd + i] = border[i];
  band_solve(sys.band, bs.data());
  for (int i = 0; i < sys.nd; ++i) x[i] = sys.dc[i] * bs[i];
}

// vilma_radial_fe.f90:447-495 radial_operator_assemble
void radial_operator_assemble(RadialOp& op, const Earth& e, const Mesh& m, int j) {
  std::vector<double> A = build_dense_operator(e, m, j, false);
  int nd = ndof_of(m.nr);
  op.j = j;
  op.nr = m.nr;
  op.ne = m.ne;
  op.ndof = nd;
  op.r_earth = e.r_earth;
  op.g_surf = earth_gravity_at(e, e.r_earth);
  if (j == 1) {
    std::vector<double> w = uniq_weight(m);
    bordered_band_factor(op.sys, A, nd, w, 1);
  } else {
    bordered_band_factor(op.sys, A, nd, {}, 0);
  }
  op.nullmode.clear();
  if (op.sys.nb > 0) {
    std::vector<double> zero(nd, 0.0);
    op.nullmode.assign(nd, 0.0);
    double one = 1.0;
    bordered_band_solve(op.sys, zero.data(), op.nullmode.data(), &one);
  }
}

// vilma_radial_fe.f90:647-671
void radial_operator_solve_vec(const RadialOp& op, const double* b, double* x, const double* border) {
  if (border && op.sys.nb > 0)
    bordered_band_solve(op.sys, b, x, border);
  else
    bordered_band_solve(op.sys, b, x, nullptr);
}

// vilma_radial_fe.f90:616-625
void radial_operator_load_rhs(const RadialOp& op, double sigma, double* b) {
  for (int i = 0; i < op.ndof; ++i) b[i] = 0.0;
  b[idx_u(op.nr - 1)] = -op.r_earth * op.r_earth * sigma * op.g_surf;
  b[idx_f(op.nr - 1)] = -op.r_earth * op.r_earth * sigma;
}

// vilma_radial_fe.f90:627-645 radial_operator_tidal_rhs: external degree-j
// potential phi_t couples to F(a) like the load's own potential, no traction on U(a)
void radial_operator_tidal_rhs(const RadialOp& op, double phi_t, double* b) {
  for (int i = 0; i < op.ndof; ++i) b[i] = 0.0;
  b[idx_f(op.nr - 1)] = -op.r_earth / (4.0 * PI * GRAV_G) * (double)(2 * op.j + 1) * phi_t;
}

// vilma_radial_fe.f90:837-866
void loading_love(const Earth& e, int j, double sigma, double Ua, double Va, double Fa, double& h,
                  double& l, double& k) {
  double a = e.r_earth, g = earth_gravity_at(e, a);
  double phiL = 4.0 * PI * GRAV_G * a * sigma / (double)(2 * j + 1);
  h = g * Ua / phiL;
  l = g * Va / phiL;
  k = -Fa / phiL - 1.0;
}

}  // namespace orc

namespace orc {

// vilma_radial_integrals.f90:117-126 elem_k4: int psi_a r^3 dr
static void K4(double rk, double rk1, double v[2]) {
  double h = rk1 - rk;
  v[0] = h / 20.0 * (rk1 * rk1 * rk1 + 2.0 * rk1 * rk1 * rk + 3.0 * rk1 * rk * rk + 4.0 * rk * rk * rk);
  v[1] = h / 20.0 * (4.0 * rk1 * rk1 * rk1 + 3.0 * rk1 * rk1 * rk + 2.0 * rk1 * rk * rk + rk * rk * rk);
}

// vilma_radial_fe.f90:699-729 build_toroidal_operator: per element
// mu_k { J [I1 - I3(b,a) - I3(a,b) + I6] + J(J-2) I6 } W^a dW^b; column-major
std::vector<double> build_toroidal_operator(const std::vector<double>& r, const std::vector<double>& mu, int j) {
  const int nr = (int)r.size(), ne = (int)mu.size();
  const double Jr = (double)j * (double)(j + 1);
  std::vector<double> A((size_t)nr * nr, 0.0);
  for (int e = 0; e < ne; ++e) {
    if (mu[e] == 0.0) continue;
    M2 i1 = I1(r[e], r[e + 1]), i3 = I3(r[e], r[e + 1]), i6 = I6(r[e], r[e + 1]);
    for (int ia = 0; ia < 2; ++ia)      // trial node
      for (int ib = 0; ib < 2; ++ib) {  // test node: row
        A[(size_t)(e + ia) * nr + (e + ib)] +=
            mu[e] * (Jr * (i1.v[ia][ib] - i3.v[ib][ia] - i3.v[ia][ib] + i6.v[ia][ib]) + Jr * (Jr - 2.0) * i6.v[ia][ib]);
      }
  }
  return A;
}

// vilma_radial_fe.f90:745-773 rotation_weights: one column per solid shell
// (a maximal run of mu > 0 elements), w_s(k) = sum_{e in s} int psi_k r^3 dr
std::vector<double> rotation_weights(const std::vector<double>& r, const std::vector<double>& mu, int& nshell) {
  const int nr = (int)r.size(), ne = (int)mu.size();
  std::vector<int> shell(ne, -1);
  int ns = 0;
  bool prev = false;
  for (int e = 0; e < ne; ++e) {
    bool solid = mu[e] > 0.0;
    if (solid && !prev) ++ns;
    if (solid) shell[e] = ns - 1;
    prev = solid;
  }
  std::vector<double> w((size_t)nr * ns, 0.0);
  for (int e = 0; e < ne; ++e) {
    if (shell[e] < 0) continue;
    double k4[2];
    K4(r[e], r[e + 1], k4);
    w[(size_t)shell[e] * nr + e] += k4[0];
    w[(size_t)shell[e] * nr + e + 1] += k4[1];
  }
  nshell = ns;
  return w;
}

// vilma_radial_fe.f90:775-799 toroidal_operator_assemble (with
// toroidal_dead_nodes, :731-743)
void toroidal_operator_assemble(TorOp& op, const std::vector<double>& r, const std::vector<double>& mu, int j) {
  if (j < 1) throw std::runtime_error("toroidal_operator_assemble: toroidal fields start at degree 1");
  const int nr = (int)r.size(), ne = (int)mu.size();
  op.j = j;
  op.nr = nr;
  op.ne = ne;
  std::vector<double> A = build_toroidal_operator(r, mu, j);
  op.pinned.assign(nr, 1);
  for (int e = 0; e < ne; ++e)
    if (mu[e] > 0.0) op.pinned[e] = op.pinned[e + 1] = 0;
  for (int k = 0; k < nr; ++k)
    if (op.pinned[k]) A[(size_t)k * nr + k] = 1.0;
  if (j == 1) {
    int ns = 0;
    std::vector<double> w = rotation_weights(r, mu, ns);
    bordered_band_factor(op.sys, A, nr, w, ns);
  } else {
    bordered_band_factor(op.sys, A, nr, {}, 0);
  }
}

// vilma_radial_fe.f90:801-810 toroidal_operator_solve_vec
void toroidal_operator_solve_vec(const TorOp& op, const double* b, double* x) {
  std::vector<double> bd(op.nr);
  for (int k = 0; k < op.nr; ++k) bd[k] = op.pinned[k] ? 0.0 : b[k];
  bordered_band_solve(op.sys, bd.data(), x, nullptr);
}

}  // namespace orc
