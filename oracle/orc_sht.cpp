// CPU ORACLE — test infrastructure only (see orc.hpp).
// Spherical-harmonic transforms on a Gauss grid, restating the conventions the
// reference fixes for SHTns 3.7.5 (vilma_sht.f90:11-15, 135-153): orthonormal
// real harmonics without the Condon-Shortley phase, Gauss-Legendre latitudes
// north first, phi-contiguous (nphi, nlat) fields, m >= 0 stored in m-major lm
// order, and f = sum_l q_l0 Y_l0 + 2 Re sum_{m>0} q_lm Y_lm for a real field.
// SHTns itself is an external dependency absent from the reference tree; the
// transforms below are derived from those conventions, with a mixed-radix FFT
// standing in for FFTW.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "orc.hpp"

namespace orc {

// Gauss-Legendre nodes (x descending, i.e. colatitude ascending) and weights.
static void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(PI * (i + 0.75) / (n + 0.5)), pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int k = 1; k <= n; ++k) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * k - 1.0) * z * p2 - (k - 1.0) * p3) / k;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-16) break;
    }
    // recompute derivative at the converged node
    double p1 = 1.0, p2 = 0.0;
    for (int k = 1; k <= n; ++k) {
      double p3 = p2;
      p2 = p1;
      p1 = ((2.0 * k - 1.0) * z * p2 - (k - 1.0) * p3) / k;
    }
    pp = n * (z * p1 - p2) / (z * z - 1.0);
    x[i] = z;
    x[n - 1 - i] = -z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    w[n - 1 - i] = w[i];
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
}

// ---- mixed-radix complex FFT (decimation in time), forward sign e^{-i} ----
static void fft_rec(const Sht& s, const cplx* in, cplx* out, int n, int stride, int fi, cplx* tmp) {
  const int N = s.nphi;
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = s.fft_factors[fi], m = n / p;
  for (int q = 0; q < p; ++q) fft_rec(s, in + (size_t)q * stride, out + (size_t)q * m, m, stride * p, fi + 1, tmp);
  const int step = N / n;
  for (int k = 0; k < m; ++k) {
    for (int r = 0; r < p; ++r) {
      cplx acc = 0.0;
      for (int q = 0; q < p; ++q) {
        int e = (q * (k + r * m)) % n;
        acc += out[(size_t)q * m + k] * s.tw[(size_t)e * step];
      }
      tmp[k + r * m] = acc;
    }
  }
  for (int t = 0; t < n; ++t) out[t] = tmp[t];
}
static void fft(const Sht& s, const cplx* in, cplx* out) {
  std::vector<cplx> tmp(s.nphi);
  fft_rec(s, in, out, s.nphi, 1, 0, tmp.data());
}

// spectrum G_m (m = 0..mmax) -> real row f_i = Re G_0 + 2 Re sum_m G_m e^{i m phi_i}
static void row_synth(const Sht& s, const cplx* G, double* f) {
  const int N = s.nphi;
  std::vector<cplx> X(N, 0.0), Y(N);
  X[0] = cplx(G[0].real(), 0.0);
  for (int m = 1; m <= s.mmax; ++m) {
    X[m] = G[m];
    X[N - m] = std::conj(G[m]);
  }
  for (int t = 0; t < N; ++t) X[t] = std::conj(X[t]);
  fft(s, X.data(), Y.data());
  for (int i = 0; i < N; ++i) f[i] = Y[i].real();
}
// real row -> F_m = (2 pi / N) sum_i f_i e^{-i m phi_i}, m = 0..mmax
static void row_analysis(const Sht& s, const double* f, cplx* F) {
  const int N = s.nphi;
  std::vector<cplx> X(N), Y(N);
  for (int i = 0; i < N; ++i) X[i] = cplx(f[i], 0.0);
  fft(s, X.data(), Y.data());
  const double sc = 2.0 * PI / (double)N;
  for (int m = 0; m <= s.mmax; ++m) F[m] = Y[m] * sc;
}

void sht_init(Sht& s, int lmax, int nlat, int nphi) {
  s.lmax = lmax;
  s.mmax = lmax;
  s.nlat = nlat;
  s.nphi = nphi;
  if (nphi <= 2 * s.mmax) throw std::runtime_error("sht_init: nphi must exceed 2*mmax");
  if (nlat < lmax + 1) throw std::runtime_error("sht_init: nlat must be >= lmax+1");
  s.nlm = (lmax + 1) * (lmax + 2) / 2;
  gauss_legendre(nlat, s.x, s.wts);
  s.colat.resize(nlat);
  s.sint.resize(nlat);
  s.cott.resize(nlat);
  s.invsin.resize(nlat);
  for (int j = 0; j < nlat; ++j) {
    s.colat[j] = std::acos(s.x[j]);
    s.sint[j] = std::sqrt((1.0 - s.x[j]) * (1.0 + s.x[j]));
    s.cott[j] = std::cos(s.colat[j]) / std::sin(s.colat[j]);  // vilma_tensor_sh.f90:95
    s.invsin[j] = 1.0 / std::sin(s.colat[j]);
  }
  s.ldeg.resize(s.nlm);
  s.mord.resize(s.nlm);
  s.llp1.resize(s.nlm);
  for (int m = 0; m <= s.mmax; ++m)
    for (int l = m; l <= lmax; ++l) {
      int lm = s.lmidx(l, m);
      s.ldeg[lm] = l;
      s.mord[lm] = m;
      s.llp1[lm] = (double)l * (double)(l + 1);
    }
  // orthonormal associated Legendre functions (no CS phase) and d/dtheta
  s.plm.assign((size_t)s.nlm * nlat, 0.0);
  s.dplm.assign((size_t)s.nlm * nlat, 0.0);
  for (int j = 0; j < nlat; ++j) {
    double x = s.x[j], st = s.sint[j];
    double pmm = 1.0 / std::sqrt(4.0 * PI);
    for (int m = 0; m <= s.mmax; ++m) {
      if (m > 0) pmm *= std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * st;
      double p_lm2 = 0.0, p_lm1 = pmm;
      s.plm[(size_t)s.lmidx(m, m) * nlat + j] = pmm;
      for (int l = m + 1; l <= lmax; ++l) {
        double a = std::sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
        double b = std::sqrt((((double)(l - 1) * (l - 1)) - (double)m * m) / (4.0 * (l - 1) * (l - 1) - 1.0));
        double p = a * (x * p_lm1 - b * p_lm2);
        s.plm[(size_t)s.lmidx(l, m) * nlat + j] = p;
        p_lm2 = p_lm1;
        p_lm1 = p;
      }
      for (int l = m; l <= lmax; ++l) {
        double p = s.plm[(size_t)s.lmidx(l, m) * nlat + j];
        double pl1 = (l > m) ? s.plm[(size_t)s.lmidx(l - 1, m) * nlat + j] : 0.0;
        double c = std::sqrt((2.0 * l + 1.0) * ((double)l * l - (double)m * m) / (2.0 * l - 1.0));
        s.dplm[(size_t)s.lmidx(l, m) * nlat + j] = (l * x * p - c * pl1) / st;
      }
    }
  }
  // FFT plan
  s.fft_factors.clear();
  int n = nphi;
  for (int p = 2; n > 1;) {
    if (n % p == 0) {
      s.fft_factors.push_back(p);
      n /= p;
    } else {
      ++p;
    }
  }
  s.tw.resize(nphi);
  for (int t = 0; t < nphi; ++t) s.tw[t] = std::polar(1.0, -2.0 * PI * (double)t / (double)nphi);
  s.n6.clear();
}

// vilma_tensor_sh.f90:99-133: per-degree spin-2 norms, a unit Z6 (and Z4)
// coefficient at the sectoral order m = l sent through the synthesis and its
// adjoint.
void sht_calibrate_n6(Sht& s) {
  if (!s.n6.empty()) return;
  std::vector<double> n6(s.lmax + 1, 0.0), n4(s.lmax + 1, 0.0);
  s.n6.assign(s.lmax + 1, 1.0);  // provisional unit norms: analysis returns the raw adjoints
  s.n4.assign(s.lmax + 1, 1.0);
  std::vector<cplx> c6((size_t)6 * s.nlm, 0.0), craw((size_t)6 * s.nlm);
  std::vector<double> dy((size_t)6 * s.nlat * s.nphi);
  for (int l = 2; l <= s.lmax; ++l) {
    int m = std::min(l, s.mmax);
    if (m < 1) continue;
    int lm = s.lmidx(l, m);
    std::fill(c6.begin(), c6.end(), cplx(0.0));
    c6[(size_t)3 * s.nlm + lm] = 1.0;
    tensor_synth(s, c6.data(), dy.data(), 6);
    tensor_analysis(s, dy.data(), craw.data(), 6);
    n6[l] = craw[(size_t)3 * s.nlm + lm].real();
    std::fill(c6.begin(), c6.end(), cplx(0.0));
    c6[(size_t)5 * s.nlm + lm] = 1.0;  // the same coefficient as Z4
    tensor_synth(s, c6.data(), dy.data(), 6);
    tensor_analysis(s, dy.data(), craw.data(), 6);
    n4[l] = craw[(size_t)5 * s.nlm + lm].real();
  }
  s.n6 = n6;
  s.n4 = n4;
}

// vilma_sht.f90:184-202
double sht_surface_integral(const Sht& s, const double* f) {
  double dlon = 2.0 * PI / (double)s.nphi, total = 0.0;
  for (int j = 0; j < s.nlat; ++j) {
    double row = 0.0;
    for (int i = 0; i < s.nphi; ++i) row += f[(size_t)j * s.nphi + i];
    total += s.wts[j] * row * dlon;
  }
  return total;
}

// generic per-m Legendre sums: G[m][j] = sum_l q_lm * T_lm(j) (T = plm or dplm)
static void legendre_sum(const Sht& s, const cplx* q, const std::vector<double>& T, std::vector<cplx>& G) {
  const int nl = s.nlat, M = s.mmax + 1;
  G.assign((size_t)M * nl, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int m = 0; m < M; ++m)
    for (int l = m; l <= s.lmax; ++l) {
      int lm = s.lmidx(l, m);
      cplx c = q[lm];
      const double* t = &T[(size_t)lm * nl];
      cplx* g = &G[(size_t)m * nl];
      for (int j = 0; j < nl; ++j) g[j] += c * t[j];
    }
}
static void fourier_synth(const Sht& s, const std::vector<cplx>& G, double* f) {
  const int nl = s.nlat, M = s.mmax + 1;
#pragma omp parallel
  {
    std::vector<cplx> row(M);
#pragma omp for schedule(static)
    for (int j = 0; j < nl; ++j) {
      for (int m = 0; m < M; ++m) row[m] = G[(size_t)m * nl + j];
      row_synth(s, row.data(), f + (size_t)j * s.nphi);
    }
  }
}
static void fourier_analysis(const Sht& s, const double* f, std::vector<cplx>& F) {
  const int nl = s.nlat, M = s.mmax + 1;
  F.assign((size_t)M * nl, 0.0);
#pragma omp parallel
  {
    std::vector<cplx> row(M);
#pragma omp for schedule(static)
    for (int j = 0; j < nl; ++j) {
      row_analysis(s, f + (size_t)j * s.nphi, row.data());
      for (int m = 0; m < M; ++m) F[(size_t)m * nl + j] = row[m];
    }
  }
}

void sht_synth(const Sht& s, const cplx* q, double* f) {
  std::vector<cplx> G;
  legendre_sum(s, q, s.plm, G);
  fourier_synth(s, G, f);
}

void sht_analysis(const Sht& s, const double* f, cplx* q) {
  std::vector<cplx> F;
  fourier_analysis(s, f, F);
  const int nl = s.nlat;
#pragma omp parallel for schedule(dynamic)
  for (int m = 0; m <= s.mmax; ++m)
    for (int l = m; l <= s.lmax; ++l) {
      int lm = s.lmidx(l, m);
      const double* t = &s.plm[(size_t)lm * nl];
      const cplx* Fm = &F[(size_t)m * nl];
      cplx acc = 0.0;
      for (int j = 0; j < nl; ++j) acc += (s.wts[j] * t[j]) * Fm[j];
      q[lm] = acc;
    }
}

// vth = d/dtheta, vph = (1/sin) d/dphi of sum S_lm Y_lm (SHsph_to_spat)
void sht_sph_synth(const Sht& s, const cplx* sl, double* vt, double* vp) {
  std::vector<cplx> Gt, Gp;
  legendre_sum(s, sl, s.dplm, Gt);
  legendre_sum(s, sl, s.plm, Gp);
  const int nl = s.nlat;
  for (int m = 0; m <= s.mmax; ++m)
    for (int j = 0; j < nl; ++j) Gp[(size_t)m * nl + j] *= cplx(0.0, (double)m * s.invsin[j]);
  fourier_synth(s, Gt, vt);
  fourier_synth(s, Gp, vp);
}

// spheroidal part of spat_to_SHsphtor: S_lm = (1/l(l+1)) <v, grad Y_lm> (quadrature)
void sht_sph_analysis(const Sht& s, const double* vt, const double* vp, cplx* sl) {
  std::vector<cplx> Ft, Fp;
  fourier_analysis(s, vt, Ft);
  fourier_analysis(s, vp, Fp);
  const int nl = s.nlat;
#pragma omp parallel for schedule(dynamic)
  for (int m = 0; m <= s.mmax; ++m)
    for (int l = m; l <= s.lmax; ++l) {
      int lm = s.lmidx(l, m);
      if (l == 0) {
        sl[lm] = 0.0;
        continue;
      }
      const double* t = &s.plm[(size_t)lm * nl];
      const double* d = &s.dplm[(size_t)lm * nl];
      cplx acc = 0.0;
      for (int j = 0; j < nl; ++j)
        acc += s.wts[j] * (d[j] * Ft[(size_t)m * nl + j] +
                           cplx(0.0, -(double)m * s.invsin[j]) * t[j] * Fp[(size_t)m * nl + j]);
      sl[lm] = acc / ((double)l * (double)(l + 1));
    }
}

// vilma_sht.f90:258-277 tor_synthesis: e_r x grad_1 T = (-F, E) with
// (E, F) = (d/dtheta, (1/sin) d/dphi) of sum T_lm Y_lm
void sht_tor_synth(const Sht& s, const cplx* tl, double* vt, double* vp) {
  const size_t ng = (size_t)s.nphi * s.nlat;
  std::vector<double> E(ng), F(ng);
  sht_sph_synth(s, tl, E.data(), F.data());
  for (size_t p = 0; p < ng; ++p) {
    vt[p] = -F[p];
    vp[p] = E[p];
  }
}

// toroidal part of spat_to_SHsphtor in this orientation (vilma_sht.f90:294-308):
// T_lm = (1/l(l+1)) <v, e_r x grad Y_lm> (quadrature)
void sht_tor_analysis(const Sht& s, const double* vt, const double* vp, cplx* tl) {
  std::vector<cplx> Ft, Fp;
  fourier_analysis(s, vt, Ft);
  fourier_analysis(s, vp, Fp);
  const int nl = s.nlat;
#pragma omp parallel for schedule(dynamic)
  for (int m = 0; m <= s.mmax; ++m)
    for (int l = m; l <= s.lmax; ++l) {
      int lm = s.lmidx(l, m);
      if (l == 0) {
        tl[lm] = 0.0;
        continue;
      }
      const double* t = &s.plm[(size_t)lm * nl];
      const double* d = &s.dplm[(size_t)lm * nl];
      cplx acc = 0.0;
      for (int j = 0; j < nl; ++j)
        acc += s.wts[j] * (cplx(0.0, (double)m * s.invsin[j]) * t[j] * Ft[(size_t)m * nl + j] +
                           d[j] * Fp[(size_t)m * nl + j]);
      tl[lm] = acc / ((double)l * (double)(l + 1));
    }
}

// ------------------------------------------------------------- tensor SH
static void byprof(const Sht& s, const double* f, const std::vector<double>& prof, double* out) {
  for (int j = 0; j < s.nlat; ++j)
    for (int i = 0; i < s.nphi; ++i) out[(size_t)j * s.nphi + i] = f[(size_t)j * s.nphi + i] * prof[j];
}

// vilma_tensor_sh.f90:244-266 spin2_fields
static void spin2_fields(const Sht& s, const cplx* c6, double* sg, double* sh) {
  const size_t ng = (size_t)s.nphi * s.nlat;
  std::vector<cplx> imc(s.nlm), lapc(s.nlm);
  for (int lm = 0; lm < s.nlm; ++lm) {
    imc[lm] = cplx(0.0, (double)s.mord[lm]) * c6[lm];
    lapc[lm] = -s.llp1[lm] * c6[lm];
  }
  std::vector<double> gt(ng), gp(ng), gtf(ng), gpf(ng), lap(ng);
  sht_sph_synth(s, c6, gt.data(), gp.data());
  sht_sph_synth(s, imc.data(), gtf.data(), gpf.data());
  sht_synth(s, lapc.data(), lap.data());
  for (int j = 0; j < s.nlat; ++j)
    for (int i = 0; i < s.nphi; ++i) {
      size_t p = (size_t)j * s.nphi + i;
      sg[p] = lap[p] - 2.0 * (gt[p] * s.cott[j]) - 2.0 * (gpf[p] * s.invsin[j]);
      sh[p] = (gtf[p] * s.invsin[j]) - (gp[p] * s.cott[j]);
    }
}

// vilma_tensor_sh.f90:168-203 tensor_sh_synth, with spin2_synth_tor (:231-242)
// for the toroidal channels
void tensor_synth(const Sht& s, const cplx* c, double* dyad, int nch) {
  const size_t ng = (size_t)s.nphi * s.nlat;
  const int nlm = s.nlm;
  double* rr = dyad;
  double* rt = dyad + ng;
  double* rp = dyad + 2 * ng;
  double* tt = dyad + 3 * ng;
  double* tp = dyad + 4 * ng;
  double* pp = dyad + 5 * ng;
  sht_synth(s, c, rr);
  sht_sph_synth(s, c + nlm, rt, rp);
  std::vector<cplx> scaled(nlm);
  for (int lm = 0; lm < nlm; ++lm) scaled[lm] = -s.llp1[lm] * c[2 * nlm + lm];
  std::vector<double> tr(ng), sg(ng), sh(ng);
  sht_synth(s, scaled.data(), tr.data());
  spin2_fields(s, c + 3 * nlm, sg.data(), sh.data());
  for (size_t p = 0; p < ng; ++p) {
    tt[p] = tr[p] + sg[p];
    pp[p] = tr[p] - sg[p];
    tp[p] = 4.0 * sh[p];
  }
  if (nch == 4) return;
  // Z3: (rt, rp) += e_r x grad_1 c5; Z4 = G e_tp - H (e_tt - e_pp): (-Sh, +Sh, Sg)
  std::vector<double> vt(ng), vp(ng);
  sht_tor_synth(s, c + 4 * nlm, vt.data(), vp.data());
  spin2_fields(s, c + 5 * nlm, sg.data(), sh.data());
  for (size_t p = 0; p < ng; ++p) {
    rt[p] += vt[p];
    rp[p] += vp[p];
    tt[p] -= sh[p];
    pp[p] += sh[p];
    tp[p] += sg[p];
  }
}

// vilma_tensor_sh.f90:270-358 tensor_sh_analysis + spin2_adjoint, with
// spin2_adjoint_tor (:360-387) for the toroidal channels
void tensor_analysis(const Sht& s, const double* dyad, cplx* c, int nch) {
  const size_t ng = (size_t)s.nphi * s.nlat;
  const int nlm = s.nlm;
  const double* rr = dyad;
  const double* rt = dyad + ng;
  const double* rp = dyad + 2 * ng;
  const double* tt = dyad + 3 * ng;
  const double* tp = dyad + 4 * ng;
  const double* pp = dyad + 5 * ng;
  sht_analysis(s, rr, c);
  sht_sph_analysis(s, rt, rp, c + nlm);
  std::vector<double> vt(ng), vp(ng, 0.0), D(ng), zero(ng, 0.0);
  std::vector<cplx> craw(nlm), q(nlm), sv(nlm);
  for (size_t p = 0; p < ng; ++p) vt[p] = tt[p] + pp[p];
  sht_analysis(s, vt.data(), craw.data());
  for (int lm = 0; lm < nlm; ++lm)
    c[2 * nlm + lm] = s.llp1[lm] > 0.0 ? craw[lm] / (-2.0 * s.llp1[lm]) : cplx(0.0);
  // spin2_adjoint
  for (size_t p = 0; p < ng; ++p) D[p] = tt[p] - pp[p];
  sht_analysis(s, D.data(), q.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] = -s.llp1[lm] * q[lm];
  byprof(s, D.data(), s.cott, vt.data());
  sht_sph_analysis(s, vt.data(), zero.data(), sv.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] -= 2.0 * s.llp1[lm] * sv[lm];
  byprof(s, D.data(), s.invsin, vp.data());
  sht_sph_analysis(s, zero.data(), vp.data(), sv.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] += 2.0 * cplx(0.0, (double)s.mord[lm]) * s.llp1[lm] * sv[lm];
  byprof(s, tp, s.invsin, vt.data());
  sht_sph_analysis(s, vt.data(), zero.data(), sv.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] -= 2.0 * cplx(0.0, (double)s.mord[lm]) * s.llp1[lm] * sv[lm];
  byprof(s, tp, s.cott, vp.data());
  sht_sph_analysis(s, zero.data(), vp.data(), sv.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] -= 2.0 * s.llp1[lm] * sv[lm];
  for (int lm = 0; lm < nlm; ++lm) {
    double n6 = s.n6[s.ldeg[lm]];
    c[3 * nlm + lm] = n6 != 0.0 ? craw[lm] / n6 : cplx(0.0);
  }
  if (nch == 4) return;
  sht_tor_analysis(s, rt, rp, c + 4 * nlm);
  // Z4 numerator: 1/2 Sg*(tp) - Sh*(tt - pp)
  sht_analysis(s, tp, q.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] = -0.5 * s.llp1[lm] * q[lm];
  byprof(s, tp, s.cott, vt.data());
  sht_sph_analysis(s, vt.data(), zero.data(), sv.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] -= s.llp1[lm] * sv[lm];
  byprof(s, tp, s.invsin, vp.data());
  sht_sph_analysis(s, zero.data(), vp.data(), sv.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] += cplx(0.0, (double)s.mord[lm]) * s.llp1[lm] * sv[lm];
  byprof(s, D.data(), s.invsin, vt.data());
  sht_sph_analysis(s, vt.data(), zero.data(), sv.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] += cplx(0.0, (double)s.mord[lm]) * s.llp1[lm] * sv[lm];
  byprof(s, D.data(), s.cott, vp.data());
  sht_sph_analysis(s, zero.data(), vp.data(), sv.data());
  for (int lm = 0; lm < nlm; ++lm) craw[lm] += s.llp1[lm] * sv[lm];
  for (int lm = 0; lm < nlm; ++lm) {
    double n4 = s.n4.empty() ? 0.0 : s.n4[s.ldeg[lm]];
    c[5 * nlm + lm] = n4 != 0.0 ? craw[lm] / n4 : cplx(0.0);
  }
}

}  // namespace orc
