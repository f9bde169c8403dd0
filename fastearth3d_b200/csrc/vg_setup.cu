// Setup of one model instance on the device: Gauss grid and Legendre tables,
// per-degree saddle-point operators assembled, equilibrated and LU-factored
// in the reference's dgbtf2 order, and the unit-load response (elastic gains
// and nodal U, V). Replaces build_sht + build_solver + response_init_ve
// (src/vilma_coupling.f90:252-318, src/vilma_response.f90:542-677).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

// ----------------------------------------------------------------- grid

// Gauss-Legendre nodes, north first (x descending), by Newton iteration on P_n.
static void gauss_nodes(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int k = 1; k <= n; ++k) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * k - 1.0) * z * p2 - (k - 1.0) * p3) / k;
      }
      double pp = n * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-16) break;
    }
    double p1 = 1.0, p2 = 0.0;
    for (int k = 1; k <= n; ++k) {
      double p3 = p2;
      p2 = p1;
      p1 = ((2.0 * k - 1.0) * z * p2 - (k - 1.0) * p3) / k;
    }
    double pp = n * (z * p1 - p2) / (z * z - 1.0);
    x[i] = z;
    x[n - 1 - i] = -z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    w[n - 1 - i] = w[i];
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
}

// Orthonormal associated Legendre functions without the Condon-Shortley phase
// and their theta derivative, one thread per (m, latitude): upward recurrence
// in l from the sectoral P_mm.
__global__ void k_legendre_tables(int lmax, int mmax, int nlat, const double* __restrict__ x,
                                  const double* __restrict__ sint, const int* __restrict__ mbeg,
                                  double* __restrict__ plm, double* __restrict__ dplm) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int m = blockIdx.y;
  if (j >= nlat || m > mmax) return;
  double xx = x[j], st = sint[j];
  double pmm = 1.0 / sqrt(4.0 * PI);
  for (int mm = 1; mm <= m; ++mm) pmm *= sqrt((2.0 * mm + 1.0) / (2.0 * mm)) * st;
  int lm0 = mbeg[m];
  double p2 = 0.0, p1 = pmm;
  plm[(size_t)lm0 * nlat + j] = pmm;
  for (int l = m + 1; l <= lmax; ++l) {
    double a = sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
    double b = sqrt((((double)(l - 1) * (l - 1)) - (double)m * m) / (4.0 * (l - 1) * (l - 1) - 1.0));
    double p = a * (xx * p1 - b * p2);
    plm[(size_t)(lm0 + l - m) * nlat + j] = p;
    p2 = p1;
    p1 = p;
  }
  for (int l = m; l <= lmax; ++l) {
    double p = plm[(size_t)(lm0 + l - m) * nlat + j];
    double pl1 = (l > m) ? plm[(size_t)(lm0 + l - m - 1) * nlat + j] : 0.0;
    double c = sqrt((2.0 * l + 1.0) * ((double)l * l - (double)m * m) / (2.0 * l - 1.0));
    dplm[(size_t)(lm0 + l - m) * nlat + j] = (l * xx * p - c * pl1) / st;
  }
}

void build_grid(Grid& G, int lmax, int nlat, int nphi, cudaStream_t s) {
  if (nphi <= 2 * lmax) throw Error("vg_create: nphi must exceed 2*lmax (m <= lmax needs nphi > 2 lmax)");
  if (nlat < lmax + 1) throw Error("vg_create: nlat must be >= lmax+1 for an exact Gauss quadrature");
  G.lmax = lmax;
  G.mmax = lmax;
  G.M = lmax + 1;
  G.nlat = nlat;
  G.nphi = nphi;
  G.ng = nlat * nphi;
  G.nlm = (lmax + 1) * (lmax + 2) / 2;
  gauss_nodes(nlat, G.x, G.wts);
  G.colat.resize(nlat);
  G.sint.resize(nlat);
  std::vector<double> cott(nlat), invsin(nlat);
  for (int j = 0; j < nlat; ++j) {
    G.colat[j] = std::acos(G.x[j]);
    G.sint[j] = std::sqrt((1.0 - G.x[j]) * (1.0 + G.x[j]));
    cott[j] = std::cos(G.colat[j]) / std::sin(G.colat[j]);
    invsin[j] = 1.0 / std::sin(G.colat[j]);
  }
  std::vector<int> lm_m(G.nlm), lm_l(G.nlm), mbeg(G.M + 1);
  for (int m = 0; m <= G.mmax; ++m) {
    mbeg[m] = m * (lmax + 1) - m * (m - 1) / 2;
    for (int l = m; l <= lmax; ++l) {
      lm_m[mbeg[m] + l - m] = m;
      lm_l[mbeg[m] + l - m] = l;
    }
  }
  mbeg[G.M] = G.nlm;
  std::vector<double> cs(nphi), sn(nphi);
  for (int t = 0; t < nphi; ++t) {
    cs[t] = std::cos(2.0 * PI * (double)t / (double)nphi);
    sn[t] = std::sin(2.0 * PI * (double)t / (double)nphi);
  }
  G.d_wts.upload(G.wts, s);
  G.d_sint.upload(G.sint, s);
  G.d_cott.upload(cott, s);
  G.d_invsin.upload(invsin, s);
  G.d_cos.upload(cs, s);
  G.d_sin.upload(sn, s);
  G.d_lm_m.upload(lm_m, s);
  G.d_lm_l.upload(lm_l, s);
  G.d_mbeg.upload(mbeg, s);
  DArr<double> d_x;
  d_x.upload(G.x, s);
  G.d_plm.alloc((size_t)G.nlm * nlat);
  G.d_dplm.alloc((size_t)G.nlm * nlat);
  dim3 grid((nlat + 63) / 64, G.M);
  k_legendre_tables<<<grid, 64, 0, s>>>(lmax, G.mmax, nlat, d_x.p, G.d_sint.p, G.d_mbeg.p, G.d_plm.p, G.d_dplm.p);
  VG_CUDA(cudaGetLastError());
  VG_CUDA(cudaStreamSynchronize(s));
}

// ------------------------------------------------------- radial operators

// Closed-form element integrals (Martinec 2000 App. C; src/vilma_radial_integrals.f90:28-126).
struct Elem {
  double i1[2][2], i2[2][2], i3[2][2], i4[2][2], i5[2][2], i6[2][2], i7[2][2], k1[2], k2[2];
};
__device__ __host__ inline void elem_integrals(double rk, double rk1, bool with_i7, Elem& E) {
  double h = rk1 - rk;
  double d = (rk1 * rk1 + rk1 * rk + rk * rk) / (3.0 * h);
  E.i1[0][0] = d;
  E.i1[0][1] = -d;
  E.i1[1][0] = -d;
  E.i1[1][1] = d;
  E.i2[0][0] = -(rk1 * rk1 + 2.0 * rk1 * rk + 3.0 * rk * rk) / 12.0;
  E.i2[0][1] = -E.i2[0][0];
  E.i2[1][1] = (3.0 * rk1 * rk1 + 2.0 * rk1 * rk + rk * rk) / 12.0;
  E.i2[1][0] = -E.i2[1][1];
  E.i3[0][0] = -(rk1 + 2.0 * rk) / 6.0;
  E.i3[0][1] = -E.i3[0][0];
  E.i3[1][1] = (2.0 * rk1 + rk) / 6.0;
  E.i3[1][0] = -E.i3[1][1];
  E.i4[0][0] = h / 30.0 * (rk1 * rk1 + 3.0 * rk1 * rk + 6.0 * rk * rk);
  E.i4[0][1] = h / 60.0 * (3.0 * rk1 * rk1 + 4.0 * rk1 * rk + 3.0 * rk * rk);
  E.i4[1][0] = E.i4[0][1];
  E.i4[1][1] = h / 30.0 * (6.0 * rk1 * rk1 + 3.0 * rk1 * rk + rk * rk);
  E.i5[0][0] = h / 12.0 * (rk1 + 3.0 * rk);
  E.i5[0][1] = h / 12.0 * (rk1 + rk);
  E.i5[1][0] = E.i5[0][1];
  E.i5[1][1] = h / 12.0 * (3.0 * rk1 + rk);
  E.i6[0][0] = h / 3.0;
  E.i6[0][1] = h / 6.0;
  E.i6[1][0] = h / 6.0;
  E.i6[1][1] = h / 3.0;
  if (with_i7) {
    double lg = log(rk1 / rk);
    E.i7[0][0] = (rk1 * rk1 / h * lg - 2.0 * rk1 + 0.5 * (rk1 + rk)) / h;
    E.i7[0][1] = (-rk1 * rk / h * lg + 0.5 * (rk1 + rk)) / h;
    E.i7[1][0] = E.i7[0][1];
    E.i7[1][1] = (rk * rk / h * lg - 2.0 * rk + 0.5 * (rk1 + rk)) / h;
  } else {
    E.i7[0][0] = E.i7[0][1] = E.i7[1][0] = E.i7[1][1] = 0.0;
  }
  E.k1[0] = -(rk1 * rk1 + rk1 * rk + rk * rk) / 3.0;
  E.k1[1] = -E.k1[0];
  E.k2[0] = h / 6.0 * (rk1 + 2.0 * rk);
  E.k2[1] = h / 6.0 * (2.0 * rk1 + rk);
}

// One element's 7x7 block of the per-degree operator (eqs 80-84,
// src/vilma_radial_fe.f90:318-395), local dof order [U1 V1 F1 U2 V2 F2 P].
__device__ __host__ inline void element_block(const Elem& E, double mu_k, double rho_k, double Rk, double Jr,
                                              double Al[7][7]) {
  const double fourpiG = 4.0 * PI * GRAV_G;
  const int lU[2] = {0, 3}, lV[2] = {1, 4}, lF[2] = {2, 5}, lP = 6;
  for (int a = 0; a < 7; ++a)
    for (int b = 0; b < 7; ++b) Al[a][b] = 0.0;
  for (int ia = 0; ia < 2; ++ia)
    for (int ib = 0; ib < 2; ++ib) {
      Al[lU[ib]][lU[ia]] += mu_k * (2.0 * E.i1[ia][ib]);
      Al[lV[ib]][lV[ia]] += mu_k * (Jr * E.i1[ia][ib]);
      Al[lV[ib]][lU[ia]] += mu_k * (Jr * E.i3[ia][ib]);
      Al[lV[ib]][lV[ia]] -= mu_k * (Jr * E.i3[ia][ib]);
      Al[lV[ib]][lV[ia]] -= mu_k * (Jr * E.i3[ib][ia]);
      Al[lU[ib]][lV[ia]] += mu_k * (Jr * E.i3[ib][ia]);
      Al[lU[ib]][lU[ia]] += mu_k * (Jr * E.i6[ia][ib]);
      Al[lU[ib]][lV[ia]] -= mu_k * (Jr * E.i6[ia][ib]);
      Al[lV[ib]][lU[ia]] -= mu_k * (Jr * E.i6[ia][ib]);
      Al[lV[ib]][lV[ia]] += mu_k * (Jr * E.i6[ia][ib]);
      Al[lU[ib]][lU[ia]] += mu_k * (4.0 * E.i6[ia][ib]);
      Al[lV[ib]][lU[ia]] -= mu_k * (2.0 * Jr * E.i6[ia][ib]);
      Al[lU[ib]][lV[ia]] -= mu_k * (2.0 * Jr * E.i6[ia][ib]);
      Al[lV[ib]][lV[ia]] += mu_k * (Jr * Jr * E.i6[ia][ib]);
      Al[lV[ib]][lV[ia]] += mu_k * (Jr * (Jr - 2.0) * E.i6[ia][ib]);
      double gg = (fourpiG / 3.0) * (rho_k * E.i4[ia][ib] + Rk * E.i7[ia][ib]);
      Al[lU[ib]][lU[ia]] += rho_k * (-4.0 * gg + fourpiG * rho_k * E.i4[ia][ib]);
      Al[lU[ib]][lV[ia]] += rho_k * (Jr * gg);
      Al[lU[ib]][lF[ia]] += rho_k * (E.i2[ib][ia]);
      Al[lV[ib]][lU[ia]] += rho_k * (Jr * gg);
      Al[lV[ib]][lF[ia]] += rho_k * (Jr * E.i5[ia][ib]);
      Al[lF[ib]][lF[ia]] += (E.i1[ia][ib] + Jr * E.i6[ia][ib]) / fourpiG;
      Al[lF[ib]][lU[ia]] += rho_k * (E.i2[ia][ib]);
      Al[lF[ib]][lV[ia]] += rho_k * (Jr * E.i5[ia][ib]);
    }
  for (int ia = 0; ia < 2; ++ia) {
    Al[lP][lU[ia]] += (E.k1[ia] + 2.0 * E.k2[ia]);
    Al[lU[ia]][lP] += (E.k1[ia] + 2.0 * E.k2[ia]);
    Al[lP][lV[ia]] -= (Jr * E.k2[ia]);
    Al[lV[ia]][lP] -= (Jr * E.k2[ia]);
  }
}

struct ElemData {
  const double* r;
  const double* mu;
  const double* rho;
  const double* Rk;
  int ne, nr, nd;
  double r_earth;
};

// Assemble the band part of degree l (>= 2) into raw band storage
// raw[(l, 6 + i - j, j)] (kl = ku = 6 by the node-interleaved layout),
// equilibrate (geometric-mean row/column scales, src/vilma_radial_fe.f90:497-538)
// and write the dgbtf2 band storage, then factor. One thread per degree; the
// arithmetic order matches the reference's serial assembly.
__device__ void band_factor_dev(double* ab, int ldab, int n, int kl, int ku, int* ipiv, int* ok) {
  const int kv = kl + ku;
#define AB(row1, col1) ab[(size_t)((col1)-1) * ldab + ((row1)-1)]
  int ju = 1;
  *ok = 1;
  for (int j = 1; j <= n; ++j) {
    if (j + kv <= n)
      for (int i = 1; i <= kl; ++i) AB(i, j + kv) = 0.0;
    int km = min(kl, n - j);
    int jp = 0;
    double piv = fabs(AB(kv + 1, j));
    for (int p = 1; p <= km; ++p)
      if (fabs(AB(kv + 1 + p, j)) > piv) {
        piv = fabs(AB(kv + 1 + p, j));
        jp = p;
      }
    ipiv[j - 1] = j + jp - 1;
    if (AB(kv + 1 + jp, j) == 0.0) {
      *ok = 0;
      return;
    }
    ju = max(ju, min(j + ku + jp, n));
    if (jp != 0)
      for (int jj = j; jj <= ju; ++jj) {
        double t = AB(kv + 1 + j - jj, jj);
        AB(kv + 1 + j - jj, jj) = AB(kv + 1 + j + jp - jj, jj);
        AB(kv + 1 + j + jp - jj, jj) = t;
      }
    if (km > 0) {
      double rp = 1.0 / AB(kv + 1, j);
      for (int p = 1; p <= km; ++p) AB(kv + 1 + p, j) *= rp;
      for (int jj = j + 1; jj <= ju; ++jj) {
        double t = AB(kv + 1 + j - jj, jj);
        if (t != 0.0)
          for (int p = 1; p <= km; ++p) AB(kv + 1 + j + p - jj, jj) -= AB(kv + 1 + p, j) * t;
      }
    }
  }
#undef AB
}

__global__ void k_build_band(ElemData ed, int lmax, double* __restrict__ raw, double* __restrict__ ab,
                             double* __restrict__ drv, double* __restrict__ dcv, int* __restrict__ ipiv,
                             double* __restrict__ rdg, int* __restrict__ status) {
  int l = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (l > lmax) return;
  const int n = ed.nd, KL = 6, NB = 13;
  double* R = raw + (size_t)(l - 2) * NB * n;  // R[(6 + i - j) * n + j], 0-based i, j
  for (size_t t = 0; t < (size_t)NB * n; ++t) R[t] = 0.0;
  const double Jr = (double)l * (double)(l + 1);
  for (int e = 0; e < ed.ne; ++e) {
    Elem E;
    elem_integrals(ed.r[e], ed.r[e + 1], ed.Rk[e] != 0.0, E);
    double Al[7][7];
    element_block(E, ed.mu[e], ed.rho[e], ed.Rk[e], Jr, Al);
    int gmap[7] = {4 * e, 4 * e + 1, 4 * e + 2, 4 * e + 4, 4 * e + 5, 4 * e + 6, 4 * e + 3};
    for (int b = 0; b < 7; ++b)
      for (int c = 0; c < 7; ++c) R[(size_t)(KL + gmap[b] - gmap[c]) * n + gmap[c]] += Al[b][c];
  }
  const double fourpiG = 4.0 * PI * GRAV_G;
  int fs = 4 * (ed.nr - 1) + 2;
  R[(size_t)KL * n + fs] += ed.r_earth / fourpiG * (double)(l + 1);
  double* dr = drv + (size_t)(l - 2) * n;
  double* dc = dcv + (size_t)(l - 2) * n;
  for (int k = 0; k < n; ++k) {
    double m = 0.0;
    for (int i = max(0, k - KL); i <= min(n - 1, k + KL); ++i) m = fmax(m, fabs(R[(size_t)(KL + i - k) * n + k]));
    dc[k] = m > 0.0 ? 1.0 / sqrt(m) : 1.0;
  }
  for (int i = 0; i < n; ++i) {
    double m = 0.0;
    for (int k = max(0, i - KL); k <= min(n - 1, i + KL); ++k)
      m = fmax(m, fabs(R[(size_t)(KL + i - k) * n + k] * dc[k]));
    dr[i] = m > 0.0 ? 1.0 / sqrt(m) : 1.0;
  }
  // dgbtf2 storage: ldab = 2 kl + ku + 1 = 19, A(i,j) at row kv + i - j (0-based), kv = 12
  const int ldab = VG_LDAB, kv = 12;
  double* A = ab + (size_t)(l - 2) * ldab * n;
  for (size_t t = 0; t < (size_t)ldab * n; ++t) A[t] = 0.0;
  for (int k = 0; k < n; ++k)
    for (int i = max(0, k - KL); i <= min(n - 1, k + KL); ++i) {
      double v = R[(size_t)(KL + i - k) * n + k];
      if (v != 0.0) A[(size_t)k * ldab + (kv + i - k)] = dr[i] * v * dc[k];
    }
  int ok;
  band_factor_dev(A, ldab, n, KL, KL, ipiv + (size_t)(l - 2) * n, &ok);
  if (!ok) {
    atomicExch(status, l);
    return;
  }
  // Two extra rows per column for the drift sweeps, so one column is one
  // contiguous record: row 19 = reciprocal pivot, row 20 = pivot offset jp.
  for (int j = 0; j < n; ++j) {
    A[(size_t)j * ldab + 19] = 1.0 / A[(size_t)j * ldab + kv];
    A[(size_t)j * ldab + 20] = (double)(ipiv[(size_t)(l - 2) * n + j] - j);
    rdg[(size_t)(l - 2) * n + j] = A[(size_t)j * ldab + 19];
  }
}

// Degree 1: band part plus the KKT border w (E_uniq weight, src/vilma_radial_fe.f90:425-443,
// 475-477), dense dgbtf2 with kl = ku = nd. Assembly by one thread, factor by the CTA.
__global__ void __launch_bounds__(512) k_build_deg1(ElemData ed, double* __restrict__ A /*dense nd x nd col-major scratch*/,
                             double* __restrict__ ab, int ldab, double* __restrict__ dr,
                             double* __restrict__ dc, double* __restrict__ w, int* __restrict__ ipiv,
                             int* __restrict__ status) {
  const int nd = ed.nd, ns = nd + 1, kl = nd, ku = nd, kv = kl + ku;
  __shared__ double s_dcb, s_drb;
  if (threadIdx.x == 0) {
    for (size_t t = 0; t < (size_t)nd * nd; ++t) A[t] = 0.0;
    const double Jr = 2.0;
    for (int e = 0; e < ed.ne; ++e) {
      Elem E;
      elem_integrals(ed.r[e], ed.r[e + 1], ed.Rk[e] != 0.0, E);
      double Al[7][7];
      element_block(E, ed.mu[e], ed.rho[e], ed.Rk[e], Jr, Al);
      int gmap[7] = {4 * e, 4 * e + 1, 4 * e + 2, 4 * e + 4, 4 * e + 5, 4 * e + 6, 4 * e + 3};
      for (int b = 0; b < 7; ++b)
        for (int c = 0; c < 7; ++c) A[(size_t)gmap[c] * nd + gmap[b]] += Al[b][c];
    }
    const double fourpiG = 4.0 * PI * GRAV_G;
    int fs = 4 * (ed.nr - 1) + 2;
    A[(size_t)fs * nd + fs] += ed.r_earth / fourpiG * 2.0;
    for (int i = 0; i < nd; ++i) w[i] = 0.0;
    for (int e = 0; e < ed.ne; ++e) {
      double rk = ed.r[e], rk1 = ed.r[e + 1], h = rk1 - rk;
      double k3a = h / 12.0 * (rk1 * rk1 + 2.0 * rk1 * rk + 3.0 * rk * rk);
      double k3b = h / 12.0 * (3.0 * rk1 * rk1 + 2.0 * rk1 * rk + rk * rk);
      w[4 * e] += k3a;
      w[4 * e + 4] += k3b;
      w[4 * e + 1] += 2.0 * k3a;
      w[4 * e + 5] += 2.0 * k3b;
    }
    // equilibration with the border folded into the maxima
    for (int k = 0; k < nd; ++k) {
      double m = 0.0;
      for (int i = 0; i < nd; ++i) m = fmax(m, fabs(A[(size_t)k * nd + i]));
      dc[k] = m > 0.0 ? 1.0 / sqrt(m) : 1.0;
      if (fabs(w[k]) > 1.0 / (dc[k] * dc[k])) dc[k] = 1.0 / sqrt(fabs(w[k]));
    }
    double m = 0.0;
    for (int i = 0; i < nd; ++i) m = fmax(m, fabs(w[i]));
    s_dcb = m > 0.0 ? 1.0 / sqrt(m) : 1.0;
    for (int i = 0; i < nd; ++i) {
      double mm = 0.0;
      for (int k = 0; k < nd; ++k) mm = fmax(mm, fabs(A[(size_t)k * nd + i] * dc[k]));
      dr[i] = mm > 0.0 ? 1.0 / sqrt(mm) : 1.0;
      if (fabs(w[i]) * s_dcb > 1.0 / (dr[i] * dr[i])) dr[i] = 1.0 / sqrt(fabs(w[i]) * s_dcb);
    }
    m = 0.0;
    for (int k = 0; k < nd; ++k) m = fmax(m, fabs(w[k] * dc[k]));
    s_drb = m > 0.0 ? 1.0 / sqrt(m) : 1.0;
  }
  __syncthreads();
  // scatter the scaled bordered matrix into dgbtf2 band storage (row kv + i - j)
  for (size_t t = threadIdx.x; t < (size_t)ldab * ns; t += blockDim.x) ab[t] = 0.0;
  __syncthreads();
  for (size_t t = threadIdx.x; t < (size_t)nd * nd; t += blockDim.x) {
    int i = (int)(t % nd), k = (int)(t / nd);
    double v = A[t];
    if (v != 0.0) ab[(size_t)k * ldab + (kv + i - k)] = dr[i] * v * dc[k];
  }
  for (int i = threadIdx.x; i < nd; i += blockDim.x) {
    if (w[i] != 0.0) {
      ab[(size_t)nd * ldab + (kv + i - nd)] = dr[i] * w[i] * s_dcb;   // border column
      ab[(size_t)i * ldab + (kv + nd - i)] = s_drb * w[i] * dc[i];    // border row
    }
  }
  __syncthreads();
  // dgbtf2, CTA-parallel over rows/columns of each rank-1 update
  __shared__ int s_jp, s_ju, s_fail;
  __shared__ double s_pv[1024];
  __shared__ int s_pi[1024];
  if (threadIdx.x == 0) {
    s_ju = 1;
    s_fail = 0;
  }
  __syncthreads();
#define AB(row1, col1) ab[(size_t)((col1)-1) * ldab + ((row1)-1)]
  for (int j = 1; j <= ns; ++j) {
    if (j + kv <= ns)
      for (int i = 1 + threadIdx.x; i <= kl; i += blockDim.x) AB(i, j + kv) = 0.0;
    int km = min(kl, ns - j);
    // pivot search: first index of the maximum, as the serial loop (strict >)
    double best = -1.0;
    int bi = 0;
    for (int p = threadIdx.x; p <= km; p += blockDim.x) {
      double v = fabs(AB(kv + 1 + p, j));
      if (v > best) {
        best = v;
        bi = p;
      }
    }
    s_pv[threadIdx.x] = best;
    s_pi[threadIdx.x] = bi;
    __syncthreads();
    if (threadIdx.x == 0) {
      // the serial loop keeps the first maximum (strict >): smallest index among ties
      double pv = s_pv[0];
      int pi = s_pi[0];
      for (int t = 1; t < (int)blockDim.x; ++t)
        if (s_pv[t] > pv || (s_pv[t] == pv && s_pi[t] < pi)) {
          pv = s_pv[t];
          pi = s_pi[t];
        }
      s_jp = pi;
      ipiv[j - 1] = j + pi - 1;
      if (AB(kv + 1 + pi, j) == 0.0) s_fail = 1;
      s_ju = max(s_ju, min(j + ku + pi, ns));
    }
    __syncthreads();
    if (s_fail) {
      if (threadIdx.x == 0) atomicExch(status, 1);
      return;
    }
    int jp = s_jp, ju = s_ju;
    if (jp != 0)
      for (int jj = j + threadIdx.x; jj <= ju; jj += blockDim.x) {
        double t = AB(kv + 1 + j - jj, jj);
        AB(kv + 1 + j - jj, jj) = AB(kv + 1 + j + jp - jj, jj);
        AB(kv + 1 + j + jp - jj, jj) = t;
      }
    __syncthreads();
    if (km > 0) {
      double rp = 1.0 / AB(kv + 1, j);
      for (int p = 1 + threadIdx.x; p <= km; p += blockDim.x) AB(kv + 1 + p, j) *= rp;
      __syncthreads();
      // rank-1 update, parallel over (p, jj); each entry sees the serial sequence of updates
      int ncol = ju - j;
      long long tot = (long long)ncol * km;
      for (long long t = threadIdx.x; t < tot; t += blockDim.x) {
        int jj = j + 1 + (int)(t / km), p = 1 + (int)(t % km);
        double u = AB(kv + 1 + j - jj, jj);
        if (u != 0.0) AB(kv + 1 + j + p - jj, jj) -= AB(kv + 1 + p, j) * u;
      }
    }
    __syncthreads();
  }
#undef AB
}

// Solve with one factored band system (dgbtrs order) for a column x with stride.

// unit surface load (sigma = 1) response for degrees >= 2, one thread per degree
__global__ void k_unit_load(int lmax, int nr, int n, double r_earth, double g_surf, const double* __restrict__ ab,
                            const double* __restrict__ drv, const double* __restrict__ dcv,
                            const int* __restrict__ ipiv, double* __restrict__ xs, double* __restrict__ gu,
                            double* __restrict__ gn, double* __restrict__ gv, double* __restrict__ xUn,
                            double* __restrict__ xVn) {
  int l = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (l > lmax) return;
  double* x = xs + (size_t)(l - 2) * n;
  const double* dr = drv + (size_t)(l - 2) * n;
  const double* dc = dcv + (size_t)(l - 2) * n;
  for (int i = 0; i < n; ++i) x[i] = 0.0;
  x[4 * (nr - 1)] = dr[4 * (nr - 1)] * (-r_earth * r_earth * 1.0 * g_surf);
  x[4 * (nr - 1) + 2] = dr[4 * (nr - 1) + 2] * (-r_earth * r_earth * 1.0);
  band_solve_strided(ab + (size_t)(l - 2) * VG_LDAB * n, VG_LDAB, n, 6, 12, ipiv + (size_t)(l - 2) * n, x, 1);
  for (int i = 0; i < n; ++i) x[i] = dc[i] * x[i];
  gu[l] = x[4 * (nr - 1)];
  gn[l] = -x[4 * (nr - 1) + 2] / g_surf;
  gv[l] = x[4 * (nr - 1) + 1];
  for (int node = 0; node < nr; ++node) {
    xUn[(size_t)l * nr + node] = x[4 * node];
    xVn[(size_t)l * nr + node] = x[4 * node + 1];
  }
}

// degree-1 unit-load response (with the CM-frame projection) and null mode
__global__ void __launch_bounds__(512) k_unit_load_deg1(int nr, int nd, double r_earth, double g_surf, int deg1_cm,
                                 const double* __restrict__ ab, int ldab, int kl, int kv, const int* __restrict__ ipiv,
                                 const double* __restrict__ dr, const double* __restrict__ dc,
                                 double* __restrict__ nullmode, double* __restrict__ gu, double* __restrict__ gn,
                                 double* __restrict__ gv, double* __restrict__ xUn, double* __restrict__ xVn) {
  extern __shared__ double xsh[];  // [2][ns]
  const int ns = nd + 1;
  for (int i = threadIdx.x; i < 2 * ns; i += blockDim.x) xsh[i] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) {
    xsh[4 * (nr - 1)] = dr[4 * (nr - 1)] * (-r_earth * r_earth * 1.0 * g_surf);
    xsh[4 * (nr - 1) + 2] = dr[4 * (nr - 1) + 2] * (-r_earth * r_earth * 1.0);
    xsh[ns + nd] = 1.0;  // null mode: zero physical RHS, border value 1
  }
  __syncthreads();
  deg1_solve_cta(ab, ldab, ns, kl, kv, ipiv, xsh, 2);
  for (int i = threadIdx.x; i < nd; i += blockDim.x) {
    xsh[i] = dc[i] * xsh[i];
    xsh[ns + i] = dc[i] * xsh[ns + i];
    nullmode[i] = xsh[ns + i];
  }
  __syncthreads();
  if (deg1_cm) {
    int fs = 4 * (nr - 1) + 2;
    double fa_n = xsh[ns + fs];
    if (fa_n != 0.0) {
      double c = -xsh[fs] / fa_n;
      __syncthreads();
      for (int i = threadIdx.x; i < nd; i += blockDim.x) xsh[i] = xsh[i] + c * xsh[ns + i];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    gu[1] = xsh[4 * (nr - 1)];
    gn[1] = deg1_cm ? -xsh[4 * (nr - 1) + 2] / g_surf : 0.0;
    gv[1] = xsh[4 * (nr - 1) + 1];
  }
  for (int node = threadIdx.x; node < nr; node += blockDim.x) {
    xUn[(size_t)nr + node] = xsh[4 * node];
    xVn[(size_t)nr + node] = xsh[4 * node + 1];
  }
}

// Degree-1 response block G1 = Dc Ahat^-1 restricted to the rows the drift
// needs (U and V of every node, then F at the surface: r = 2 node + {0,1},
// r = 2 nr) and to the columns the dissipative forcing can reach (U and V of
// every node: c = 2 node + {0,1}), in the equilibrated-RHS space. One thread
// per column solves the bordered system (dgbtrs order) for a unit RHS.
__global__ void k_deg1_green(int nr, int nd, const double* __restrict__ ab, int ldab, int kl, int kv,
                             const int* __restrict__ ipiv, const double* __restrict__ dc,
                             double* __restrict__ scratch, double* __restrict__ G1) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int ncol = 2 * nr, ns = nd + 1;
  if (c >= ncol) return;
  double* x = scratch + (size_t)c * ns;
  for (int i = 0; i < ns; ++i) x[i] = 0.0;
  x[4 * (c / 2) + (c % 2)] = 1.0;
#define AB(row1, col1) ab[(size_t)((col1)-1) * ldab + ((row1)-1)]
  for (int j = 1; j <= ns - 1; ++j) {
    int lm = min(kl, ns - j);
    int l = ipiv[j - 1] + 1;
    if (l != j) {
      double t = x[l - 1];
      x[l - 1] = x[j - 1];
      x[j - 1] = t;
    }
    double t = x[j - 1];
    if (t != 0.0)
      for (int i = 1; i <= lm; ++i) x[j + i - 1] -= AB(kv + 1 + i, j) * t;
  }
  for (int j = ns; j >= 1; --j) {
    double xj = x[j - 1] / AB(kv + 1, j);
    x[j - 1] = xj;
    int lm = min(kv, j - 1);
    if (xj != 0.0)
      for (int i = 1; i <= lm; ++i) x[j - i - 1] -= AB(kv + 1 - i, j) * xj;
  }
#undef AB
  for (int node = 0; node < nr; ++node) {
    G1[(size_t)(2 * node) * ncol + c] = dc[4 * node] * x[4 * node];
    G1[(size_t)(2 * node + 1) * ncol + c] = dc[4 * node + 1] * x[4 * node + 1];
  }
  int fs = 4 * (nr - 1) + 2;
  G1[(size_t)(2 * nr) * ncol + c] = dc[fs] * x[fs];
}

// Dissipative forcing as a linear map of one element's memory: the 2-point
// Gauss quadrature of dissipative_rhs (src/vilma_viscoelastic.f90:441-480)
// folded into K[t][s][m] with floc_t = sum_{s,m} K[t][s][m] mem_s[m] for the
// test dofs t = (U_e, U_e+1, V_e, V_e+1), shape coefficients s = (A, B, C) and
// channels m. One thread per (degree, element).
__global__ void k_rhs_coeffs(int lmax, int ne, const double* __restrict__ r, const double* __restrict__ sa,
                             const double* __restrict__ sb, const double* __restrict__ sc,
                             const double* __restrict__ nrmc, double* __restrict__ K) {
  int e = blockIdx.x * blockDim.x + threadIdx.x, l = blockIdx.y + 1;
  if (e >= ne || l > lmax) return;
  const double xg = 0.5773502691896257;
  double rk = r[e], rk1 = r[e + 1], h = rk1 - rk;
  double acc[4][3][4] = {};
  for (int ig = 0; ig < 2; ++ig) {
    double ra = 0.5 * (h * (ig ? xg : -xg) + rk + rk1);
    double psik = (rk1 - ra) / h, psik1 = (ra - rk) / h;
    double w = ra * ra * h * 0.5;
    double basis[3] = {1.0 / h, psik / ra, psik1 / ra};
    for (int t = 0; t < 4; ++t)
      for (int m = 0; m < 4; ++m) {
        double deps = sa[l * 16 + t * 4 + m] / h + sb[l * 16 + t * 4 + m] * psik / ra + sc[l * 16 + t * 4 + m] * psik1 / ra;
        double c = w * nrmc[l * 4 + m] * deps;
        for (int s3 = 0; s3 < 3; ++s3) acc[t][s3][m] -= c * basis[s3];
      }
  }
  double* out = K + ((size_t)l * ne + e) * 48;
  for (int t = 0; t < 4; ++t)
    for (int s3 = 0; s3 < 3; ++s3)
      for (int m = 0; m < 4; ++m) out[(t * 3 + s3) * 4 + m] = acc[t][s3][m];
}

// ----------------------------------------------------------------- setup

static double mass_below(const vg_params& p, double r) {
  double m = 0.0;
  for (int i = 0; i < p.n_layer; ++i) {
    double lo = p.r_bot[i], hi = std::min(p.r_top[i], r);
    if (hi > lo) m += (4.0 / 3.0) * PI * p.rho[i] * (hi * hi * hi - lo * lo * lo);
  }
  return m;
}

// src/vilma_radial_fe.f90:153-224 (with the optional per-layer element counts)
static void build_mesh(vg_handle* h) {
  const vg_params& p = h->p;
  const int nl = p.n_layer;
  if (nl < 1 || nl > VG_MAX_LAYER) throw Error("vg_create: n_layer out of range");
  if (std::fabs(p.r_top[0] - p.r_earth) > 1.0)
    throw Error("radial_mesh_build: r_top(1) must equal r_earth (layers are surface-first)");
  if (p.r_bot[nl - 1] != 0.0) throw Error("radial_mesh_build: the innermost layer must reach r = 0");
  for (int i = 0; i < nl; ++i) {
    if (p.r_top[i] <= p.r_bot[i]) throw Error("radial_mesh_build: every layer needs r_top > r_bot");
    if (i < nl - 1 && std::fabs(p.r_bot[i] - p.r_top[i + 1]) > 1.0)
      throw Error("radial_mesh_build: layers must be contiguous, r_bot(k) = r_top(k+1)");
  }
  bool expl = false;
  for (int i = 0; i < nl; ++i) expl |= p.ne_layer[i] > 0;
  auto dr_target = [](double depth) { return depth <= 70.0e3 ? 5.0e3 : (depth <= 670.0e3 ? 10.0e3 : 40.0e3); };
  auto count = [&](int i) {
    if (expl) return std::max(1, p.ne_layer[i]);
    double depth_mid = p.r_earth - 0.5 * (p.r_bot[i] + p.r_top[i]);
    return std::max(1, (int)std::ceil((p.r_top[i] - p.r_bot[i]) / dr_target(depth_mid)));
  };
  int ntot = 0;
  for (int i = 0; i < nl; ++i) ntot += count(i);
  h->ne = ntot;
  h->nr = ntot + 1;
  h->r.assign(h->nr, 0.0);
  h->elem_layer.assign(h->ne, 0);
  int off = 0;
  for (int i = nl - 1; i >= 0; --i) {
    int nel = count(i);
    double hh = (p.r_top[i] - p.r_bot[i]) / (double)nel;
    for (int k = 1; k <= nel; ++k) {
      h->r[off + k] = p.r_bot[i] + (double)k * hh;
      h->elem_layer[off + k - 1] = i;
    }
    off += nel;
  }
  h->r[h->nr - 1] = p.r_earth;
}

// Degree-2 band operator of the handle's earth with every Maxwell element
// fluidised (mu = 0; elastic and fluid elements unchanged), factored like the
// response's own bands: the relaxed tidal limit k^T_f of the rotational
// feedback (fluid_tidal_k, src/vilma_rotation.f90:342-371). Setup only.
void build_fluid_deg2_band(vg_handle* h, DArr<double>& ab, DArr<double>& dr, DArr<double>& dc, DArr<int>& ipiv) {
  const vg_params& p = h->p;
  cudaStream_t s = h->stream;
  const int ne = h->ne, nr = h->nr, nd = h->ndof;
  std::vector<double> mu(ne), rho(ne), Rk(ne, 0.0);
  for (int e = 0; e < ne; ++e) {
    int L = h->elem_layer[e];
    mu[e] = p.rheology[L] == VG_RHEOL_MAXWELL ? 0.0 : p.mu[L];
    rho[e] = p.rho[L];
  }
  for (int k = 1; k < ne; ++k) Rk[k] = Rk[k - 1] + (rho[k - 1] - rho[k]) * std::pow(h->r[k], 3);
  DArr<double> d_mu, d_rho, d_Rk, raw, rdg;
  DArr<int> status;
  d_mu.upload(mu, s);
  d_rho.upload(rho, s);
  d_Rk.upload(Rk, s);
  ElemData ed{h->d_r.p, d_mu.p, d_rho.p, d_Rk.p, ne, nr, nd, p.r_earth};
  raw.alloc((size_t)13 * nd);
  rdg.alloc(nd);
  status.alloc(1);
  ab.alloc((size_t)VG_LDAB * nd);
  dr.alloc(nd);
  dc.alloc(nd);
  ipiv.alloc(nd);
  k_build_band<<<1, 32, 0, s>>>(ed, 2, raw.p, ab.p, dr.p, dc.p, ipiv.p, rdg.p, status.p);
  VG_CUDA(cudaGetLastError());
  int st = 0;
  status.download(&st, 1, s);
  VG_CUDA(cudaStreamSynchronize(s));
  if (st) throw Error("rotation_init: fluid-limit degree-2 factorization failed (zero pivot)");
}

// The toroidal W operator of degree j (src/vilma_radial_fe.f90:699-729),
// symmetric tridiagonal: per element mu_k { J [I1 - I3(b,a) - I3(a,b) + I6]
// + J(J-2) I6 } W^a dW^b into diag (nr) and off (nr - 1, row i column i + 1).
// Nodes all of whose elements have mu = 0 carry no W: their rows and columns
// stay empty, and dead[i] says so (toroidal_dead_nodes, :731-743).
void toroidal_tridiag(const std::vector<double>& r, const std::vector<double>& mu, int j, std::vector<double>& diag,
                      std::vector<double>& off, std::vector<char>& dead) {
  const int nr = (int)r.size(), ne = (int)mu.size();
  const double Jr = (double)j * (double)(j + 1);
  diag.assign(nr, 0.0);
  off.assign(std::max(nr - 1, 0), 0.0);
  dead.assign(nr, 1);
  for (int e = 0; e < ne; ++e) {
    if (mu[e] == 0.0) continue;
    dead[e] = dead[e + 1] = 0;
    Elem E;
    elem_integrals(r[e], r[e + 1], false, E);
    double v[2][2];  // [trial a][test b]
    for (int ia = 0; ia < 2; ++ia)
      for (int ib = 0; ib < 2; ++ib)
        v[ia][ib] = mu[e] * (Jr * (E.i1[ia][ib] - E.i3[ib][ia] - E.i3[ia][ib] + E.i6[ia][ib]) +
                             Jr * (Jr - 2.0) * E.i6[ia][ib]);
    diag[e] += v[0][0];
    diag[e + 1] += v[1][1];
    off[e] += v[1][0];  // row e (test b = 0), column e + 1 (trial a = 1)
  }
}

// Degree-1 net-rotation constraints, one column per solid shell (a maximal run
// of mu > 0 elements): w_s(k) = sum_{e in s} int psi_k r^3 dr
// (rotation_weights, src/vilma_radial_fe.f90:745-773; elem_k4,
// src/vilma_radial_integrals.f90:117-126). Column-major (nr, nshell).
std::vector<double> toroidal_rotation_weights(const std::vector<double>& r, const std::vector<double>& mu,
                                              int& nshell) {
  const int nr = (int)r.size(), ne = (int)mu.size();
  std::vector<int> shell(ne, -1);
  int ns = 0;
  bool prev = false;
  for (int e = 0; e < ne; ++e) {
    const bool solid = mu[e] > 0.0;
    if (solid && !prev) ++ns;
    if (solid) shell[e] = ns - 1;
    prev = solid;
  }
  std::vector<double> w((size_t)nr * ns, 0.0);
  for (int e = 0; e < ne; ++e) {
    if (shell[e] < 0) continue;
    const double rk = r[e], rk1 = r[e + 1], h = rk1 - rk;
    w[(size_t)shell[e] * nr + e] += h / 20.0 * (rk1 * rk1 * rk1 + 2.0 * rk1 * rk1 * rk + 3.0 * rk1 * rk * rk +
                                                4.0 * rk * rk * rk);
    w[(size_t)shell[e] * nr + e + 1] += h / 20.0 * (4.0 * rk1 * rk1 * rk1 + 3.0 * rk1 * rk1 * rk +
                                                    2.0 * rk1 * rk * rk + rk * rk * rk);
  }
  nshell = ns;
  return w;
}

void setup_handle(vg_handle* h) {
  const vg_params& p = h->p;
  if (p.scheme != VG_SCHEME_FE && p.scheme != VG_SCHEME_TRAP)
    throw Error("vg_create: the memory scheme must be \"fe\" (VG_SCHEME_FE) or \"trap\" (VG_SCHEME_TRAP)");
  if (p.lmax < 2) throw Error("vg_create: lmax must be >= 2");
  if (p.visc3d_precision != VG_VISC3D_FP64 && p.visc3d_precision != VG_VISC3D_SPLIT_TC &&
      p.visc3d_precision != VG_VISC3D_EXACT_TC)
    throw Error("vg_create: visc3d_precision must be VG_VISC3D_FP64, VG_VISC3D_SPLIT_TC or VG_VISC3D_EXACT_TC");
  cudaStream_t s = h->stream;
  build_grid(h->grid, p.lmax, p.nlat, p.nphi, s);
  build_mesh(h);
  const int lmax = p.lmax, nr = h->nr, ne = h->ne;
  h->ndof = 4 * nr - 1;
  const int nd = h->ndof;
  h->a = p.r_earth;
  h->g = GRAV_G * mass_below(p, p.r_earth) / (p.r_earth * p.r_earth);
  h->dt = p.dt_init > 0.0 ? p.dt_init : KYR;
  // element fields
  std::vector<double> rho(ne), Rk(ne, 0.0);
  h->mu.assign(ne, 0.0);
  h->MkPerDt.assign(ne, 0.0);
  h->active1d_h.assign(ne, 1);
  for (int e = 0; e < ne; ++e) {
    int L = h->elem_layer[e];
    h->mu[e] = p.mu[L];
    rho[e] = p.rho[L];
    if (p.rheology[L] == VG_RHEOL_MAXWELL) h->MkPerDt[e] = h->mu[e] / p.eta[L];
  }
  for (int k = 1; k < ne; ++k) Rk[k] = Rk[k - 1] + (rho[k - 1] - rho[k]) * std::pow(h->r[k], 3);
  h->max_rate = 0.0;
  for (double v : h->MkPerDt) h->max_rate = std::max(h->max_rate, v);
  h->d_r.upload(h->r, s);
  h->d_mu.upload(h->mu, s);
  h->d_MkPerDt.upload(h->MkPerDt, s);
  h->d_active1d.upload(h->active1d_h, s);
  DArr<double> d_rho, d_Rk;
  d_rho.upload(rho, s);
  d_Rk.upload(Rk, s);
  ElemData ed{h->d_r.p, h->d_mu.p, d_rho.p, d_Rk.p, ne, nr, nd, p.r_earth};
  // band operators for l >= 2
  h->kl = h->ku = 6;
  h->kv = 12;
  h->ldab = VG_LDAB;
  DArr<double> raw;
  DArr<int> status;
  raw.alloc((size_t)(lmax - 1) * 13 * nd);
  status.alloc(1);
  h->d_ab.alloc((size_t)(lmax - 1) * VG_LDAB * nd);
  h->d_dr.alloc((size_t)(lmax - 1) * nd);
  h->d_dc.alloc((size_t)(lmax - 1) * nd);
  h->d_ipiv.alloc((size_t)(lmax - 1) * nd);
  h->d_rdiag.alloc((size_t)(lmax - 1) * nd);
  k_build_band<<<(lmax - 1 + 31) / 32, 32, 0, s>>>(ed, lmax, raw.p, h->d_ab.p, h->d_dr.p, h->d_dc.p, h->d_ipiv.p,
                                                    h->d_rdiag.p, status.p);
  VG_CUDA(cudaGetLastError());
  // degree 1 (bordered, dense)
  h->ns1 = nd + 1;
  h->kl1 = nd;
  h->kv1 = 2 * nd;
  h->ldab1 = 3 * nd + 1;
  DArr<double> Adense, w;
  Adense.alloc((size_t)nd * nd);
  w.alloc(nd);
  h->d_ab1.alloc((size_t)h->ldab1 * h->ns1);
  h->d_dr1.alloc(nd);
  h->d_dc1.alloc(nd);
  h->d_ipiv1.alloc(h->ns1);
  h->d_null1.alloc(nd);
  k_build_deg1<<<1, 512, 0, s>>>(ed, Adense.p, h->d_ab1.p, h->ldab1, h->d_dr1.p, h->d_dc1.p, w.p, h->d_ipiv1.p,
                                  status.p);
  VG_CUDA(cudaGetLastError());
  int st = 0;
  status.download(&st, 1, s);
  VG_CUDA(cudaStreamSynchronize(s));
  if (st) throw Error("bordered_band_factor: band LU factorization failed (zero pivot)");
  // per-degree constants (ve_strain_constants, src/vilma_viscoelastic.f90:361-371)
  std::vector<double> Jr(lmax + 1, 0.0), nrmc((lmax + 1) * 4, 0.0), sa((lmax + 1) * 16, 0.0), sb = sa, sc = sa;
  for (int l = 1; l <= lmax; ++l) {
    double J = (double)l * (double)(l + 1);
    Jr[l] = J;
    nrmc[l * 4 + 0] = 1.0;
    nrmc[l * 4 + 1] = 0.5 * J;
    nrmc[l * 4 + 2] = 2.0 * J * J;
    nrmc[l * 4 + 3] = 2.0 * J * (J - 2.0);
    for (int t = 0; t < 4; ++t) {
      double u1 = t == 0, u2 = t == 1, v1 = t == 2, v2 = t == 3;
      double* A = &sa[l * 16 + t * 4];
      double* B = &sb[l * 16 + t * 4];
      double* Cc = &sc[l * 16 + t * 4];
      A[0] = -u1 + u2;
      B[0] = 0.0;
      Cc[0] = 0.0;
      A[1] = -v1 + v2;
      B[1] = u1 - v1;
      Cc[1] = u2 - v2;
      A[2] = 0.0;
      B[2] = -u1 / J + 0.5 * v1;
      Cc[2] = -u2 / J + 0.5 * v2;
      A[3] = 0.0;
      B[3] = 0.5 * v1;
      Cc[3] = 0.5 * v2;
      if (J <= 2.0) {
        B[3] = 0.0;
        Cc[3] = 0.0;
      }
    }
  }
  h->d_Jr.upload(Jr, s);
  h->d_nrmc.upload(nrmc, s);
  h->d_sa.upload(sa, s);
  h->d_sb.upload(sb, s);
  h->d_sc.upload(sc, s);
  h->d_Krhs.alloc((size_t)(lmax + 1) * ne * 48);
  {
    dim3 g((ne + 63) / 64, lmax);
    k_rhs_coeffs<<<g, 64, 0, s>>>(lmax, ne, h->d_r.p, h->d_sa.p, h->d_sb.p, h->d_sc.p, h->d_nrmc.p, h->d_Krhs.p);
    VG_CUDA(cudaGetLastError());
  }
  // unit-load response
  h->d_gu.alloc(lmax + 1);
  h->d_gn.alloc(lmax + 1);
  h->d_gv.alloc(lmax + 1);
  h->d_xUn.alloc((size_t)(lmax + 1) * nr);
  h->d_xVn.alloc((size_t)(lmax + 1) * nr);
  DArr<double> xs;
  xs.alloc((size_t)(lmax - 1) * nd);
  k_unit_load<<<(lmax - 1 + 31) / 32, 32, 0, s>>>(lmax, nr, nd, p.r_earth, h->g, h->d_ab.p, h->d_dr.p, h->d_dc.p,
                                                   h->d_ipiv.p, xs.p, h->d_gu.p, h->d_gn.p, h->d_gv.p, h->d_xUn.p,
                                                   h->d_xVn.p);
  VG_CUDA(cudaGetLastError());
  size_t shm = 2 * (size_t)h->ns1 * sizeof(double);
  if (shm > 48 * 1024) raise_smem_limit((const void*)k_unit_load_deg1, shm);
  k_unit_load_deg1<<<1, 512, shm, s>>>(nr, nd, p.r_earth, h->g, p.deg1_cm, h->d_ab1.p, h->ldab1, h->kl1, h->kv1,
                                       h->d_ipiv1.p, h->d_dr1.p, h->d_dc1.p, h->d_null1.p, h->d_gu.p, h->d_gn.p,
                                       h->d_gv.p, h->d_xUn.p, h->d_xVn.p);
  VG_CUDA(cudaGetLastError());
  {  // degree-1 response block for the drift
    DArr<double> scratch;
    scratch.alloc((size_t)2 * nr * h->ns1);
    h->d_G1.alloc((size_t)(2 * nr + 1) * 2 * nr);
    k_deg1_green<<<(2 * nr + 63) / 64, 64, 0, s>>>(nr, nd, h->d_ab1.p, h->ldab1, h->kl1, h->kv1, h->d_ipiv1.p,
                                                  h->d_dc1.p, scratch.p, h->d_G1.p);
    VG_CUDA(cudaGetLastError());
    VG_CUDA(cudaStreamSynchronize(s));
  }
  // degree 0: monopole geoid (src/vilma_response.f90:603-605)
  double gn0 = 4.0 * PI * GRAV_G * h->a / h->g, zero = 0.0;
  VG_CUDA(cudaMemcpyAsync(h->d_gn.p, &gn0, sizeof(double), cudaMemcpyHostToDevice, s));
  VG_CUDA(cudaMemcpyAsync(h->d_gu.p, &zero, sizeof(double), cudaMemcpyHostToDevice, s));
  VG_CUDA(cudaMemcpyAsync(h->d_gv.p, &zero, sizeof(double), cudaMemcpyHostToDevice, s));
  // slot maps (src/vilma_response.f90:629-648)
  h->nk = 0;
  for (int l = 1; l <= lmax; ++l) h->nk += l + 1;
  const int nk = h->nk;
  h->kdeg_h.assign(nk, 0);
  h->k2lm_h.assign(nk, 0);
  h->kbeg_h.assign(lmax + 2, 0);
  std::vector<int> lm2k(h->grid.nlm, -1);
  int k = 0;
  for (int l = 1; l <= lmax; ++l) {
    h->kbeg_h[l] = k;
    for (int m = 0; m <= l; ++m) {
      int lm = m * (lmax + 1) - m * (m - 1) / 2 + (l - m);
      h->k2lm_h[k] = lm;
      h->kdeg_h[k] = l;
      lm2k[lm] = k;
      ++k;
    }
  }
  h->kbeg_h[lmax + 1] = k;
  h->d_kdeg.upload(h->kdeg_h, s);
  h->d_k2lm.upload(h->k2lm_h, s);
  h->d_lm2k.upload(lm2k, s);
  {  // drift sweep tasks: one warp = up to 16 slots of ONE degree (x re/im = 32 lanes)
    std::vector<int4> tasks;
    for (int l = 2; l <= lmax; ++l)
      for (int s0 = 0; s0 < l + 1; s0 += 16) tasks.push_back(make_int4(l, h->kbeg_h[l] + s0, std::min(16, l + 1 - s0), 0));
    h->ntask = (int)tasks.size();
    h->d_tasks.upload(tasks, s);
  }
  // state and work buffers
  const size_t nmem = (size_t)6 * ne * 4 * nk;
  h->d_mem[0].alloc(nmem);
  h->d_mem[1].alloc(nmem);
  h->cur = 0;
  h->d_dUn.alloc((size_t)2 * nr * nk);
  h->d_dVn.alloc((size_t)2 * nr * nk);
  h->d_drift.alloc((size_t)6 * nk);
  h->d_mnorm.alloc((size_t)2 * nk);
  h->d_maxbits.alloc(3);  // two buffer norms + kernel status bits
  h->d_xs.alloc((size_t)2 * nd * nk);
  h->d_bh.alloc((size_t)2 * 2 * nr * nk);
  h->d_sc_.alloc(1);
  VG_CUDA(cudaMallocHost(&h->h_sc, sizeof(SleScalars)));
  std::memset(h->h_sc, 0, sizeof(SleScalars));
  const int ng = h->grid.ng, M = h->grid.M, nlat = h->grid.nlat;
  for (DArr<double>* a : {&h->d_z_bed_eq, &h->d_h_ice_eq, &h->d_h_ice, &h->d_ice1, &h->d_ice_now, &h->d_dice_now,
                          &h->d_rsl, &h->d_rsl_n, &h->d_C, &h->d_C0, &h->d_C_next, &h->d_dig, &h->d_wcorr,
                          &h->d_Sraw, &h->d_zbed, &h->d_tmp})
    a->alloc(ng);
  h->d_F.alloc((size_t)2 * M * nlat * 2);
  h->d_Gs.alloc((size_t)2 * M * nlat * 2);
  h->d_sigma.alloc((size_t)2 * h->grid.nlm);
  h->d_ulm.alloc((size_t)2 * h->grid.nlm * 2);
  h->d_nlm.alloc((size_t)2 * h->grid.nlm);
  h->d_rowpart.alloc((size_t)8 * nlat);
  VG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace vg
