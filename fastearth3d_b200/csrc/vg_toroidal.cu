// The toroidal degree of freedom (l_toroidal; src/vilma_response.f90:126-146,
// 679-809, 944-992, 1055-1118; src/vilma_viscoelastic.f90:373-439, 591-629;
// src/vilma_radial_fe.f90:699-810).
//
// A laterally varying viscosity drives toroidal flow u = W(r) e_r x grad_1 Y
// through the pointwise M(theta, phi) tau product; once a genuinely 3-D element
// exists (and p.toroidal is set) the response carries W as pure drift (nothing
// loads it) and the lambda 3, 4 memory beside the spheroidal lambda 1, 2, 5, 6:
//   memory     tmem[buf][((s*2 + ri)*ne + e)*2 + lam][k], double-buffered with
//              the spheroidal state (same current buffer)
//   drift      per (l, m): the dissipative forcing -int tau^V : d eps on the
//              nodal W test dofs, then the degree's W operator: symmetric
//              tridiagonal for l >= 2 (dead nodes pinned to zero), bordered by
//              one net-rotation constraint per solid shell at l = 1
//   advance    the lambda 3, 4 Maxwell update of the spectrally advanced
//              elements from the strain of W (the 3-D elements go through the
//              six-channel pseudo-spectral advance of vg_visc3d.cu)
//
// The operators are factored once on the host at enable time: l >= 2 as a
// Thomas factorisation (the system is symmetric positive definite on the live
// nodes, so no pivoting; a pinned node has 1/pivot = 0, which zeroes its W),
// l = 1 as the explicit solution map G1W (nr x nr) of the bordered system,
// equilibrated and solved by partial-pivoting elimination.
// Kernels:
//   k_drift_tor     one thread per (slot, re/im): forcing and forward sweep in
//                   one pass over the elements (the sweep output y goes
//                   through the W target, coalesced along the slot), then the
//                   back substitution; degree 1 leaves the raw forcing there
//   k_drift_tor1    degree 1: W = G1W g for its two slots
//   k_advance_1d_tor  one thread per (slot, element, re/im), like k_advance_1d
#include <algorithm>
#include <cmath>
#include <cstring>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

// ------------------------------------------------------------------ setup

// Dense solve of the degree-1 bordered W system for every unit forcing of a
// live node: G1W[i][j] = W_i for g = e_j (pinned columns stay zero).
static std::vector<double> degree1_solution_map(const std::vector<double>& diag, const std::vector<double>& off,
                                                const std::vector<char>& dead, const std::vector<double>& w, int nr,
                                                int ns) {
  const int n = nr + ns;
  std::vector<double> K((size_t)n * n, 0.0);  // row-major
  for (int i = 0; i < nr; ++i) {
    K[(size_t)i * n + i] = dead[i] ? 1.0 : diag[i];
    if (i + 1 < nr) {
      K[(size_t)i * n + i + 1] = off[i];
      K[(size_t)(i + 1) * n + i] = off[i];
    }
  }
  for (int b = 0; b < ns; ++b)
    for (int i = 0; i < nr; ++i) {
      K[(size_t)i * n + nr + b] = w[(size_t)b * nr + i];
      K[(size_t)(nr + b) * n + i] = w[(size_t)b * nr + i];
    }
  // equilibrate: columns, then rows, by their largest entries
  std::vector<double> dc(n, 1.0), dr(n, 1.0);
  for (int c = 0; c < n; ++c) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) m = std::max(m, std::fabs(K[(size_t)i * n + c]));
    dc[c] = m > 0.0 ? 1.0 / m : 1.0;
  }
  for (int i = 0; i < n; ++i) {
    double m = 0.0;
    for (int c = 0; c < n; ++c) m = std::max(m, std::fabs(K[(size_t)i * n + c] * dc[c]));
    dr[i] = m > 0.0 ? 1.0 / m : 1.0;
  }
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < n; ++c) K[(size_t)i * n + c] *= dr[i] * dc[c];
  // LU with partial pivoting
  std::vector<int> piv(n);
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int i = c + 1; i < n; ++i)
      if (std::fabs(K[(size_t)i * n + c]) > std::fabs(K[(size_t)p * n + c])) p = i;
    if (K[(size_t)p * n + c] == 0.0) throw Error("toroidal operator: the degree-1 bordered system is singular");
    piv[c] = p;
    if (p != c)
      for (int q = 0; q < n; ++q) std::swap(K[(size_t)c * n + q], K[(size_t)p * n + q]);
    const double inv = 1.0 / K[(size_t)c * n + c];
    for (int i = c + 1; i < n; ++i) {
      const double f = K[(size_t)i * n + c] * inv;
      K[(size_t)i * n + c] = f;
      if (f != 0.0)
        for (int q = c + 1; q < n; ++q) K[(size_t)i * n + q] -= f * K[(size_t)c * n + q];
    }
  }
  std::vector<double> G((size_t)nr * nr, 0.0), x(n);
  for (int j = 0; j < nr; ++j) {
    if (dead[j]) continue;
    std::fill(x.begin(), x.end(), 0.0);
    x[j] = dr[j];  // scaled forcing of a unit g_j
    for (int c = 0; c < n; ++c) std::swap(x[c], x[piv[c]]);
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < i; ++c) x[i] -= K[(size_t)i * n + c] * x[c];
    for (int i = n - 1; i >= 0; --i) {
      for (int c = i + 1; c < n; ++c) x[i] -= K[(size_t)i * n + c] * x[c];
      x[i] /= K[(size_t)i * n + i];
    }
    for (int i = 0; i < nr; ++i) G[(size_t)i * nr + j] = dead[i] ? 0.0 : dc[i] * x[i];
  }
  return G;
}

// enable_toroidal (src/vilma_response.f90:1055-1118): per-degree W operators,
// the W drift arrays and zero toroidal memory
void toroidal_enable(vg_handle* h) {
  cudaStream_t s = h->stream;
  const int nr = h->nr, nk = h->nk, L = h->grid.lmax;
  std::vector<double> tw((size_t)(L + 1) * nr, 0.0), tib(tw.size(), 0.0), tc(tw.size(), 0.0);
  std::vector<double> diag, off;
  std::vector<char> dead;
  for (int l = 2; l <= L; ++l) {
    toroidal_tridiag(h->r, h->mu, l, diag, off, dead);
    double* w = &tw[(size_t)l * nr];
    double* ib = &tib[(size_t)l * nr];
    double* c = &tc[(size_t)l * nr];
    double bp = 1.0;
    for (int i = 0; i < nr; ++i) {
      const double d = dead[i] ? 1.0 : diag[i];
      const double a = i > 0 ? off[i - 1] : 0.0;  // sub-diagonal = super-diagonal of the row above
      w[i] = i > 0 ? a / bp : 0.0;
      bp = d - w[i] * a;
      if (!dead[i] && !(bp > 0.0)) throw Error("toroidal operator: non-positive pivot (degree " + std::to_string(l) + ")");
      ib[i] = dead[i] ? 0.0 : 1.0 / bp;
      c[i] = i + 1 < nr ? off[i] : 0.0;
    }
  }
  toroidal_tridiag(h->r, h->mu, 1, diag, off, dead);
  int ns = 0;
  std::vector<double> wrot = toroidal_rotation_weights(h->r, h->mu, ns);
  std::vector<double> G1 = degree1_solution_map(diag, off, dead, wrot, nr, ns);
  h->d_tw.upload(tw, s);
  h->d_tib.upload(tib, s);
  h->d_tc.upload(tc, s);
  h->d_tG1.upload(G1, s);
  const size_t nmem = (size_t)6 * h->ne * 2 * nk, nd2 = (size_t)2 * nr * nk;
  h->d_tmem[0].alloc(nmem);
  h->d_tmem[1].alloc(nmem);
  h->d_dWn.alloc(nd2);
  h->d_dWa.alloc((size_t)2 * nk);
  if (h->p.scheme == VG_SCHEME_TRAP) {
    h->d_edWn.alloc(nd2);
    h->d_dW_avg.alloc(nd2);
    h->d_dWa_prev.alloc((size_t)2 * nk);
    h->d_tmem_s.alloc(nmem);
    h->d_tmem_c.alloc(nmem);
  }
  VG_CUDA(cudaStreamSynchronize(s));
  h->tor_on = true;
}

// ------------------------------------------------------------------ drift

struct TorDriftArgs {
  const double* tmem;
  const double* mnorm;
  const unsigned long long* maxbits;
  double skip_tol;
  const double *r, *Jr;
  const int* kdeg;
  const double *tw, *tib, *tc, *G1;
  double *dWn, *dWa;
  int ne, nr, nk, k1, n1;  // degree-1 slots k1 .. k1 + n1 - 1
};

// dissipative_rhs_tor (src/vilma_viscoelastic.f90:403-439) of one element:
// its forcing on the test dofs dW_e (f0) and dW_{e+1} (f1)
__device__ __forceinline__ void element_floc_tor(const TorDriftArgs& A, int k, int ri, int e, double J, double& f0,
                                                 double& f1) {
  const double xg = 0.5773502691896257;
  const double nrm[2] = {0.5 * J, 0.5 * J * (J - 2.0)};
  double sa[2][2], sb[2][2], sc[2][2];
  strain_coeffs_tor(1.0, 0.0, J, sa[0], sb[0], sc[0]);
  strain_coeffs_tor(0.0, 1.0, J, sa[1], sb[1], sc[1]);
  const double rk = A.r[e], rk1 = A.r[e + 1], h = rk1 - rk;
  double Am[2], Bm[2], Cm[2];
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    Am[m] = A.tmem[tmem_idx(0, ri, e, m, k, A.ne, A.nk)];
    Bm[m] = A.tmem[tmem_idx(1, ri, e, m, k, A.ne, A.nk)];
    Cm[m] = A.tmem[tmem_idx(2, ri, e, m, k, A.ne, A.nk)];
  }
  double floc[2] = {0.0, 0.0};
#pragma unroll
  for (int ig = 0; ig < 2; ++ig) {
    const double ra = 0.5 * (h * (ig ? xg : -xg) + rk + rk1);
    const double psik = (rk1 - ra) / h, psik1 = (ra - rk) / h;
    double tauV[2];
#pragma unroll
    for (int m = 0; m < 2; ++m) tauV[m] = Am[m] / h + Bm[m] * psik / ra + Cm[m] * psik1 / ra;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      double D = 0.0;
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const double deps = sa[t][m] / h + sb[t][m] * psik / ra + sc[t][m] * psik1 / ra;
        D = D + nrm[m] * tauV[m] * deps;
      }
      floc[t] = floc[t] - D * ra * ra * h * 0.5;
    }
  }
  f0 = floc[0];
  f1 = floc[1];
}

__global__ void __launch_bounds__(128) k_drift_tor(TorDriftArgs A) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x, ri = blockIdx.y;
  if (k >= A.nk) return;
  double* W = A.dWn + (size_t)ri * A.nr * A.nk + k;  // node i at W[i * nk]
  const size_t nk = A.nk;
  const double thr = A.skip_tol * __longlong_as_double((long long)*A.maxbits);
  if (A.mnorm[k] <= thr) {  // negligible memory => negligible drift
    for (int i = 0; i < A.nr; ++i) W[i * nk] = 0.0;
    A.dWa[(size_t)ri * nk + k] = 0.0;
    return;
  }
  const int l = A.kdeg[k];
  const double J = A.Jr[l];
  const double* w = A.tw + (size_t)l * A.nr;
  double prev1 = 0.0, y = 0.0;
  for (int i = 0; i < A.nr; ++i) {
    double f0 = 0.0, f1 = 0.0;
    if (i < A.ne) element_floc_tor(A, k, ri, i, J, f0, f1);
    const double g = prev1 + f0;  // element i - 1's second test dof, then element i's first
    prev1 = f1;
    y = (l == 1) ? g : g - __ldg(&w[i]) * y;
    W[i * nk] = y;
  }
  if (l == 1) return;  // k_drift_tor1 applies the bordered solution map
  const double* ib = A.tib + (size_t)l * A.nr;
  const double* c = A.tc + (size_t)l * A.nr;
  double x = W[(size_t)(A.nr - 1) * nk] * __ldg(&ib[A.nr - 1]);
  W[(size_t)(A.nr - 1) * nk] = x;
  A.dWa[(size_t)ri * nk + k] = x;
  for (int i = A.nr - 2; i >= 0; --i) {
    x = (W[i * nk] - __ldg(&c[i]) * x) * __ldg(&ib[i]);
    W[i * nk] = x;
  }
}

// degree 1: W = G1W g for each (slot, re/im) that the gate let through
__global__ void __launch_bounds__(256) k_drift_tor1(TorDriftArgs A) {
  extern __shared__ double g[];  // nr
  const double thr = A.skip_tol * __longlong_as_double((long long)*A.maxbits);
  const size_t nk = A.nk;
  for (int q = 0; q < 2 * A.n1; ++q) {
    const int k = A.k1 + q / 2, ri = q % 2;
    if (A.mnorm[k] <= thr) continue;  // k_drift_tor zeroed it
    double* W = A.dWn + (size_t)ri * A.nr * nk + k;
    __syncthreads();
    for (int i = threadIdx.x; i < A.nr; i += blockDim.x) g[i] = W[i * nk];
    __syncthreads();
    for (int i = threadIdx.x; i < A.nr; i += blockDim.x) {
      const double* row = A.G1 + (size_t)i * A.nr;
      double acc = 0.0;
      for (int j = 0; j < A.nr; ++j) acc += __ldg(&row[j]) * g[j];
      W[i * nk] = acc;
      if (i == A.nr - 1) A.dWa[(size_t)ri * nk + k] = acc;
    }
  }
}

void launch_drift_tor(vg_handle* h, int buf, double* dWn) {
  TorDriftArgs A;
  A.tmem = h->d_tmem[buf].p;
  A.mnorm = h->d_mnorm.p + (size_t)buf * h->nk;
  A.maxbits = h->d_maxbits.p + buf;
  A.skip_tol = h->p.skip_tol;
  A.r = h->d_r.p;
  A.Jr = h->d_Jr.p;
  A.kdeg = h->d_kdeg.p;
  A.tw = h->d_tw.p;
  A.tib = h->d_tib.p;
  A.tc = h->d_tc.p;
  A.G1 = h->d_tG1.p;
  A.dWn = dWn ? dWn : h->d_dWn.p;
  A.dWa = h->d_dWa.p;
  A.ne = h->ne;
  A.nr = h->nr;
  A.nk = h->nk;
  A.k1 = h->kbeg_h[1];
  A.n1 = h->kbeg_h[2] - h->kbeg_h[1];
  k_drift_tor<<<dim3((h->nk + 127) / 128, 2), 128, 0, h->stream>>>(A);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  k_drift_tor1<<<1, 256, (size_t)h->nr * sizeof(double), h->stream>>>(A);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------ advance

// advance_memory_tor (src/vilma_viscoelastic.f90:591-629) with maxwell_fe
// (:640-654), or maxwell_trap (:683-700) with W the mean of the step's two
// ends; 3-D elements (already written by the pseudo-spectral pass) only enter
// the per-slot norm
__global__ void __launch_bounds__(256) k_advance_1d_tor(const double* __restrict__ tmem, double* __restrict__ tnxt,
                                                        int ne, int nr, int nk, double dt,
                                                        const int* __restrict__ kdeg, const double* __restrict__ Jrv,
                                                        const double* __restrict__ dWn, const double* __restrict__ mu,
                                                        const double* __restrict__ MkPerDt,
                                                        const char* __restrict__ active, double* __restrict__ mnorm,
                                                        int trap) {
  const int k = blockIdx.x * 32 + threadIdx.x, e = blockIdx.y * 8 + threadIdx.y, ri = blockIdx.z;
  double amax = 0.0;
  if (k < nk && e < ne) {
    if (active[e]) {
      const int l = kdeg[k];
      const double W0 = dWn[((size_t)ri * nr + e) * nk + k], W1 = dWn[((size_t)ri * nr + e + 1) * nk + k];
      double a[2], b[2], c[2];
      strain_coeffs_tor(W0, W1, Jrv[l], a, b, c);
      const double Me = MkPerDt[e] * dt;
      double om = 1.0 - Me, two_muM = 2.0 * mu[e] * Me;
      if (trap) {
        const double denom = 1.0 + 0.5 * Me;
        om = (1.0 - 0.5 * Me) / denom;
        two_muM = 2.0 * (mu[e] * Me / denom);
      }
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const size_t iA = tmem_idx(0, ri, e, m, k, ne, nk), iB = tmem_idx(1, ri, e, m, k, ne, nk),
                     iC = tmem_idx(2, ri, e, m, k, ne, nk);
        const double An = om * tmem[iA] - two_muM * a[m];
        const double Bn = om * tmem[iB] - two_muM * b[m];
        const double Cn = om * tmem[iC] - two_muM * c[m];
        tnxt[iA] = An;
        tnxt[iB] = Bn;
        tnxt[iC] = Cn;
        amax = nanmax(amax, nanmax(fabs(An), nanmax(fabs(Bn), fabs(Cn))));
      }
    } else {
#pragma unroll
      for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int s3 = 0; s3 < 3; ++s3) amax = nanmax(amax, fabs(tnxt[tmem_idx(s3, ri, e, m, k, ne, nk)]));
    }
  }
  __shared__ double red[8][33];
  red[threadIdx.y][threadIdx.x] = amax;
  __syncthreads();
  if (threadIdx.y == 0 && k < nk) {
    double v = red[0][threadIdx.x];
#pragma unroll
    for (int t = 1; t < 8; ++t) v = nanmax(v, red[t][threadIdx.x]);
    atomic_max_bits(reinterpret_cast<unsigned long long*>(mnorm) + k, v);
  }
}

void launch_advance_1d_tor(vg_handle* h, double dt, const double* dWn, bool trap, double* mn) {
  const int nxt = 1 - h->cur;
  dim3 grid((h->nk + 31) / 32, (h->ne + 7) / 8, 2);
  k_advance_1d_tor<<<grid, dim3(32, 8), 0, h->stream>>>(h->d_tmem[h->cur].p, h->d_tmem[nxt].p, h->ne, h->nr, h->nk,
                                                        dt, h->d_kdeg.p, h->d_Jr.p, dWn ? dWn : h->d_dWn.p,
                                                        h->d_mu.p, h->d_MkPerDt.p, h->d_active1d.p, mn,
                                                        trap ? 1 : 0);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// |toroidal memory| of one buffer folded into its per-slot norms
__global__ void k_mem_norm_tor(const double* __restrict__ tmem, int ne, int nk, double* __restrict__ mnorm) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  double amax = mnorm[k];
  for (int q = 0; q < 6 * ne * 2; ++q) amax = nanmax(amax, fabs(tmem[(size_t)q * nk + k]));
  mnorm[k] = amax;
}

void mem_norm_tor(vg_handle* h, int buf, double* mn) {
  k_mem_norm_tor<<<(h->nk + 255) / 256, 256, 0, h->stream>>>(h->d_tmem[buf].p, h->ne, h->nk, mn);
  VG_CUDA(cudaGetLastError());
}

}  // namespace vg
