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
// The W operators are small (nr x nr) and never change, so enable time inverts
// them on the host: l >= 2 by Thomas solves of the unit forcings (the system is
// symmetric positive definite on the live nodes, so no pivoting is needed),
// l = 1 through the bordered system, equilibrated and solved by
// partial-pivoting elimination; pinned rows and columns are zero. The drift is
// then two bandwidth-friendly kernels instead of a serial sweep per slot:
//   k_drift_tor_rhs  one thread per (slot, node, re/im): the forcing g at the
//                    node from its two elements through per-(degree, element)
//                    maps of the memory (the memory read along the slot)
//   k_drift_tor_mm   per degree, W = G_l g for all 2 (l + 1) columns (slot,
//                    re/im) of the degree: the forcing tile staged in shared
//                    memory, the inverse streamed from L2
//   k_advance_1d_tor one thread per (slot, element, re/im), like k_advance_1d
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
  const size_t nr2 = (size_t)nr * nr;
  std::vector<double> Ginv((size_t)L * nr2, 0.0);  // degree l at (l - 1) nr^2, row-major [i][j]
  std::vector<double> diag, off, w(nr), ib(nr), y(nr);
  std::vector<char> dead;
  for (int l = 2; l <= L; ++l) {
    toroidal_tridiag(h->r, h->mu, l, diag, off, dead);
    double bp = 1.0;
    for (int i = 0; i < nr; ++i) {  // Thomas factorisation
      const double d = dead[i] ? 1.0 : diag[i];
      const double a = i > 0 ? off[i - 1] : 0.0;
      w[i] = i > 0 ? a / bp : 0.0;
      bp = d - w[i] * a;
      if (!dead[i] && !(bp > 0.0)) throw Error("toroidal operator: non-positive pivot (degree " + std::to_string(l) + ")");
      ib[i] = dead[i] ? 0.0 : 1.0 / bp;
    }
    double* G = &Ginv[(size_t)(l - 1) * nr2];
    for (int j = 0; j < nr; ++j) {  // column j: the response to a unit forcing of node j
      if (dead[j]) continue;
      for (int i = 0; i < nr; ++i) y[i] = (i == j ? 1.0 : 0.0) - (i > 0 ? w[i] * y[i - 1] : 0.0);
      double x = y[nr - 1] * ib[nr - 1];
      G[(size_t)(nr - 1) * nr + j] = x;
      for (int i = nr - 2; i >= 0; --i) {
        x = (y[i] - (i + 1 < nr ? off[i] : 0.0) * x) * ib[i];
        G[(size_t)i * nr + j] = x;
      }
    }
  }
  toroidal_tridiag(h->r, h->mu, 1, diag, off, dead);
  int ns = 0;
  std::vector<double> wrot = toroidal_rotation_weights(h->r, h->mu, ns);
  std::vector<double> G1 = degree1_solution_map(diag, off, dead, wrot, nr, ns);
  std::copy(G1.begin(), G1.end(), Ginv.begin());
  h->d_tGinv.upload(Ginv, s);
  // forcing map per (degree, element): floc_t = sum_{s, m} K[t][s][m] tau_s^m, the
  // 2-point Gauss quadrature of dissipative_rhs_tor (src/vilma_viscoelastic.f90:403-439)
  // with the memory factored out
  const int ne = h->ne;
  std::vector<double> Kt((size_t)(L + 1) * ne * 12, 0.0);
  const double xg = 0.5773502691896257;
  for (int l = 1; l <= L; ++l) {
    const double J = (double)l * (double)(l + 1);
    const double nrm[2] = {0.5 * J, 0.5 * J * (J - 2.0)};
    // unit-dof strain coefficients (strain_coeffs_tor of dW_e = 1, dW_{e+1} = 1)
    const double sa[2][2] = {{-1.0, 0.0}, {1.0, 0.0}};
    const double sb[2][2] = {{-1.0, J <= 2.0 ? 0.0 : 1.0}, {0.0, 0.0}};
    const double sc[2][2] = {{0.0, 0.0}, {-1.0, J <= 2.0 ? 0.0 : 1.0}};
    for (int e = 0; e < ne; ++e) {
      const double rk = h->r[e], rk1 = h->r[e + 1], hh = rk1 - rk;
      double* K = &Kt[((size_t)l * ne + e) * 12];
      for (int ig = 0; ig < 2; ++ig) {
        const double ra = 0.5 * (hh * (ig ? xg : -xg) + rk + rk1);
        const double psik = (rk1 - ra) / hh, psik1 = (ra - rk) / hh;
        const double phi[3] = {1.0 / hh, psik / ra, psik1 / ra};
        for (int t = 0; t < 2; ++t)
          for (int m = 0; m < 2; ++m) {
            const double deps = sa[t][m] / hh + sb[t][m] * psik / ra + sc[t][m] * psik1 / ra;
            for (int s3 = 0; s3 < 3; ++s3) K[(t * 3 + s3) * 2 + m] -= nrm[m] * phi[s3] * deps * ra * ra * hh * 0.5;
          }
      }
    }
  }
  h->d_tK.upload(Kt, s);
  const size_t nmem = (size_t)6 * h->ne * 2 * nk, nd2 = (size_t)2 * nr * nk;
  h->d_tmem[0].alloc(nmem);
  h->d_tmem[1].alloc(nmem);
  h->d_dWn.alloc(nd2);
  h->d_tg.alloc(nd2);
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
  const double* K;  // forcing maps (lmax + 1, ne, 12)
  const int *kdeg, *kbeg;
  const double* Ginv;
  double *g, *dWn, *dWa;
  int ne, nr, nk, lmax;
};

// g(node) = element node-1's second test dof + element node's first (the
// reference's accumulation order) through the precomputed forcing maps; zero
// for slots the gate skips, whose W (and W(a)) then come out zero
__global__ void __launch_bounds__(128) k_drift_tor_rhs(TorDriftArgs A) {
  const int k = blockIdx.x * 32 + threadIdx.x, node = blockIdx.y * 4 + threadIdx.y, ri = blockIdx.z;
  if (k >= A.nk || node >= A.nr) return;
  double g = 0.0;
  if (!(A.mnorm[k] <= A.skip_tol * __longlong_as_double((long long)*A.maxbits))) {
    const int l = A.kdeg[k];
#pragma unroll
    for (int side = 0; side < 2; ++side) {  // element node - 1 (test dof 1), then element node (test dof 0)
      const int e = node - 1 + side, t = 1 - side;
      if (e < 0 || e >= A.ne) continue;
      const double* K = A.K + ((size_t)l * A.ne + e) * 12 + t * 6;
      double f = 0.0;
#pragma unroll
      for (int s3 = 0; s3 < 3; ++s3)
#pragma unroll
        for (int m = 0; m < 2; ++m) f = fma(__ldg(&K[s3 * 2 + m]), A.tmem[tmem_idx(s3, ri, e, m, k, A.ne, A.nk)], f);
      g = g + f;
    }
  }
  A.g[((size_t)ri * A.nr + node) * A.nk + k] = g;
}

// W = G_l g over the 2 (l + 1) columns (slot, re/im) of degree l = blockIdx.y + 1,
// TOR_MC columns per CTA; the forcing tile [node][column] in shared memory, each
// thread TOR_RB rows of one column
constexpr int TOR_MC = 16, TOR_MR = 16, TOR_RB = 4;
__global__ void __launch_bounds__(TOR_MC * TOR_MR) k_drift_tor_mm(TorDriftArgs A) {
  extern __shared__ double gs[];  // [nr][TOR_MC]
  const int l = blockIdx.y + 1, n0 = blockIdx.x * TOR_MC;
  const int k0 = A.kbeg[l], ncol = 2 * (A.kbeg[l + 1] - k0);
  if (n0 >= ncol) return;
  const int c = threadIdx.x % TOR_MC, rg = threadIdx.x / TOR_MC;
  const int n = n0 + c, k = k0 + n / 2, ri = n % 2;
  const bool live = n < ncol;
  for (int j = rg; j < A.nr; j += TOR_MR)
    gs[j * TOR_MC + c] = live ? A.g[((size_t)ri * A.nr + j) * A.nk + k] : 0.0;
  __syncthreads();
  if (!live) return;
  const double* G = A.Ginv + (size_t)(l - 1) * A.nr * A.nr;
  for (int i0 = rg * TOR_RB; i0 < A.nr; i0 += TOR_MR * TOR_RB) {
    const double* row[TOR_RB];
    double acc[TOR_RB];
#pragma unroll
    for (int b = 0; b < TOR_RB; ++b) {
      row[b] = G + (size_t)min(i0 + b, A.nr - 1) * A.nr;
      acc[b] = 0.0;
    }
    for (int j = 0; j < A.nr; ++j) {
      const double gj = gs[j * TOR_MC + c];
#pragma unroll
      for (int b = 0; b < TOR_RB; ++b) acc[b] = fma(__ldg(&row[b][j]), gj, acc[b]);
    }
#pragma unroll
    for (int b = 0; b < TOR_RB; ++b) {
      const int i = i0 + b;
      if (i >= A.nr) break;
      A.dWn[((size_t)ri * A.nr + i) * A.nk + k] = acc[b];
      if (i == A.nr - 1) A.dWa[(size_t)ri * A.nk + k] = acc[b];
    }
  }
}

void launch_drift_tor(vg_handle* h, int buf, double* dWn) {
  TorDriftArgs A;
  A.tmem = h->d_tmem[buf].p;
  A.mnorm = h->d_mnorm.p + (size_t)buf * h->nk;
  A.maxbits = h->d_maxbits.p + buf;
  A.skip_tol = h->p.skip_tol;
  A.K = h->d_tK.p;
  A.kdeg = h->d_kdeg.p;
  A.kbeg = h->d_kbeg.p;
  A.Ginv = h->d_tGinv.p;
  A.g = h->d_tg.p;
  A.dWn = dWn ? dWn : h->d_dWn.p;
  A.dWa = h->d_dWa.p;
  A.ne = h->ne;
  A.nr = h->nr;
  A.nk = h->nk;
  A.lmax = h->grid.lmax;
  k_drift_tor_rhs<<<dim3((h->nk + 31) / 32, (h->nr + 3) / 4, 2), dim3(32, 4), 0, h->stream>>>(A);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  const size_t smem = (size_t)h->nr * TOR_MC * sizeof(double);
  static std::atomic<bool> attr{false};  // set once; concurrent handles may race to it
  if (!attr) {
    VG_CUDA(cudaFuncSetAttribute(k_drift_tor_mm, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    attr = true;
  }
  if (smem > 96 * 1024) throw Error("toroidal drift: too many radial nodes for the shared forcing tile");
  const int nchunk = (2 * (h->grid.lmax + 1) + TOR_MC - 1) / TOR_MC;
  k_drift_tor_mm<<<dim3(nchunk, h->grid.lmax), TOR_MC * TOR_MR, smem, h->stream>>>(A);
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

// ------------------------------------------------------------------ adjoint

namespace vg {

// advance_memory_tor transposed for the spectrally advanced (1-D) elements, a
// thread per (slot, element, re/im): lam_t_new = (1 - M) lam_t; the strain
// adjoint -2 mu M lam_t through strain_coeffs_tor transposed into the W
// adjoints of the element's two nodes (Et planes W0, W1; zero for elements
// that are not spectrally advanced: the 3-D pass writes its own)
__global__ void __launch_bounds__(256) k_adv1d_tor_T(int ne, int nk, double dt, const int* __restrict__ kdeg,
                                                     const double* __restrict__ Jrv, const double* __restrict__ mu,
                                                     const double* __restrict__ MkPerDt,
                                                     const char* __restrict__ active, const double* __restrict__ lam_t,
                                                     double* __restrict__ lam_t_new, double* __restrict__ Et) {
  const int k = blockIdx.x * 32 + threadIdx.x, e = blockIdx.y * 8 + threadIdx.y, ri = blockIdx.z;
  if (k >= nk || e >= ne) return;
  const size_t plane = (size_t)2 * ne * nk, at = ((size_t)ri * ne + e) * nk + k;
  if (!active[e]) {  // (3-D elements: the 3-D pass's adjoint overwrites both)
    Et[0 * plane + at] = 0.0;
    Et[1 * plane + at] = 0.0;
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int s3 = 0; s3 < 3; ++s3) lam_t_new[tmem_idx(s3, ri, e, m, k, ne, nk)] = 0.0;
    return;
  }
  const double J = Jrv[kdeg[k]];
  const double Me = MkPerDt[e] * dt, om = 1.0 - Me, two_muM = 2.0 * mu[e] * Me;
  double w1 = 0.0, w2 = 0.0;
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const size_t iA = tmem_idx(0, ri, e, m, k, ne, nk), iB = tmem_idx(1, ri, e, m, k, ne, nk),
                 iC = tmem_idx(2, ri, e, m, k, ne, nk);
    const double la = lam_t[iA], lb = lam_t[iB], lc = lam_t[iC];
    lam_t_new[iA] = om * la;
    lam_t_new[iB] = om * lb;
    lam_t_new[iC] = om * lc;
    const double ga = -two_muM * la, gb = -two_muM * lb, gc = -two_muM * lc;
    if (m == 0) {  // a = -w1 + w2, b = -w1, c = -w2
      w1 += -ga - gb;
      w2 += ga - gc;
    } else if (J > 2.0) {  // b = w1, c = w2 (a[1] = 0)
      w1 += gb;
      w2 += gc;
    }
  }
  Et[0 * plane + at] = w1;
  Et[1 * plane + at] = w2;
}

// the nodal W adjoints from the two elements that share each node
__global__ void __launch_bounds__(256) k_tor_node_T(int ne, int nr, int nk, const double* __restrict__ Et,
                                                    double* __restrict__ Wb) {
  const int k = blockIdx.x * 32 + threadIdx.x, node = blockIdx.y * 8 + threadIdx.y, ri = blockIdx.z;
  if (k >= nk || node >= nr) return;
  const size_t plane = (size_t)2 * ne * nk;
  const double* Er = Et + (size_t)ri * ne * nk + k;
  double w = 0.0;
  if (node < ne) w += Er[0 * plane + (size_t)node * nk];
  if (node >= 1) w += Er[1 * plane + (size_t)(node - 1) * nk];
  Wb[((size_t)ri * nr + node) * nk + k] = w;
}

// the forcing maps transposed: lam_t_new += K^T g_bar (element e's test dof 1
// at node e + 1, test dof 0 at node e)
__global__ void __launch_bounds__(256) k_drift_tor_rhs_T(int ne, int nr, int nk, const int* __restrict__ kdeg,
                                                         const double* __restrict__ K, const double* __restrict__ gb,
                                                         double* __restrict__ lam_t_new) {
  const int k = blockIdx.x * 32 + threadIdx.x, e = blockIdx.y * 8 + threadIdx.y, ri = blockIdx.z;
  if (k >= nk || e >= ne) return;
  const int l = kdeg[k];
  const double g0 = gb[((size_t)ri * nr + e) * nk + k], g1 = gb[((size_t)ri * nr + e + 1) * nk + k];
  const double* K0 = K + ((size_t)l * ne + e) * 12;  // test dof 0 (node e), then test dof 1 (node e + 1)
#pragma unroll
  for (int s3 = 0; s3 < 3; ++s3)
#pragma unroll
    for (int m = 0; m < 2; ++m)
      lam_t_new[tmem_idx(s3, ri, e, m, k, ne, nk)] += K0[s3 * 2 + m] * g0 + K0[6 + s3 * 2 + m] * g1;
}

void advance_1d_tor_T(vg_handle* h, double dt, const double* lam_t, double* lam_t_new, double* Et) {
  dim3 grid((h->nk + 31) / 32, (h->ne + 7) / 8, 2);
  k_adv1d_tor_T<<<grid, dim3(32, 8), 0, h->stream>>>(h->ne, h->nk, dt, h->d_kdeg.p, h->d_Jr.p, h->d_mu.p,
                                                     h->d_MkPerDt.p, h->d_active1d.p, lam_t, lam_t_new, Et);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// W drift transposed: the nodal W adjoints (from the element strain adjoints
// Et) through the transposed inverse W operators, then the forcing maps
// transposed into lam_t_new (adds); Wb and gb are (2, nr, nk) work arrays
void drift_tor_T(vg_handle* h, const double* Et, double* Wb, double* gb, double* lam_t_new) {
  const int nr = h->nr, nk = h->nk, ne = h->ne, L = h->grid.lmax;
  cudaStream_t s = h->stream;
  k_tor_node_T<<<dim3((nk + 31) / 32, (nr + 7) / 8, 2), dim3(32, 8), 0, s>>>(ne, nr, nk, Et, Wb);
  if (h->d_tGinvT.n != h->d_tGinv.n) {  // the transposed inverses, once
    std::vector<double> G(h->d_tGinv.n), GT(h->d_tGinv.n);
    h->d_tGinv.download(G.data(), G.size(), s);
    VG_CUDA(cudaStreamSynchronize(s));
    const size_t nr2 = (size_t)nr * nr;
    for (int l = 1; l <= L; ++l)
      for (int i = 0; i < nr; ++i)
        for (int j = 0; j < nr; ++j) GT[(l - 1) * nr2 + (size_t)j * nr + i] = G[(l - 1) * nr2 + (size_t)i * nr + j];
    h->d_tGinvT.upload(GT, s);
    if (h->d_tWa_scratch.n < (size_t)2 * nk) h->d_tWa_scratch.alloc((size_t)2 * nk);
  }
  TorDriftArgs A;
  A.tmem = nullptr;
  A.mnorm = nullptr;
  A.maxbits = nullptr;
  A.skip_tol = 0.0;
  A.K = h->d_tK.p;
  A.kdeg = h->d_kdeg.p;
  A.kbeg = h->d_kbeg.p;
  A.Ginv = h->d_tGinvT.p;
  A.g = Wb;
  A.dWn = gb;
  A.dWa = h->d_tWa_scratch.p;
  A.ne = ne;
  A.nr = nr;
  A.nk = nk;
  A.lmax = L;
  const size_t smem = (size_t)nr * TOR_MC * sizeof(double);
  if (smem > 96 * 1024) throw Error("toroidal drift: too many radial nodes for the shared forcing tile");
  VG_CUDA(cudaFuncSetAttribute(k_drift_tor_mm, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  const int nchunk = (2 * (L + 1) + TOR_MC - 1) / TOR_MC;
  k_drift_tor_mm<<<dim3(nchunk, L), TOR_MC * TOR_MR, smem, s>>>(A);
  k_drift_tor_rhs_T<<<dim3((nk + 31) / 32, (ne + 7) / 8, 2), dim3(32, 8), 0, s>>>(ne, nr, nk, h->d_kdeg.p, h->d_tK.p,
                                                                                   gb, lam_t_new);
  h->n_launch += 3;
  VG_CUDA(cudaGetLastError());
}

}  // namespace vg
