// Field-driver kernels of the 1-D (spectral) path: the per-(l,m) drift solve
// with the reference's skip gate, the affine apply, and the forward-Euler
// memory advance fused with the per-slot memory norm that the next drift gate
// and the stepper's guard read (src/vilma_response.f90:679-864, 944-992;
// src/vilma_viscoelastic.f90:329-589).
#include <cstring>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

struct DriftArgs {
  const double* mem;            // current buffer
  const double* mnorm;          // per-slot norms of the current buffer
  const unsigned long long* maxbits;  // global max of the current buffer
  double skip_tol;
  const double* r;
  const double *sa, *sb, *sc, *nrmc;
  const double *ab, *dr, *dc;
  const int* ipiv;
  const int* kdeg;
  double* xs;                   // scratch (2, nd, nk)
  double *dUn, *dVn, *drift;
  int ne, nr, nd, nk, lmax;
  // degree 1
  const double *ab1, *dr1, *dc1, *null1;
  const int* ipiv1;
  int kl1, kv1, deg1_cm;
};

// Dissipative forcing -(tau^V : d eps) of one (slot, ri) into a strided column x
// (src/vilma_viscoelastic.f90:441-480). x must be zero on entry.
__device__ __forceinline__ void dissipative_rhs_col(const DriftArgs& A, int l, int k, int ri, double* x, size_t st) {
  const double xg = 0.5773502691896257;
  const double* sa = A.sa + l * 16;
  const double* sb = A.sb + l * 16;
  const double* sc = A.sc + l * 16;
  const double* nrm = A.nrmc + l * 4;
  for (int e = 0; e < A.ne; ++e) {
    double rk = A.r[e], rk1 = A.r[e + 1], h = rk1 - rk;
    double Am[4], Bm[4], Cm[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      Am[m] = A.mem[mem_idx(0, ri, e, m, k, A.ne, A.nk)];
      Bm[m] = A.mem[mem_idx(1, ri, e, m, k, A.ne, A.nk)];
      Cm[m] = A.mem[mem_idx(2, ri, e, m, k, A.ne, A.nk)];
    }
    double floc[4] = {0, 0, 0, 0};
#pragma unroll
    for (int ig = 0; ig < 2; ++ig) {
      double ra = 0.5 * (h * (ig ? xg : -xg) + rk + rk1);
      double psik = (rk1 - ra) / h, psik1 = (ra - rk) / h;
      double tauV[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) tauV[m] = Am[m] / h + Bm[m] * psik / ra + Cm[m] * psik1 / ra;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        double D = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          double deps = sa[t * 4 + m] / h + sb[t * 4 + m] * psik / ra + sc[t * 4 + m] * psik1 / ra;
          D = D + nrm[m] * tauV[m] * deps;
        }
        floc[t] = floc[t] - D * ra * ra * h * 0.5;
      }
    }
    x[(size_t)(4 * e) * st] += floc[0];
    x[(size_t)(4 * e + 4) * st] += floc[1];
    x[(size_t)(4 * e + 1) * st] += floc[2];
    x[(size_t)(4 * e + 5) * st] += floc[3];
  }
}

__device__ __forceinline__ void band_solve_col(const double* __restrict__ ab, int n, const int* __restrict__ ipiv,
                                               double* x, size_t st) {
  // dgbtrs order, kl = 6, kv = 12; ab[(row - 1) * n + (col - 1)] (band storage row kv + 1 + i - j)
  constexpr int kl = 6, kv = 12;
  for (int j = 1; j <= n - 1; ++j) {
    int lm = min(kl, n - j);
    int l = __ldg(&ipiv[j - 1]) + 1;
    if (l != j) {
      double t = x[(size_t)(l - 1) * st];
      x[(size_t)(l - 1) * st] = x[(size_t)(j - 1) * st];
      x[(size_t)(j - 1) * st] = t;
    }
    double t = x[(size_t)(j - 1) * st];
    for (int i = 1; i <= lm; ++i) x[(size_t)(j + i - 1) * st] -= __ldg(&ab[(size_t)(kv + i) * n + (j - 1)]) * t;
  }
  for (int j = n; j >= 1; --j) {
    double xj = x[(size_t)(j - 1) * st] / __ldg(&ab[(size_t)kv * n + (j - 1)]);
    x[(size_t)(j - 1) * st] = xj;
    int lm = min(kv, j - 1);
    for (int i = 1; i <= lm; ++i) x[(size_t)(j - i - 1) * st] -= __ldg(&ab[(size_t)(kv - i) * n + (j - 1)]) * xj;
  }
}

// Drift solve for degrees >= 2: one thread per slot k, real and imaginary
// histories one after the other (src/vilma_response.f90:744-802).
__global__ void __launch_bounds__(128) k_drift(DriftArgs A) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= A.nk) return;
  int l = A.kdeg[k];
  if (l < 2) return;
  const double thr = A.skip_tol * __longlong_as_double((long long)*A.maxbits);
  const int nr = A.nr, nd = A.nd, nk = A.nk;
  if (A.mnorm[k] <= thr) {
    for (int q = 0; q < 6; ++q) A.drift[(size_t)q * nk + k] = 0.0;
    for (int ri = 0; ri < 2; ++ri)
      for (int node = 0; node < nr; ++node) {
        A.dUn[((size_t)ri * nr + node) * nk + k] = 0.0;
        A.dVn[((size_t)ri * nr + node) * nk + k] = 0.0;
      }
    return;
  }
  const double* ab = A.ab + (size_t)(l - 2) * 19 * nd;
  const double* dr = A.dr + (size_t)(l - 2) * nd;
  const double* dc = A.dc + (size_t)(l - 2) * nd;
  const int* ipiv = A.ipiv + (size_t)(l - 2) * nd;
  for (int ri = 0; ri < 2; ++ri) {
    double* x = A.xs + (size_t)ri * nd * nk + k;
    for (int i = 0; i < nd; ++i) x[(size_t)i * nk] = 0.0;
    dissipative_rhs_col(A, l, k, ri, x, nk);
    for (int i = 0; i < nd; ++i) x[(size_t)i * nk] = __ldg(&dr[i]) * x[(size_t)i * nk];
    band_solve_col(ab, nd, ipiv, x, nk);
    for (int node = 0; node < nr; ++node) {
      A.dUn[((size_t)ri * nr + node) * nk + k] = __ldg(&dc[4 * node]) * x[(size_t)(4 * node) * nk];
      A.dVn[((size_t)ri * nr + node) * nk + k] = __ldg(&dc[4 * node + 1]) * x[(size_t)(4 * node + 1) * nk];
    }
    int us = 4 * (nr - 1);
    A.drift[(size_t)(0 + ri) * nk + k] = dc[us] * x[(size_t)us * nk];            // dUa
    A.drift[(size_t)(2 + ri) * nk + k] = dc[us + 2] * x[(size_t)(us + 2) * nk];  // dFa
    A.drift[(size_t)(4 + ri) * nk + k] = dc[us + 1] * x[(size_t)(us + 1) * nk];  // dVa
  }
}

// Degree-1 drift (slots k = 0, 1): bordered dense system, CTA-parallel sweeps,
// CM-frame projection with the stored null mode (src/vilma_response.f90:770-779).
__global__ void __launch_bounds__(256) k_drift_deg1(DriftArgs A) {
  extern __shared__ double xsh[];  // [4][ns]
  const int nd = A.nd, ns = nd + 1, nr = A.nr, nk = A.nk;
  const double thr = A.skip_tol * __longlong_as_double((long long)*A.maxbits);
  __shared__ int s_active[2];
  if (threadIdx.x < 2) s_active[threadIdx.x] = !(A.mnorm[threadIdx.x] <= thr);
  for (int i = threadIdx.x; i < 4 * ns; i += blockDim.x) xsh[i] = 0.0;
  __syncthreads();
  if (!s_active[0] && !s_active[1]) {
    for (int t = threadIdx.x; t < 2; t += blockDim.x) {
      int k = t;
      for (int q = 0; q < 6; ++q) A.drift[(size_t)q * nk + k] = 0.0;
    }
    for (int t = threadIdx.x; t < 2 * 2 * nr; t += blockDim.x) {
      int k = t % 2, rest = t / 2, ri = rest % 2, node = rest / 2;
      A.dUn[((size_t)ri * nr + node) * nk + k] = 0.0;
      A.dVn[((size_t)ri * nr + node) * nk + k] = 0.0;
    }
    return;
  }
  if (threadIdx.x < 4) {  // rhs index q = k*2 + ri
    int k = threadIdx.x / 2, ri = threadIdx.x % 2;
    if (s_active[k]) {
      dissipative_rhs_col(A, 1, k, ri, xsh + threadIdx.x * ns, 1);
      for (int i = 0; i < nd; ++i) xsh[threadIdx.x * ns + i] = A.dr1[i] * xsh[threadIdx.x * ns + i];
    }
  }
  __syncthreads();
  deg1_solve_cta(A.ab1, ns, A.kl1, A.kv1, A.ipiv1, xsh, 4);
  for (int t = threadIdx.x; t < 4 * nd; t += blockDim.x) {
    int q = t / nd, i = t % nd;
    xsh[q * ns + i] = A.dc1[i] * xsh[q * ns + i];
  }
  __syncthreads();
  if (A.deg1_cm) {
    int fs = 4 * (nr - 1) + 2;
    double fa_n = A.null1[fs];
    if (fa_n != 0.0) {
      __shared__ double s_c[4];
      if (threadIdx.x < 4) s_c[threadIdx.x] = -xsh[threadIdx.x * ns + fs] / fa_n;
      __syncthreads();
      for (int t = threadIdx.x; t < 4 * nd; t += blockDim.x) {
        int q = t / nd, i = t % nd;
        xsh[q * ns + i] = xsh[q * ns + i] + s_c[q] * A.null1[i];
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < 4 * nr; t += blockDim.x) {
    int q = t / nr, node = t % nr, k = q / 2, ri = q % 2;
    double u = s_active[k] ? xsh[q * ns + 4 * node] : 0.0;
    double v = s_active[k] ? xsh[q * ns + 4 * node + 1] : 0.0;
    A.dUn[((size_t)ri * nr + node) * nk + k] = u;
    A.dVn[((size_t)ri * nr + node) * nk + k] = v;
  }
  if (threadIdx.x < 4) {
    int q = threadIdx.x, k = q / 2, ri = q % 2, us = 4 * (nr - 1);
    bool act = s_active[k];
    A.drift[(size_t)(0 + ri) * nk + k] = act ? xsh[q * ns + us] : 0.0;
    // N_1 == 0 in the "cf" frame (src/vilma_response.f90:779)
    A.drift[(size_t)(2 + ri) * nk + k] = (act && A.deg1_cm) ? xsh[q * ns + us + 2] : 0.0;
    A.drift[(size_t)(4 + ri) * nk + k] = act ? xsh[q * ns + us + 1] : 0.0;
  }
}

void launch_drift(vg_handle* h) {
  PhaseScope ps(h, VG_PH_DRIFT);
  DriftArgs A;
  A.mem = h->d_mem[h->cur].p;
  A.mnorm = h->d_mnorm.p + (size_t)h->cur * h->nk;
  A.maxbits = h->d_maxbits.p + h->cur;
  A.skip_tol = h->p.skip_tol;
  A.r = h->d_r.p;
  A.sa = h->d_sa.p;
  A.sb = h->d_sb.p;
  A.sc = h->d_sc.p;
  A.nrmc = h->d_nrmc.p;
  A.ab = h->d_ab.p;
  A.dr = h->d_dr.p;
  A.dc = h->d_dc.p;
  A.ipiv = h->d_ipiv.p;
  A.kdeg = h->d_kdeg.p;
  A.xs = h->d_xs.p;
  A.dUn = h->d_dUn.p;
  A.dVn = h->d_dVn.p;
  A.drift = h->d_drift.p;
  A.ne = h->ne;
  A.nr = h->nr;
  A.nd = h->ndof;
  A.nk = h->nk;
  A.lmax = h->p.lmax;
  A.ab1 = h->d_ab1.p;
  A.dr1 = h->d_dr1.p;
  A.dc1 = h->d_dc1.p;
  A.null1 = h->d_null1.p;
  A.ipiv1 = h->d_ipiv1.p;
  A.kl1 = h->kl1;
  A.kv1 = h->kv1;
  A.deg1_cm = h->p.deg1_cm;
  k_drift<<<(h->nk + 127) / 128, 128, 0, h->stream>>>(A); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  size_t shm = 4 * (size_t)(h->ndof + 1) * sizeof(double);
  static bool attr_set = false;
  if (!attr_set && shm > 48 * 1024) {
    VG_CUDA(cudaFuncSetAttribute(k_drift_deg1, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr_set = true;
  }
  k_drift_deg1<<<1, 256, shm, h->stream>>>(A); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// src/vilma_response.f90:842-864 ve_response_apply: u = gu(l) sigma + dUa, N = gn(l) sigma - dFa/g
__global__ void k_apply(int nlm, int nk, double g, const int* __restrict__ lm_l, const int* __restrict__ lm2k,
                        const double* __restrict__ gu, const double* __restrict__ gn,
                        const double* __restrict__ drift, const double* __restrict__ sigma, double* __restrict__ u,
                        double* __restrict__ n) {
  int lm = blockIdx.x * blockDim.x + threadIdx.x;
  if (lm >= nlm) return;
  int l = lm_l[lm];
  double sr = sigma[2 * lm], si = sigma[2 * lm + 1];
  if (l == 0) {
    u[2 * lm] = gu[0] * sr;
    u[2 * lm + 1] = gu[0] * si;
    n[2 * lm] = gn[0] * sr;
    n[2 * lm + 1] = gn[0] * si;
    return;
  }
  int k = lm2k[lm];
  u[2 * lm] = gu[l] * sr + drift[(size_t)0 * nk + k];
  u[2 * lm + 1] = gu[l] * si + drift[(size_t)1 * nk + k];
  n[2 * lm] = gn[l] * sr - drift[(size_t)2 * nk + k] / g;
  n[2 * lm + 1] = gn[l] * si - drift[(size_t)3 * nk + k] / g;
}

void launch_apply(vg_handle* h, const double* d_sigma, double* d_u, double* d_n) {
  int nlm = h->grid.nlm;
  k_apply<<<(nlm + 255) / 256, 256, 0, h->stream>>>(nlm, h->nk, h->g, h->grid.d_lm_l.p, h->d_lm2k.p, h->d_gu.p,
                                                    h->d_gn.p, h->d_drift.p, d_sigma, d_u, d_n); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// Forward-Euler memory advance of the spectrally advanced elements, one thread
// per slot, out of place (cur -> nxt), with the per-slot norm of the new
// state over ALL elements (the 3-D elements were written to nxt before).
__global__ void __launch_bounds__(256) k_advance_1d(const double* __restrict__ mem, double* __restrict__ nxt, int ne, int nr, int nk,
                             double dt, const double* __restrict__ sigma, const int* __restrict__ kdeg,
                             const int* __restrict__ k2lm, const double* __restrict__ Jrv,
                             const double* __restrict__ xUn, const double* __restrict__ xVn,
                             const double* __restrict__ dUn, const double* __restrict__ dVn,
                             const double* __restrict__ mu, const double* __restrict__ MkPerDt,
                             const char* __restrict__ active, double* __restrict__ mnorm,
                             unsigned long long* __restrict__ maxbits) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  double amax = 0.0;
  if (k < nk) {
    int l = kdeg[k], lm = k2lm[k];
    double Jr = Jrv[l];
    const double* xu = xUn + (size_t)l * nr;
    const double* xv = xVn + (size_t)l * nr;
    for (int ri = 0; ri < 2; ++ri) {
      double s = sigma[2 * lm + ri];
      double U0 = s * xu[0] + dUn[((size_t)ri * nr + 0) * nk + k];
      double V0 = s * xv[0] + dVn[((size_t)ri * nr + 0) * nk + k];
      for (int e = 0; e < ne; ++e) {
        double U1 = s * xu[e + 1] + dUn[((size_t)ri * nr + e + 1) * nk + k];
        double V1 = s * xv[e + 1] + dVn[((size_t)ri * nr + e + 1) * nk + k];
        if (active[e]) {
          double a[4], b[4], c[4];
          strain_coeffs(U0, U1, V0, V1, Jr, a, b, c);
          double Me = MkPerDt[e] * dt;
          double om = 1.0 - Me, two_muM = 2.0 * mu[e] * Me;
#pragma unroll
          for (int m = 0; m < 4; ++m) {
            size_t iA = mem_idx(0, ri, e, m, k, ne, nk), iB = mem_idx(1, ri, e, m, k, ne, nk),
                   iC = mem_idx(2, ri, e, m, k, ne, nk);
            double An = om * mem[iA] - two_muM * a[m];
            double Bn = om * mem[iB] - two_muM * b[m];
            double Cn = om * mem[iC] - two_muM * c[m];
            nxt[iA] = An;
            nxt[iB] = Bn;
            nxt[iC] = Cn;
            amax = nanmax(amax, nanmax(fabs(An), nanmax(fabs(Bn), fabs(Cn))));
          }
        } else {
#pragma unroll
          for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int s3 = 0; s3 < 3; ++s3) amax = nanmax(amax, fabs(nxt[mem_idx(s3, ri, e, m, k, ne, nk)]));
        }
        U0 = U1;
        V0 = V1;
      }
    }
    mnorm[k] = amax;
  }
  // block max, then one atomic per block
  __shared__ double red[256];
  red[threadIdx.x] = amax;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = nanmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomic_max_bits(maxbits, red[0]);
}

void launch_advance_1d(vg_handle* h, const double* d_sigma, double dt) {
  PhaseScope ps(h, VG_PH_ADVANCE_1D);
  int nxt = 1 - h->cur;
  VG_CUDA(cudaMemsetAsync(h->d_maxbits.p + nxt, 0, sizeof(unsigned long long), h->stream));
  k_advance_1d<<<(h->nk + 255) / 256, 256, 0, h->stream>>>(
      h->d_mem[h->cur].p, h->d_mem[nxt].p, h->ne, h->nr, h->nk, dt, d_sigma, h->d_kdeg.p, h->d_k2lm.p, h->d_Jr.p,
      h->d_xUn.p, h->d_xVn.p, h->d_dUn.p, h->d_dVn.p, h->d_mu.p, h->d_MkPerDt.p, h->d_active1d.p,
      h->d_mnorm.p + (size_t)nxt * h->nk, h->d_maxbits.p + nxt); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// per-slot norm and global max of one buffer (after vg_set_state / reset)
__global__ void k_mem_norm(const double* __restrict__ mem, int ne, int nk, double* __restrict__ mnorm,
                           unsigned long long* __restrict__ maxbits) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  double amax = 0.0;
  if (k < nk) {
    for (int q = 0; q < 6 * ne * 4; ++q) amax = nanmax(amax, fabs(mem[(size_t)q * nk + k]));
    mnorm[k] = amax;
  }
  __shared__ double red[256];
  red[threadIdx.x] = amax;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = nanmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomic_max_bits(maxbits, red[0]);
}

void compute_mem_norm(vg_handle* h, int buf) {
  VG_CUDA(cudaMemsetAsync(h->d_maxbits.p + buf, 0, sizeof(unsigned long long), h->stream));
  k_mem_norm<<<(h->nk + 255) / 256, 256, 0, h->stream>>>(h->d_mem[buf].p, h->ne, h->nk,
                                                         h->d_mnorm.p + (size_t)buf * h->nk, h->d_maxbits.p + buf); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

double read_mem_norm(vg_handle* h, int buf) {
  unsigned long long bits = 0;
  VG_CUDA(cudaMemcpyAsync(&bits, h->d_maxbits.p + buf, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
  VG_CUDA(cudaStreamSynchronize(h->stream));
  double v;
  std::memcpy(&v, &bits, sizeof(v));
  return v;
}

}  // namespace vg
