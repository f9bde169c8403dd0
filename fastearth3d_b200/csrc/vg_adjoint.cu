// Hand-written discrete adjoint of the response-level time step, for the
// gradient of a relative-sea-level misfit at land sites.
//
// Forward model (the response stepping of tests/bench_visc3d.f90 and
// src/vilma_response.f90:228-319: begin_step, apply, advance), from the
// handle's current memory tau_0, with a prescribed surface load sigma_n held
// over each step of length dt and no sea-level equation (land sites, no ocean):
//   drift_n = D(tau_n)                      (dissipative RHS + band solves)
//   u_n = gu sigma_n + dUa_n, N_n = gn sigma_n - dFa_n / g     (apply)
//   rsl_n(s) = synthesis of (N_n - u_n) at site s               (no ocean: rsl = N - u)
//   tau_{n+1} = advance(tau_n, sigma_n, drift_n)                (forward Euler)
//   J = sum_n sum_s (rsl_n(s) - obs_n(s))^2
// The map (tau_0, sigma) -> rsl is linear, so the reverse sweep needs only the
// stored residuals; it runs the transposes backwards in time:
//   site synthesis^T, apply^T, advance^T (1-D elements: (1 - M) and the
//   strain of -2 mu M), drift^T (the dissipative map's transpose after an
//   equilibrated transposed band solve, U^T then L^T with the pivots undone;
//   degree 1 through the transposed Green's block and CM projection).
// All in FP64. The drift skip gate is off inside these entry points: with a
// zero threshold it only skips slots whose memory is exactly zero, whose drift
// is zero anyway, so the forward stays exactly linear.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

// rsl at the sites from the spectrum q = N - u: one block per site
__global__ void k_site_synth(int nsite, const int* __restrict__ site, int nlm, int nlat, int nphi,
                             const int* __restrict__ lm_m, const double* __restrict__ plm,
                             const double* __restrict__ cs, const double* __restrict__ sn,
                             const double* __restrict__ u, const double* __restrict__ nn,
                             const double* __restrict__ obs, double* __restrict__ resid) {
  __shared__ double red[256];
  const int s = blockIdx.x;
  if (s >= nsite) return;
  const int g = site[s], j = g / nphi, i = g % nphi;
  double acc = 0.0;
  for (int lm = threadIdx.x; lm < nlm; lm += blockDim.x) {
    const int m = lm_m[lm];
    const int t = (int)(((long long)m * i) % nphi);
    const double c = (m == 0 ? 1.0 : 2.0) * plm[(size_t)lm * nlat + j];
    const double qr = nn[2 * lm] - u[2 * lm], qi = nn[2 * lm + 1] - u[2 * lm + 1];
    acc += c * (qr * cs[t] - qi * sn[t]);
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) resid[s] = acc - obs[s];
}

// q_bar = (site synthesis)^T (2 r): one thread per lm, sites in order
__global__ void k_site_synth_T(int nsite, const int* __restrict__ site, int nlm, int nlat, int nphi,
                               const int* __restrict__ lm_m, const double* __restrict__ plm,
                               const double* __restrict__ cs, const double* __restrict__ sn,
                               const double* __restrict__ resid, double* __restrict__ qbar) {
  const int lm = blockIdx.x * blockDim.x + threadIdx.x;
  if (lm >= nlm) return;
  const int m = lm_m[lm];
  double br = 0.0, bi = 0.0;
  for (int s = 0; s < nsite; ++s) {
    const int g = site[s], j = g / nphi, i = g % nphi;
    const int t = (int)(((long long)m * i) % nphi);
    const double c = (m == 0 ? 1.0 : 2.0) * plm[(size_t)lm * nlat + j] * 2.0 * resid[s];
    br += c * cs[t];
    bi -= c * sn[t];
  }
  qbar[2 * lm] = br;
  qbar[2 * lm + 1] = (m == 0) ? 0.0 : bi;
}

// apply^T: sigma_bar += (gn - gu) q_bar; surface drift adjoints dUa_bar = -q_bar,
// dFa_bar = -q_bar / g (slot layout [dUa re, dUa im, dFa re, dFa im][nk])
__global__ void k_apply_T(int nlm, int nk, double g, const int* __restrict__ lm_l, const int* __restrict__ lm2k,
                          const double* __restrict__ gu, const double* __restrict__ gn,
                          const double* __restrict__ qbar, double* __restrict__ sbar, double* __restrict__ surf_bar) {
  const int lm = blockIdx.x * blockDim.x + threadIdx.x;
  if (lm >= nlm) return;
  const int l = lm_l[lm];
  const double qr = qbar[2 * lm], qi = qbar[2 * lm + 1];
  sbar[2 * lm] += (gn[l] - gu[l]) * qr;
  sbar[2 * lm + 1] += (gn[l] - gu[l]) * qi;
  if (l == 0) return;
  const int k = lm2k[lm];
  surf_bar[(size_t)0 * nk + k] = -qr;
  surf_bar[(size_t)1 * nk + k] = -qi;
  surf_bar[(size_t)2 * nk + k] = -qr / g;
  surf_bar[(size_t)3 * nk + k] = -qi / g;
}

// strain_coeffs transposed: (a, b, c)_bar -> (U0, U1, V0, V1)_bar
__device__ __forceinline__ void strain_T(const double ab[4], const double bb[4], const double cb[4], double J,
                                         double& u0, double& u1, double& v0, double& v1) {
  const double b3 = (J <= 2.0) ? 0.0 : bb[3], c3 = (J <= 2.0) ? 0.0 : cb[3];
  u0 = -ab[0] + bb[1] - bb[2] / J;
  u1 = ab[0] + cb[1] - cb[2] / J;
  v0 = -ab[1] - bb[1] + 0.5 * bb[2] + 0.5 * b3;
  v1 = ab[1] - cb[1] + 0.5 * cb[2] + 0.5 * c3;
}

// advance^T of the spectrally advanced (1-D) elements, one thread per (slot,
// re/im), elements in order: lam_new = (1 - M) lam; the strain adjoint
// -2 mu M lam goes to the nodal drift adjoints (this thread owns the column)
// and to sigma_bar through the unit-load response.
__global__ void k_adv1d_T(int ne, int nr, int nk, double dt, const int* __restrict__ kdeg,
                          const int* __restrict__ k2lm, const double* __restrict__ Jrv,
                          const double* __restrict__ xUn, const double* __restrict__ xVn,
                          const double* __restrict__ mu, const double* __restrict__ MkPerDt,
                          const char* __restrict__ active, const double* __restrict__ lam,
                          double* __restrict__ lam_new, double* __restrict__ dUn_bar, double* __restrict__ dVn_bar,
                          double* __restrict__ sbar) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x, ri = blockIdx.y;
  if (k >= nk) return;
  const int l = kdeg[k], lm = k2lm[k];
  const double J = Jrv[l];
  const double* xu = xUn + (size_t)l * nr;
  const double* xv = xVn + (size_t)l * nr;
  double* ub = dUn_bar + (size_t)ri * nr * nk + k;
  double* vb = dVn_bar + (size_t)ri * nr * nk + k;
  for (int node = 0; node < nr; ++node) {
    ub[(size_t)node * nk] = 0.0;
    vb[(size_t)node * nk] = 0.0;
  }
  double s_acc = 0.0;
  for (int e = 0; e < ne; ++e) {
    if (!active[e]) continue;
    const double Me = MkPerDt[e] * dt, om = 1.0 - Me, two_muM = 2.0 * mu[e] * Me;
    double ab[4], bb[4], cb[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const size_t iA = mem_idx(0, ri, e, m, k, ne, nk), iB = mem_idx(1, ri, e, m, k, ne, nk),
                   iC = mem_idx(2, ri, e, m, k, ne, nk);
      const double la = lam[iA], lb = lam[iB], lc = lam[iC];
      lam_new[iA] = om * la;
      lam_new[iB] = om * lb;
      lam_new[iC] = om * lc;
      ab[m] = -two_muM * la;
      bb[m] = -two_muM * lb;
      cb[m] = -two_muM * lc;
    }
    double u0, u1, v0, v1;
    strain_T(ab, bb, cb, J, u0, u1, v0, v1);
    ub[(size_t)e * nk] += u0;
    ub[(size_t)(e + 1) * nk] += u1;
    vb[(size_t)e * nk] += v0;
    vb[(size_t)(e + 1) * nk] += v1;
    s_acc += u0 * xu[e] + u1 * xu[e + 1] + v0 * xv[e] + v1 * xv[e + 1];
  }
  sbar[2 * lm + ri] += s_acc;
}

// transposed band solve with the dgbtf2 factor (A = P L U): U^T, then L^T with
// the row interchanges applied in reverse; right-hand side stride st
__device__ void band_solve_T_strided(const double* __restrict__ ab, int ldab, int n, int kl, int kv,
                                     const int* __restrict__ ipiv, double* x, size_t st) {
#define AB(row1, col1) ab[(size_t)((col1)-1) * ldab + ((row1)-1)]
  for (int j = 1; j <= n; ++j) {
    double t = x[(size_t)(j - 1) * st];
    const int lm = min(kv, j - 1);
    for (int i = 1; i <= lm; ++i) t -= AB(kv + 1 - i, j) * x[(size_t)(j - i - 1) * st];
    x[(size_t)(j - 1) * st] = t / AB(kv + 1, j);
  }
  for (int j = n - 1; j >= 1; --j) {
    const int lm = min(kl, n - j);
    double t = x[(size_t)(j - 1) * st];
    for (int i = 1; i <= lm; ++i) t -= AB(kv + 1 + i, j) * x[(size_t)(j + i - 1) * st];
    x[(size_t)(j - 1) * st] = t;
    const int p = ipiv[j - 1] + 1;
    if (p != j) {
      const double tmp = x[(size_t)(p - 1) * st];
      x[(size_t)(p - 1) * st] = x[(size_t)(j - 1) * st];
      x[(size_t)(j - 1) * st] = tmp;
    }
  }
#undef AB
}

// K^T: f_bar at an element's four test dofs (U_e, U_e+1, V_e, V_e+1) into the
// memory adjoint of that element (adds)
__device__ __forceinline__ void rhs_T(const double* __restrict__ Kp, const double fb[4], double* lam_new, int ri,
                                      int e, int k, int ne, int nk) {
#pragma unroll
  for (int s3 = 0; s3 < 3; ++s3)
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      double acc = 0.0;
#pragma unroll
      for (int t = 0; t < 4; ++t) acc += Kp[(t * 3 + s3) * 4 + m] * fb[t];
      lam_new[mem_idx(s3, ri, e, m, k, ne, nk)] += acc;
    }
}

// drift^T for degrees >= 2, one thread per (slot, re/im)
__global__ void k_drift_T(int ne, int nr, int nd, int nk, const int* __restrict__ kdeg, const double* __restrict__ ab,
                          const double* __restrict__ drv, const double* __restrict__ dcv, const int* __restrict__ ipiv,
                          const double* __restrict__ K, const double* __restrict__ dUn_bar,
                          const double* __restrict__ dVn_bar, const double* __restrict__ surf_bar,
                          double* __restrict__ w, double* __restrict__ lam_new) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x, ri = blockIdx.y;
  if (k >= nk) return;
  const int l = kdeg[k];
  if (l < 2) return;
  const double* dr = drv + (size_t)(l - 2) * nd;
  const double* dc = dcv + (size_t)(l - 2) * nd;
  double* x = w + (size_t)ri * nd * nk + k;
  for (int i = 0; i < nd; ++i) x[(size_t)i * nk] = 0.0;
  for (int node = 0; node < nr; ++node) {
    x[(size_t)(4 * node) * nk] = dUn_bar[((size_t)ri * nr + node) * nk + k];
    x[(size_t)(4 * node + 1) * nk] = dVn_bar[((size_t)ri * nr + node) * nk + k];
  }
  x[(size_t)(4 * (nr - 1)) * nk] += surf_bar[(size_t)(0 + ri) * nk + k];
  x[(size_t)(4 * (nr - 1) + 2) * nk] += surf_bar[(size_t)(2 + ri) * nk + k];
  for (int i = 0; i < nd; ++i) x[(size_t)i * nk] *= dc[i];
  band_solve_T_strided(ab + (size_t)(l - 2) * VG_LDAB * nd, VG_LDAB, nd, 6, 12, ipiv + (size_t)(l - 2) * nd, x, nk);
  for (int e = 0; e < ne; ++e) {
    const double fb[4] = {dr[4 * e] * x[(size_t)(4 * e) * nk], dr[4 * (e + 1)] * x[(size_t)(4 * (e + 1)) * nk],
                          dr[4 * e + 1] * x[(size_t)(4 * e + 1) * nk],
                          dr[4 * (e + 1) + 1] * x[(size_t)(4 * (e + 1) + 1) * nk]};
    rhs_T(K + ((size_t)l * ne + e) * 48, fb, lam_new, ri, e, k, ne, nk);
  }
}

// drift^T for degree 1 (slots 0, 1; four right-hand sides): the CM projection
// transposed, then the transposed Green's block
__global__ void __launch_bounds__(512) k_drift_T_deg1(int ne, int nr, int nk, int deg1_cm,
                                                      const double* __restrict__ dr1,
                                                      const double* __restrict__ null1,
                                                      const double* __restrict__ G1, const double* __restrict__ K,
                                                      const double* __restrict__ dUn_bar,
                                                      const double* __restrict__ dVn_bar,
                                                      const double* __restrict__ surf_bar,
                                                      double* __restrict__ lam_new) {
  extern __shared__ double sh[];
  const int ncol = 2 * nr, nrow = 2 * nr + 1;
  double* xb = sh;              // [4][nrow]
  double* fb = sh + 4 * nrow;   // [4][ncol]
  __shared__ double s_c[4];
  for (int t = threadIdx.x; t < 4 * nrow; t += blockDim.x) {
    const int q = t / nrow, r = t % nrow, kk = q >> 1, ri = q & 1;
    double v = 0.0;
    if (r < 2 * nr) {
      const int node = r >> 1;
      v = (r & 1) ? dVn_bar[((size_t)ri * nr + node) * nk + kk] : dUn_bar[((size_t)ri * nr + node) * nk + kk];
      if (node == nr - 1 && !(r & 1)) v += surf_bar[(size_t)(0 + ri) * nk + kk];
    } else if (deg1_cm) {
      v = surf_bar[(size_t)(2 + ri) * nk + kk];
    }
    xb[t] = v;
  }
  __syncthreads();
  const int fs = 4 * (nr - 1) + 2;
  const double fa_n = null1[fs];
  if (deg1_cm && fa_n != 0.0) {
    // forward: x += c null, c = -x[F] / fa_n  =>  c_bar = <x_bar, null>, x_bar[F] -= c_bar / fa_n
    if (threadIdx.x < 4) {
      double c = 0.0;
      for (int r = 0; r < nrow; ++r) {
        const int dof = (r < 2 * nr) ? 4 * (r >> 1) + (r & 1) : fs;
        c += xb[threadIdx.x * nrow + r] * null1[dof];
      }
      s_c[threadIdx.x] = c;
    }
    __syncthreads();
    if (threadIdx.x < 4) xb[threadIdx.x * nrow + 2 * nr] -= s_c[threadIdx.x] / fa_n;
    __syncthreads();
  }
  for (int t = threadIdx.x; t < 4 * ncol; t += blockDim.x) {
    const int q = t / ncol, c = t % ncol;
    double acc = 0.0;
    for (int r = 0; r < nrow; ++r) acc += G1[(size_t)r * ncol + c] * xb[q * nrow + r];
    const int node = c >> 1;
    fb[t] = dr1[4 * node + (c & 1)] * acc;  // bh row c = dr1 * f at (node, U or V)
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 4 * ne; t += blockDim.x) {
    const int q = t / ne, e = t % ne, kk = q >> 1, ri = q & 1;
    const double* f = fb + q * ncol;
    const double fe[4] = {f[2 * e], f[2 * (e + 1)], f[2 * e + 1], f[2 * (e + 1) + 1]};
    rhs_T(K + ((size_t)1 * ne + e) * 48, fe, lam_new, ri, e, kk, ne, nk);
  }
}

// ------------------------------------------------------------------ host

namespace {

struct AdjWork {
  DArr<double> sig, obs, resid, lam, lam_new, dUn_bar, dVn_bar, surf_bar, qbar, w, gsig, ckpt;
  DArr<int> site;
};

struct SkipOff {  // the drift skip gate is off inside the misfit entry points
  vg_handle* h;
  double saved;
  explicit SkipOff(vg_handle* hh) : h(hh), saved(hh->p.skip_tol) { h->p.skip_tol = 0.0; }
  ~SkipOff() { h->p.skip_tol = saved; }
};

void check_args(vg_handle* h, int nsteps, double dt, int nsite, const int* site) {
  if (nsteps < 1) throw Error("vg_misfit: nsteps must be >= 1");
  if (!(dt > 0.0)) throw Error("vg_misfit: dt_s must be > 0");
  if (nsite < 1 || !site) throw Error("vg_misfit: at least one site is required");
  for (int s = 0; s < nsite; ++s)
    if (site[s] < 0 || site[s] >= h->grid.ng) throw Error("vg_misfit: site index outside the Gauss grid");
}

void upload_inputs(vg_handle* h, AdjWork& W, int nsteps, const double* sigma, int nsite, const int* site,
                   const double* obs) {
  const size_t n2 = 2 * (size_t)h->grid.nlm;
  cudaStream_t s = h->stream;
  W.sig.alloc((size_t)nsteps * n2);
  W.sig.upload(sigma, (size_t)nsteps * n2, s);
  W.obs.alloc((size_t)nsteps * nsite);
  W.obs.upload(obs, (size_t)nsteps * nsite, s);
  W.resid.alloc((size_t)nsteps * nsite);
  W.site.alloc(nsite);
  W.site.upload(site, nsite, s);
}

// one forward step: drift, apply, site residuals of step n, memory advance
void fwd_step(vg_handle* h, AdjWork& W, int n, int nsite, double dt) {
  const Grid& G = h->grid;
  const size_t n2 = 2 * (size_t)G.nlm;
  const double* sig = W.sig.p + (size_t)n * n2;
  launch_drift(h);
  launch_apply(h, sig, h->d_ulm.p, h->d_ulm.p + n2);
  k_site_synth<<<nsite, 256, 0, h->stream>>>(nsite, W.site.p, G.nlm, G.nlat, G.nphi, G.d_lm_m.p, G.d_plm.p,
                                            G.d_cos.p, G.d_sin.p, h->d_ulm.p, h->d_ulm.p + n2,
                                            W.obs.p + (size_t)n * nsite, W.resid.p + (size_t)n * nsite);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  if (h->lat_visc) visc3d_advance(h, sig, dt);
  launch_advance_1d(h, sig, dt);
  h->cur = 1 - h->cur;
}

double sum_squares(vg_handle* h, const AdjWork& W, size_t count) {
  std::vector<double> r(count);
  W.resid.download(r.data(), count, h->stream);
  VG_CUDA(cudaStreamSynchronize(h->stream));
  double J = 0.0;
  for (double v : r) J += v * v;
  return J;
}

// the handle's memory at entry, put back at exit
struct StateGuard {
  vg_handle* h;
  DArr<double> saved;
  int cur;
  explicit StateGuard(vg_handle* hh) : h(hh), cur(hh->cur) {
    const size_t S = h->d_mem[h->cur].n;
    saved.alloc(S);
    VG_CUDA(cudaMemcpyAsync(saved.p, h->d_mem[h->cur].p, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  }
  void restore() {
    h->cur = cur;
    VG_CUDA(cudaMemcpyAsync(h->d_mem[h->cur].p, saved.p, saved.n * sizeof(double), cudaMemcpyDeviceToDevice,
                            h->stream));
    compute_mem_norm(h, h->cur);
    h->mem_norm = read_mem_norm(h, h->cur);
  }
};

}  // namespace

double misfit_dev(vg_handle* h, int nsteps, double dt, const double* sigma, int nsite, const int* site,
                  const double* obs) {
  check_args(h, nsteps, dt, nsite, site);
  SkipOff skip(h);
  StateGuard guard(h);
  AdjWork W;
  upload_inputs(h, W, nsteps, sigma, nsite, site, obs);
  compute_mem_norm(h, h->cur);
  for (int n = 0; n < nsteps; ++n) fwd_step(h, W, n, nsite, dt);
  const double J = sum_squares(h, W, (size_t)nsteps * nsite);
  guard.restore();
  return J;
}

double misfit_grad_dev(vg_handle* h, int nsteps, double dt, const double* sigma, int nsite, const int* site,
                       const double* obs, int ckpt, double* grad_sigma) {
  check_args(h, nsteps, dt, nsite, site);
  if (h->lat_visc && h->ne3d > 0)
    throw Error("vg_misfit_grad: elements with lateral viscosity are not differentiated yet");
  if (ckpt < 1) throw Error("vg_misfit_grad: ckpt_every must be >= 1");
  SkipOff skip(h);
  StateGuard guard(h);
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  const size_t n2 = 2 * (size_t)G.nlm, S = h->d_mem[0].n;
  const int nk = h->nk, nr = h->nr, ne = h->ne, nd = h->ndof;
  AdjWork W;
  upload_inputs(h, W, nsteps, sigma, nsite, site, obs);
  // forward sweep with checkpoints of the memory every `ckpt` steps (the
  // reverse sweep recomputes a segment from its checkpoint when it needs the
  // states; the transposes of the 1-D step do not depend on them)
  const int nck = (nsteps + ckpt - 1) / ckpt;
  W.ckpt.alloc((size_t)nck * S);
  compute_mem_norm(h, h->cur);
  for (int n = 0; n < nsteps; ++n) {
    if (n % ckpt == 0)
      VG_CUDA(cudaMemcpyAsync(W.ckpt.p + (size_t)(n / ckpt) * S, h->d_mem[h->cur].p, S * sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
    fwd_step(h, W, n, nsite, dt);
  }
  const double J = sum_squares(h, W, (size_t)nsteps * nsite);
  // reverse sweep
  W.lam.alloc(S);
  W.lam_new.alloc(S);
  W.dUn_bar.alloc((size_t)2 * nr * nk);
  W.dVn_bar.alloc((size_t)2 * nr * nk);
  W.surf_bar.alloc((size_t)4 * nk);
  W.qbar.alloc(n2);
  W.w.alloc((size_t)2 * nd * nk);
  W.gsig.alloc((size_t)nsteps * n2);
  const dim3 kg((nk + 127) / 128, 2);
  const size_t shm1 = (size_t)(4 * (2 * nr + 1) + 4 * 2 * nr) * sizeof(double);
  for (int n = nsteps - 1; n >= 0; --n) {
    double* sbar = W.gsig.p + (size_t)n * n2;
    k_site_synth_T<<<(G.nlm + 127) / 128, 128, 0, s>>>(nsite, W.site.p, G.nlm, G.nlat, G.nphi, G.d_lm_m.p, G.d_plm.p,
                                                      G.d_cos.p, G.d_sin.p, W.resid.p + (size_t)n * nsite, W.qbar.p);
    VG_CUDA(cudaMemsetAsync(W.surf_bar.p, 0, W.surf_bar.n * sizeof(double), s));
    k_apply_T<<<(G.nlm + 255) / 256, 256, 0, s>>>(G.nlm, nk, h->g, G.d_lm_l.p, h->d_lm2k.p, h->d_gu.p, h->d_gn.p,
                                                 W.qbar.p, sbar, W.surf_bar.p);
    k_adv1d_T<<<kg, 128, 0, s>>>(ne, nr, nk, dt, h->d_kdeg.p, h->d_k2lm.p, h->d_Jr.p, h->d_xUn.p, h->d_xVn.p,
                                 h->d_mu.p, h->d_MkPerDt.p, h->d_active1d.p, W.lam.p, W.lam_new.p, W.dUn_bar.p,
                                 W.dVn_bar.p, sbar);
    k_drift_T<<<kg, 128, 0, s>>>(ne, nr, nd, nk, h->d_kdeg.p, h->d_ab.p, h->d_dr.p, h->d_dc.p, h->d_ipiv.p,
                                 h->d_Krhs.p, W.dUn_bar.p, W.dVn_bar.p, W.surf_bar.p, W.w.p, W.lam_new.p);
    k_drift_T_deg1<<<1, 512, shm1, s>>>(ne, nr, nk, h->p.deg1_cm, h->d_dr1.p, h->d_null1.p, h->d_G1.p, h->d_Krhs.p,
                                        W.dUn_bar.p, W.dVn_bar.p, W.surf_bar.p, W.lam_new.p);
    h->n_launch += 5;
    VG_CUDA(cudaGetLastError());
    std::swap(W.lam.p, W.lam_new.p);
  }
  if (grad_sigma) W.gsig.download(grad_sigma, (size_t)nsteps * n2, s);
  VG_CUDA(cudaStreamSynchronize(s));
  guard.restore();
  return J;
}

}  // namespace vg

extern "C" int vg_misfit(vg_handle* h, int nsteps, double dt_s, const double* sigma_lm, int nsite, const int* site,
                         const double* obs, double* J) {
  if (!h) return 1;
  try {
    if (!sigma_lm || !obs || !J) throw vg::Error("vg_misfit: null argument");
    *J = vg::misfit_dev(h, nsteps, dt_s, sigma_lm, nsite, site, obs);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}

extern "C" int vg_misfit_grad(vg_handle* h, int nsteps, double dt_s, const double* sigma_lm, int nsite,
                              const int* site, const double* obs, int ckpt_every, double* J, double* grad_sigma) {
  if (!h) return 1;
  try {
    if (!sigma_lm || !obs || !J) throw vg::Error("vg_misfit_grad: null argument");
    *J = vg::misfit_grad_dev(h, nsteps, dt_s, sigma_lm, nsite, site, obs, ckpt_every, grad_sigma);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}
