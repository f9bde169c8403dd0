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
// With 3-D elements (FP64 path) the reverse sweep also runs the transposed
// pseudo-spectral advance (vg_visc3d.cu: scatter^T, analysis^T, longitude^T,
// synthesis^T, gather^T). Of the forward it needs only each step's grid of
// dyadic components before the factor -M dt (the longitude pass stores it,
// nlat x 3 ne3d x 6 x nphi doubles a step), for d J / d(M dt) and so the
// gradient with respect to the lateral log10-viscosity: a segment's grids are
// recomputed from its checkpoint, the last segment's kept from the forward.
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

// q_bar = (site synthesis)^T (2 r): a warp per lm, lanes over the sites
__global__ void __launch_bounds__(256) k_site_synth_T(int nsite, const int* __restrict__ site, int nlm, int nlat,
                                                      int nphi, const int* __restrict__ lm_m,
                                                      const double* __restrict__ plm, const double* __restrict__ cs,
                                                      const double* __restrict__ sn, const double* __restrict__ resid,
                                                      double* __restrict__ qbar) {
  const int lm = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (lm >= nlm) return;
  const int m = lm_m[lm];
  const double* P = plm + (size_t)lm * nlat;
  double br = 0.0, bi = 0.0;
  for (int s = lane; s < nsite; s += 32) {
    const int g = site[s], j = g / nphi, i = g % nphi;
    const int t = (int)(((long long)m * i) % nphi);
    const double c = (m == 0 ? 1.0 : 2.0) * P[j] * 2.0 * resid[s];
    br += c * cs[t];
    bi -= c * sn[t];
  }
  for (int o = 16; o > 0; o >>= 1) {
    br += __shfl_down_sync(0xffffffffu, br, o);
    bi += __shfl_down_sync(0xffffffffu, bi, o);
  }
  if (lane == 0) {
    qbar[2 * lm] = br;
    qbar[2 * lm + 1] = (m == 0) ? 0.0 : bi;
  }
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

// advance^T of the spectrally advanced (1-D) elements, a thread per (slot,
// element, re/im): lam_new = (1 - M) lam; the strain adjoint -2 mu M lam,
// transposed through the strain coefficients, kept per element as
// E[c][ri][e][k] (c: U0, U1, V0, V1 and the element's sigma_bar share)
__global__ void __launch_bounds__(256) k_adv1d_T_elem(int ne, int nr, int nk, double dt,
                                                      const int* __restrict__ kdeg, const double* __restrict__ Jrv,
                                                      const double* __restrict__ xUn, const double* __restrict__ xVn,
                                                      const double* __restrict__ mu,
                                                      const double* __restrict__ MkPerDt,
                                                      const char* __restrict__ active,
                                                      const double* __restrict__ lam, double* __restrict__ lam_new,
                                                      double* __restrict__ E) {
  const int k = blockIdx.x * 32 + threadIdx.x, e = blockIdx.y * 8 + threadIdx.y, ri = blockIdx.z;
  if (k >= nk || e >= ne) return;
  const size_t plane = (size_t)2 * ne * nk, at = ((size_t)ri * ne + e) * nk + k;
  if (!active[e]) {
    for (int c = 0; c < 5; ++c) E[c * plane + at] = 0.0;
    return;
  }
  const int l = kdeg[k];
  const double J = Jrv[l];
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
  const double* xu = xUn + (size_t)l * nr;
  const double* xv = xVn + (size_t)l * nr;
  E[0 * plane + at] = u0;
  E[1 * plane + at] = u1;
  E[2 * plane + at] = v0;
  E[3 * plane + at] = v1;
  E[4 * plane + at] = u0 * xu[e] + u1 * xu[e + 1] + v0 * xv[e] + v1 * xv[e + 1];
}

// nodal drift adjoints from the two elements that share each node; the node-0
// thread of each slot also adds the slot's sigma_bar (elements in order)
__global__ void __launch_bounds__(256) k_adv1d_T_node(int ne, int nr, int nk, const int* __restrict__ k2lm,
                                                      const double* __restrict__ E, double* __restrict__ dUn_bar,
                                                      double* __restrict__ dVn_bar, double* __restrict__ sbar) {
  const int k = blockIdx.x * 32 + threadIdx.x, node = blockIdx.y * 8 + threadIdx.y, ri = blockIdx.z;
  if (k >= nk || node >= nr) return;
  const size_t plane = (size_t)2 * ne * nk;
  const double* Er = E + (size_t)ri * ne * nk + k;
  double u = 0.0, v = 0.0;
  if (node < ne) {
    u += Er[0 * plane + (size_t)node * nk];
    v += Er[2 * plane + (size_t)node * nk];
  }
  if (node >= 1) {
    u += Er[1 * plane + (size_t)(node - 1) * nk];
    v += Er[3 * plane + (size_t)(node - 1) * nk];
  }
  dUn_bar[((size_t)ri * nr + node) * nk + k] = u;
  dVn_bar[((size_t)ri * nr + node) * nk + k] = v;
  if (node == 0) {
    double acc = 0.0;
    for (int e = 0; e < ne; ++e) acc += Er[4 * plane + (size_t)e * nk];
    sbar[2 * k2lm[k] + ri] += acc;
  }
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

// ---- shared-memory staging of the transposed sweeps (cp.async, double-buffered) ----
constexpr int TS_CH = 32;                     // band columns (sweep steps) per chunk
constexpr int TS_BAND = 2 * TS_CH * VG_LDAB;  // two band chunks
constexpr int TS_AUX = 2 * TS_CH * 32;        // two chunks of per-lane entering values
constexpr int TS_WARP = TS_BAND + TS_AUX;     // doubles of shared memory per warp
constexpr int TS_WARPS = 4;                   // warps (tasks) per block

__device__ __forceinline__ void ts_cp8(double* s, const double* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void ts_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void ts_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// band records of columns [c0, c0 + TS_CH) of one degree; zero outside [0, nd)
__device__ __forceinline__ void ts_stage_band(double* dst, const double* ab, int c0, int nd, int lane) {
  for (int t = lane; t < TS_CH * VG_LDAB; t += 32) {
    const int col = c0 + t / VG_LDAB;
    if (col >= 0 && col < nd)
      ts_cp8(dst + t, ab + (size_t)col * VG_LDAB + (t % VG_LDAB));
    else
      dst[t] = 0.0;
  }
}

// Transposed drift solves (degrees >= 2), one warp per task: up to 16 slots of
// one degree x (re, im), the forward sweeps' task list. With A = P L U the
// dgbtf2 factor (kl = 6, kv = 12) and the drift's right-hand side scaled by
// the column equilibration dc:
//   U^T sweep (ascending): x_j = (z_j - sum_{i<=12} U(j-i, j) x_{j-i}) / U(j, j),
//     z_j = dc_j (U-bar, V-bar, F-bar at the dofs of node j/4; surface terms at
//     the last node), the 12 previous values in registers;
//   L^T sweep (descending, pivots undone): x_j -= sum_{i<=6} L(j+i, j) x_{j+i},
//     then swap x_j and x_{j + jp_j}; a value leaves the 7-value window once
//     no later swap can reach it.
// The degree's band columns stream through shared memory in chunks of 32 so
// that every load on the recurrences is a shared-memory load; the per-lane
// entering values (U-bar / V-bar in the U^T sweep, its output in the L^T
// sweep) are staged the same way one chunk ahead.
__global__ void __launch_bounds__(32 * TS_WARPS) k_drift_T(int nr, int nd, int nk, const int4* __restrict__ tasks,
                                                           int ntask, const double* __restrict__ ab_all,
                                                           const double* __restrict__ dcv,
                                                           const double* __restrict__ dUn_bar,
                                                           const double* __restrict__ dVn_bar,
                                                           const double* __restrict__ surf_bar,
                                                           double* __restrict__ w) {
  constexpr int KL = 6, KV = 12;
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tix = blockIdx.x * TS_WARPS + warp;
  if (tix >= ntask) return;  // whole warp
  const int4 T = tasks[tix];
  const int l = T.x, k0 = T.y, nsl = T.z;
  const int sl = lane & 15, ri = lane >> 4;
  const bool valid = sl < nsl;
  const int k = k0 + (valid ? sl : 0);
  double* sband = smem + (size_t)warp * TS_WARP;
  double* saux = sband + TS_BAND;
  const double* ab = ab_all + (size_t)(l - 2) * VG_LDAB * nd;
  const double* dc = dcv + (size_t)(l - 2) * nd;
  const double* ub = dUn_bar + (size_t)ri * nr * nk + k;
  const double* vb = dVn_bar + (size_t)ri * nr * nk + k;
  double* x = w + (size_t)ri * nd * nk + k;
  const double sU = surf_bar[(size_t)(0 + ri) * nk + k], sF = surf_bar[(size_t)(2 + ri) * nk + k];
  // ---- U^T sweep ----
  // entering U-bar, V-bar of chunk c (columns 32c .. 32c+31 = nodes 8c .. 8c+7) at slot (2 node' + uv)
  auto stage_z = [&](double* dst, int c) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int node = 8 * c + (q >> 1);
      if (node < nr)
        ts_cp8(dst + q * 32 + lane, ((q & 1) ? vb : ub) + (size_t)node * nk);
      else
        dst[q * 32 + lane] = 0.0;
    }
  };
  const int nch = (nd + TS_CH - 1) / TS_CH;
  ts_stage_band(sband, ab, 0, nd, lane);
  stage_z(saux, 0);
  ts_commit();
  double wv[KV];  // wv[i] = x_{j-1-i}
#pragma unroll
  for (int i = 0; i < KV; ++i) wv[i] = 0.0;
  for (int c = 0; c < nch; ++c) {
    const int cur = c & 1;
    if (c + 1 < nch) {
      ts_stage_band(sband + (cur ^ 1) * TS_CH * VG_LDAB, ab, TS_CH * (c + 1), nd, lane);
      stage_z(saux + (cur ^ 1) * TS_CH * 32, c + 1);
      ts_commit();
      ts_wait<1>();
    } else {
      ts_wait<0>();
    }
    __syncwarp();
    const double* bandc = sband + cur * TS_CH * VG_LDAB;
    const double* zin = saux + cur * TS_CH * 32;
#pragma unroll 4
    for (int jj = 0; jj < TS_CH; ++jj) {
      const int j = TS_CH * c + jj;
      if (j >= nd) break;
      const int node = j >> 2, typ = j & 3;
      double raw = (typ == 0) ? zin[(2 * (jj >> 2)) * 32 + lane] : (typ == 1) ? zin[(2 * (jj >> 2) + 1) * 32 + lane] : 0.0;
      if (node == nr - 1) {
        if (typ == 0) raw += sU;
        if (typ == 2) raw = sF;
      }
      const double* col = bandc + jj * VG_LDAB;
      double t = __ldg(&dc[j]) * raw;
#pragma unroll
      for (int i = 1; i <= KV; ++i)
        if (i <= j) t -= col[KV - i] * wv[i - 1];
      t = t / col[KV];
      if (valid) x[(size_t)j * nk] = t;
#pragma unroll
      for (int i = KV - 1; i > 0; --i) wv[i] = wv[i - 1];
      wv[0] = t;
    }
    __syncwarp();  // the buffer just read is refilled by the next prefetch
  }
  __threadfence_block();  // x stores before this lane's own cp.async reads of them
  // ---- L^T sweep: steps j = nd-2 .. 0; chunk c covers j = jhi-31 .. jhi, jhi = nd-2-32c ----
  auto stage_x = [&](double* dst, int c) {
    const int jlo = nd - 2 - TS_CH * c - (TS_CH - 1);
#pragma unroll 4
    for (int q = 0; q < TS_CH; ++q) {
      const int j = jlo + q;
      if (j >= 0 && valid)
        ts_cp8(dst + q * 32 + lane, x + (size_t)j * nk);
      else
        dst[q * 32 + lane] = 0.0;
    }
  };
  double v[KL + 1];  // v[i] = x_{j+i}, starting at j = nd - 1 (nothing beyond it)
  v[0] = valid ? x[(size_t)(nd - 1) * nk] : 0.0;
#pragma unroll
  for (int i = 1; i <= KL; ++i) v[i] = 0.0;
  const int nchl = (nd - 1 + TS_CH - 1) / TS_CH;
  if (nchl > 0) {
    ts_stage_band(sband, ab, nd - 2 - (TS_CH - 1), nd, lane);
    stage_x(saux, 0);
    ts_commit();
  }
  for (int c = 0; c < nchl; ++c) {
    const int cur = c & 1, jlo = nd - 2 - TS_CH * c - (TS_CH - 1);
    if (c + 1 < nchl) {
      ts_stage_band(sband + (cur ^ 1) * TS_CH * VG_LDAB, ab, jlo - TS_CH, nd, lane);
      stage_x(saux + (cur ^ 1) * TS_CH * 32, c + 1);
      ts_commit();
      ts_wait<1>();
    } else {
      ts_wait<0>();
    }
    __syncwarp();
    const double* bandc = sband + cur * TS_CH * VG_LDAB;
    const double* xin = saux + cur * TS_CH * 32;
#pragma unroll 4
    for (int jj = TS_CH - 1; jj >= 0; --jj) {
      const int j = jlo + jj;
      if (j < 0) break;
      const double out = v[KL];  // x_{j+1+KL} is final
      if (valid && j + 1 + KL <= nd - 1) x[(size_t)(j + 1 + KL) * nk] = out;
#pragma unroll
      for (int i = KL; i > 0; --i) v[i] = v[i - 1];
      const double* col = bandc + jj * VG_LDAB;
      double t = xin[jj * 32 + lane];
#pragma unroll
      for (int i = 1; i <= KL; ++i)
        if (j + i <= nd - 1) t -= col[KV + i] * v[i];
      v[0] = t;
      const int d = (int)col[20];  // jp_j = ipiv_j - j, 0 .. KL
      if (d != 0) {
        double vd = v[0];
#pragma unroll
        for (int i = 1; i <= KL; ++i)
          if (i == d) {
            vd = v[i];
            v[i] = v[0];
          }
        v[0] = vd;
      }
    }
    __syncwarp();
  }
  if (valid) {
#pragma unroll
    for (int i = 0; i <= KL; ++i)
      if (i <= nd - 1) x[(size_t)i * nk] = v[i];
  }
}

// K^T after the transposed solves (degrees >= 2): a thread per (slot,
// element, re/im), f_bar = dr x at the element's four test dofs
__global__ void __launch_bounds__(256) k_rhs_T(int ne, int nd, int nk, const int* __restrict__ kdeg,
                                               const double* __restrict__ drv, const double* __restrict__ K,
                                               const double* __restrict__ w, double* __restrict__ lam_new) {
  const int k = blockIdx.x * 32 + threadIdx.x, e = blockIdx.y * 8 + threadIdx.y, ri = blockIdx.z;
  if (k >= nk || e >= ne) return;
  const int l = kdeg[k];
  if (l < 2) return;
  const double* dr = drv + (size_t)(l - 2) * nd;
  const double* x = w + (size_t)ri * nd * nk + k;
  const double fb[4] = {dr[4 * e] * x[(size_t)(4 * e) * nk], dr[4 * (e + 1)] * x[(size_t)(4 * (e + 1)) * nk],
                        dr[4 * e + 1] * x[(size_t)(4 * e + 1) * nk],
                        dr[4 * (e + 1) + 1] * x[(size_t)(4 * (e + 1) + 1) * nk]};
  rhs_T(K + ((size_t)l * ne + e) * 48, fb, lam_new, ri, e, k, ne, nk);
}

// drift^T for degree 1 (slots 0, 1; four right-hand sides): the CM projection
// transposed, then the transposed Green's block
__global__ void __launch_bounds__(512) k_drift_T_deg1(int ne, int nr, int nk, int deg1_cm,
                                                      const double* __restrict__ dr1,
                                                      const double* __restrict__ null1,
                                                      const double* __restrict__ G1T, const double* __restrict__ K,
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
  {  // f_bar = G1^T x_bar: a warp per column c (rows of G1T contiguous), lanes over r
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int c = wid; c < ncol; c += nw) {
      const double* gc = G1T + (size_t)c * nrow;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      for (int r = lane; r < nrow; r += 32) {
        const double gv = gc[r];
        a0 += gv * xb[r];
        a1 += gv * xb[nrow + r];
        a2 += gv * xb[2 * nrow + r];
        a3 += gv * xb[3 * nrow + r];
      }
      for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        a3 += __shfl_xor_sync(0xffffffffu, a3, o);
      }
      if (lane == 0) {
        const double sc = dr1[4 * (c >> 1) + (c & 1)];  // bh row c = dr1 * f at (node, U or V)
        fb[c] = sc * a0;
        fb[ncol + c] = sc * a1;
        fb[2 * ncol + c] = sc * a2;
        fb[3 * ncol + c] = sc * a3;
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 4 * ne; t += blockDim.x) {
    const int q = t / ne, e = t % ne, kk = q >> 1, ri = q & 1;
    const double* f = fb + q * ncol;
    const double fe[4] = {f[2 * e], f[2 * (e + 1)], f[2 * e + 1], f[2 * (e + 1) + 1]};
    rhs_T(K + ((size_t)1 * ne + e) * 48, fe, lam_new, ri, e, kk, ne, nk);
  }
}

// G1T[c][r] = G1[r][c] (degree-1 Green's block, rows r < nrow, columns c < ncol)
// d J / d pert = scale * rate * d J / d (M dt), in place (scale = -ln 10 dt)
__global__ void k_grad_pert(size_t n, double scale, const double* __restrict__ rate, double* __restrict__ g) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) g[t] *= scale * rate[t];
}

__global__ void k_transpose(int nrow, int ncol, const double* __restrict__ A, double* __restrict__ AT) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrow * ncol) return;
  const int r = t / ncol, c = t % ncol;
  AT[(size_t)c * nrow + r] = A[t];
}

// ------------------------------------------------------------------ host

namespace {

struct AdjWork {
  DArr<double> sig, obs, resid, lam, lam_new, dUn_bar, dVn_bar, surf_bar, qbar, w, gsig, ckpt, E, G1T;
  DArr<double> ckpt_norm, gseg, gradMdt;  // checkpoint norms, a segment's longitude grids, d J / d (M dt)
  DArr<int> site;
};

void adj_release(void* p) { delete static_cast<AdjWork*>(p); }

// the handle's work buffers, kept across calls (grown when a call needs more)
AdjWork& work_of(vg_handle* h) {
  if (!h->adj_work) {
    h->adj_work = new AdjWork();
    h->adj_release = adj_release;
  }
  return *static_cast<AdjWork*>(h->adj_work);
}

template <class T>
void ensure(DArr<T>& a, size_t count) {
  if (a.n < count) a.alloc(count);
}

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
  ensure(W.sig, (size_t)nsteps * n2);
  W.sig.upload(sigma, (size_t)nsteps * n2, s);
  ensure(W.obs, (size_t)nsteps * nsite);
  W.obs.upload(obs, (size_t)nsteps * nsite, s);
  ensure(W.resid, (size_t)nsteps * nsite);
  ensure(W.site, (size_t)nsite);
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
  advance_memory(h, sig, dt);
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
  DArr<double>& saved;
  int cur;
  StateGuard(vg_handle* hh, DArr<double>& buf) : h(hh), saved(buf), cur(hh->cur) {
    const size_t S = h->d_mem[h->cur].n;
    ensure(saved, S);
    VG_CUDA(cudaMemcpyAsync(saved.p, h->d_mem[h->cur].p, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  }
  void restore() {
    h->cur = cur;
    VG_CUDA(cudaMemcpyAsync(h->d_mem[h->cur].p, saved.p, h->d_mem[h->cur].n * sizeof(double),
                            cudaMemcpyDeviceToDevice, h->stream));
    compute_mem_norm(h, h->cur);
    h->mem_norm = read_mem_norm(h, h->cur);
  }
};

}  // namespace

double misfit_dev(vg_handle* h, int nsteps, double dt, const double* sigma, int nsite, const int* site,
                  const double* obs) {
  check_args(h, nsteps, dt, nsite, site);
  if (h->p.scheme != VG_SCHEME_FE) throw Error("vg_misfit: the response-level run follows the forward-Euler scheme");
  SkipOff skip(h);
  AdjWork& W = work_of(h);
  StateGuard guard(h, W.lam_new);
  upload_inputs(h, W, nsteps, sigma, nsite, site, obs);
  compute_mem_norm(h, h->cur);
  for (int n = 0; n < nsteps; ++n) fwd_step(h, W, n, nsite, dt);
  const double J = sum_squares(h, W, (size_t)nsteps * nsite);
  guard.restore();
  return J;
}

double misfit_grad_dev(vg_handle* h, int nsteps, double dt, const double* sigma, int nsite, const int* site,
                       const double* obs, int ckpt, double* grad_sigma, double* grad_pert) {
  check_args(h, nsteps, dt, nsite, site);
  const bool v3 = h->lat_visc && h->ne3d > 0;
  if (v3 && h->p.visc3d_precision != VG_VISC3D_FP64)
    throw Error("vg_misfit_grad: the 3-D adjoint follows the FP64 path (visc3d_precision = FP64)");
  if (ckpt < 1) throw Error("vg_misfit_grad: ckpt_every must be >= 1");
  if (h->p.scheme != VG_SCHEME_FE) throw Error("vg_misfit_grad: the adjoint follows the forward-Euler scheme");
  SkipOff skip(h);
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  const size_t n2 = 2 * (size_t)G.nlm, S = h->d_mem[0].n;
  const int nk = h->nk, nr = h->nr, ne = h->ne, nd = h->ndof;
  AdjWork& W = work_of(h);
  const int cur0 = h->cur;  // the entry state is checkpoint 0, put back at the end
  upload_inputs(h, W, nsteps, sigma, nsite, site, obs);
  // forward sweep with checkpoints of the memory every `ckpt` steps (the
  // reverse sweep recomputes a segment from its checkpoint when it needs the
  // states; the transposes of the 1-D step do not depend on them)
  const int nck = (nsteps + ckpt - 1) / ckpt;
  ensure(W.ckpt, (size_t)nck * S);
  ensure(W.ckpt_norm, (size_t)nck * nk);
  compute_mem_norm(h, h->cur);
  auto snapshot = [&](double* st, double* nm) {  // the state and its per-slot norms (the drift's gate)
    VG_CUDA(cudaMemcpyAsync(st, h->d_mem[h->cur].p, S * sizeof(double), cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(nm, h->d_mnorm.p + (size_t)h->cur * nk, nk * sizeof(double), cudaMemcpyDeviceToDevice,
                            s));
  };
  auto restore = [&](const double* st, const double* nm) {
    VG_CUDA(cudaMemcpyAsync(h->d_mem[h->cur].p, st, S * sizeof(double), cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(h->d_mnorm.p + (size_t)h->cur * nk, nm, nk * sizeof(double), cudaMemcpyDeviceToDevice,
                            s));
  };
  // with 3-D elements the reverse sweep needs every step's longitude grid; the
  // last segment's are kept from this sweep, the others recomputed from their
  // checkpoints
  const int last0 = ((nsteps - 1) / ckpt) * ckpt;
  const size_t gsz = (size_t)G.nlat * 3 * h->ne3d * 6 * G.nphi;
  if (v3) ensure(W.gseg, (size_t)std::min(ckpt, nsteps) * gsz);
  struct GridStore {  // the longitude pass stores its grid while set
    vg_handle* h;
    ~GridStore() { h->v3_gstore = nullptr; }
  } gstore_off{h};
  for (int n = 0; n < nsteps; ++n) {
    if (n % ckpt == 0) snapshot(W.ckpt.p + (size_t)(n / ckpt) * S, W.ckpt_norm.p + (size_t)(n / ckpt) * nk);
    h->v3_gstore = (v3 && n >= last0) ? W.gseg.p + (size_t)(n - last0) * gsz : nullptr;
    fwd_step(h, W, n, nsite, dt);
  }
  h->v3_gstore = nullptr;
  const double J = sum_squares(h, W, (size_t)nsteps * nsite);
  // reverse sweep
  ensure(W.lam, S);
  ensure(W.lam_new, S);
  ensure(W.dUn_bar, (size_t)2 * nr * nk);
  ensure(W.dVn_bar, (size_t)2 * nr * nk);
  ensure(W.surf_bar, (size_t)4 * nk);
  ensure(W.qbar, n2);
  ensure(W.w, (size_t)2 * nd * nk);
  ensure(W.gsig, (size_t)nsteps * n2);
  VG_CUDA(cudaMemsetAsync(W.lam.p, 0, S * sizeof(double), s));  // no terminal cost: lam_N = 0
  VG_CUDA(cudaMemsetAsync(W.gsig.p, 0, (size_t)nsteps * n2 * sizeof(double), s));
  const dim3 eg((nk + 31) / 32, (ne + 7) / 8, 2), ng_((nk + 31) / 32, (nr + 7) / 8, 2);
  ensure(W.E, (size_t)5 * 2 * ne * nk);
  {
    const int nrow = 2 * nr + 1, ncol = 2 * nr;
    if (W.G1T.n != (size_t)nrow * ncol) {
      W.G1T.alloc((size_t)nrow * ncol);
      k_transpose<<<(nrow * ncol + 255) / 256, 256, 0, s>>>(nrow, ncol, h->d_G1.p, W.G1T.p);
      VG_CUDA(cudaGetLastError());
    }
  }
  const size_t shm1 = (size_t)(4 * (2 * nr + 1) + 4 * 2 * nr) * sizeof(double);
  const size_t ts_smem = (size_t)TS_WARPS * TS_WARP * sizeof(double);
  static std::atomic<bool> ts_attr{false};  // set once; concurrent handles may race to it
  if (!ts_attr) {
    VG_CUDA(cudaFuncSetAttribute(k_drift_T, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ts_smem));
    ts_attr = true;
  }
  if (v3) {
    const size_t ngm = (size_t)h->ne3d * G.ng;
    ensure(W.gradMdt, ngm);
    VG_CUDA(cudaMemsetAsync(W.gradMdt.p, 0, ngm * sizeof(double), s));
  }
  for (int n = nsteps - 1; n >= 0; --n) {
    double* sbar = W.gsig.p + (size_t)n * n2;
    const int n0 = (n / ckpt) * ckpt;
    if (v3 && n < last0 && n % ckpt == ckpt - 1) {
      // this segment's longitude grids, recomputed from its checkpoint
      restore(W.ckpt.p + (size_t)(n / ckpt) * S, W.ckpt_norm.p + (size_t)(n / ckpt) * nk);
      for (int q = n0; q <= n; ++q) {
        h->v3_gstore = W.gseg.p + (size_t)(q - n0) * gsz;
        fwd_step(h, W, q, nsite, dt);
      }
      h->v3_gstore = nullptr;
    }
    k_site_synth_T<<<(G.nlm * 32 + 255) / 256, 256, 0, s>>>(nsite, W.site.p, G.nlm, G.nlat, G.nphi, G.d_lm_m.p, G.d_plm.p,
                                                      G.d_cos.p, G.d_sin.p, W.resid.p + (size_t)n * nsite, W.qbar.p);
    VG_CUDA(cudaMemsetAsync(W.surf_bar.p, 0, W.surf_bar.n * sizeof(double), s));
    k_apply_T<<<(G.nlm + 255) / 256, 256, 0, s>>>(G.nlm, nk, h->g, G.d_lm_l.p, h->d_lm2k.p, h->d_gu.p, h->d_gn.p,
                                                 W.qbar.p, sbar, W.surf_bar.p);
    k_adv1d_T_elem<<<eg, dim3(32, 8), 0, s>>>(ne, nr, nk, dt, h->d_kdeg.p, h->d_Jr.p, h->d_xUn.p, h->d_xVn.p,
                                               h->d_mu.p, h->d_MkPerDt.p, h->d_active1d.p, W.lam.p, W.lam_new.p,
                                               W.E.p);
    if (v3) visc3d_adjoint(h, W.gseg.p + (size_t)(n - n0) * gsz, dt, W.lam.p, W.lam_new.p, W.E.p, W.gradMdt.p);
    k_adv1d_T_node<<<ng_, dim3(32, 8), 0, s>>>(ne, nr, nk, h->d_k2lm.p, W.E.p, W.dUn_bar.p, W.dVn_bar.p, sbar);
    k_drift_T<<<(h->ntask + TS_WARPS - 1) / TS_WARPS, 32 * TS_WARPS, ts_smem, s>>>(
        nr, nd, nk, h->d_tasks.p, h->ntask, h->d_ab.p, h->d_dc.p, W.dUn_bar.p, W.dVn_bar.p, W.surf_bar.p, W.w.p);
    k_rhs_T<<<eg, dim3(32, 8), 0, s>>>(ne, nd, nk, h->d_kdeg.p, h->d_dr.p, h->d_Krhs.p, W.w.p, W.lam_new.p);
    k_drift_T_deg1<<<1, 512, shm1, s>>>(ne, nr, nk, h->p.deg1_cm, h->d_dr1.p, h->d_null1.p, W.G1T.p, h->d_Krhs.p,
                                        W.dUn_bar.p, W.dVn_bar.p, W.surf_bar.p, W.lam_new.p);
    h->n_launch += 7;
    VG_CUDA(cudaGetLastError());
    std::swap(W.lam.p, W.lam_new.p);
  }
  if (grad_sigma) W.gsig.download(grad_sigma, (size_t)nsteps * n2, s);
  if (grad_pert) {
    // d J / d pert = d J / d(M dt) * (-ln 10) M dt on the 3-D elements' grid,
    // (nphi, nlat, ne) like vg_enable_visc3d's input; zero elsewhere. Formed
    // on the device; each 3-D element's slab is copied into place.
    const size_t ng = G.ng;
    if (v3) {
      const size_t n3 = (size_t)h->ne3d * ng;
      k_grad_pert<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(n3, -std::log(10.0) * dt, h->d_MkPerDt3.p,
                                                              W.gradMdt.p);
      ++h->n_launch;
      VG_CUDA(cudaGetLastError());
    }
    int e3 = 0;
    for (int e = 0; e < ne; ++e) {
      if (e3 < h->ne3d && h->e3d_h[e3] == e) {
        VG_CUDA(cudaMemcpyAsync(grad_pert + (size_t)e * ng, W.gradMdt.p + (size_t)e3 * ng, ng * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
        ++e3;
      } else {
        std::fill(grad_pert + (size_t)e * ng, grad_pert + (size_t)(e + 1) * ng, 0.0);
      }
    }
  }
  h->cur = cur0;
  VG_CUDA(cudaMemcpyAsync(h->d_mem[h->cur].p, W.ckpt.p, S * sizeof(double), cudaMemcpyDeviceToDevice, s));
  compute_mem_norm(h, h->cur);
  h->mem_norm = read_mem_norm(h, h->cur);
  return J;
}

}  // namespace vg

extern "C" int vg_misfit(vg_handle* h, int nsteps, double dt_s, const double* sigma_lm, int nsite, const int* site,
                         const double* obs, double* J) {
  if (!h) return 1;
  try {
    if (!sigma_lm || !obs || !J) throw vg::Error("vg_misfit: null argument");
    if (h->tor_on) throw vg::Error("vg_misfit: the misfit runs carry no toroidal channels (toroidal = 0)");
    *J = vg::misfit_dev(h, nsteps, dt_s, sigma_lm, nsite, site, obs);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}

extern "C" int vg_misfit_grad(vg_handle* h, int nsteps, double dt_s, const double* sigma_lm, int nsite,
                              const int* site, const double* obs, int ckpt_every, double* J, double* grad_sigma,
                              double* grad_pert) {
  if (!h) return 1;
  try {
    if (!sigma_lm || !obs || !J) throw vg::Error("vg_misfit_grad: null argument");
    if (h->tor_on) throw vg::Error("vg_misfit_grad: the toroidal channels are not differentiated (toroidal = 0)");
    *J = vg::misfit_grad_dev(h, nsteps, dt_s, sigma_lm, nsite, site, obs, ckpt_every, grad_sigma, grad_pert);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}
