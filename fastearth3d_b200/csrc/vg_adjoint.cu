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


// ------------------------------------------------------------------ sea-level misfit
//
// The coupled forward (vg_update: forward-Euler sub-steps, each a drift, a
// sea-level solve and a memory advance) with its discrete decisions held
// fixed (the sub-steps, the ocean function of every pass, the inner
// iterations done) is linear in the ice thickness, so its adjoint runs the
// transposes backwards through the recorded decisions. One sea-level pass
// (src/vilma_sle.f90:248-340) with ocean function C:
//   dig = ice (1 - C) - ice_ref (1 - C0),  ice_int = -(rho_i / rho_w) <dig>
//   K iterations of  r <- Sraw + dphi,  Sraw = Synth(apply(A(rho_i dig + rho_w C r + wcorr)))  (N - u),
//                    dphi = (ice_int - <C Sraw> + zeta_int) / <C>
// (<f> = sum w_j dlon f, the surface integral), from r_0 = the previous pass's
// r (the first pass: the previous sub-step's rsl, or zero without a warm
// start); the closing load sigma = A(rho_i dig + rho_w C r + wcorr) drives
// the memory advance. The transposes of the grid transforms are scaled
// transforms: Synth^T(y) = (c_m / sc) A(y / w_j) and A^T(s) = sc w_j
// Synth(s / c_m), with sc = 2 pi / nphi, c_0 = 1, c_m = 2.

// residuals of one interval's rsl at the sites
__global__ void k_site_resid(int nsite, const int* __restrict__ site, const double* __restrict__ rsl,
                             const double* __restrict__ obs, double* __restrict__ resid) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsite) resid[s] = rsl[site[s]] - obs[s];
}

// rbar(site) += 2 resid: one thread, sites in order (a repeated site adds up
// in a fixed order)
__global__ void k_site_scatter(int nsite, const int* __restrict__ site, const double* __restrict__ resid,
                               double* __restrict__ rbar) {
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (int s = 0; s < nsite; ++s) rbar[site[s]] += 2.0 * resid[s];
}

// a pass's ocean function (0 / 1 doubles) as bytes
__global__ void k_c_bytes(int ng, const double* __restrict__ C, unsigned char* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ng) out[i] = C[i] != 0.0 ? 1 : 0;
}

// per-row sums of lam
__global__ void k_rev_rows(int nphi, const double* __restrict__ lam, double* __restrict__ rows) {
  __shared__ double red[128];
  const int j = blockIdx.x;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) acc += lam[(size_t)j * nphi + i];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) rows[j] = acc;
}

// dphi_bar = sum of lam (rows in order): scal[0] = <C Sraw>_bar = -dphi_bar / <C>,
// scal[1] += ice_int_bar = dphi_bar / <C>
__global__ void k_rev_scal(int nlat, const double* __restrict__ rows, double C_int, double* __restrict__ scal) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double acc = 0.0;
  for (int j = 0; j < nlat; ++j) acc += rows[j];
  scal[0] = -acc / C_int;
  scal[1] += acc / C_int;
}

// Sraw_bar = lam + scal[0] C w_j dlon, divided by w_j for the analysis that
// forms the synthesis transpose
__global__ void k_rev_y(int ng, int nphi, const double* __restrict__ lam, const unsigned char* __restrict__ C,
                        const double* __restrict__ wts, double dlon, const double* __restrict__ scal,
                        double* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ng) return;
  const double w = wts[p / nphi];
  out[p] = (lam[p] + (C[p] ? scal[0] * w * dlon : 0.0)) / w;
}

// q_bar = (c_m / sc) q (the synthesis transpose of Sraw_bar, q the analysis of
// Sraw_bar / w_j); apply^T: sigma_bar = (gn - gu) q_bar, the surface drift
// adjoints dUa_bar -= q_bar, dFa_bar -= q_bar / g; out = sigma_bar / c_m for
// the synthesis that forms the analysis transpose
__global__ void k_rev_apply(int nlm, int nk, double g, double sc, const int* __restrict__ lm_l,
                            const int* __restrict__ lm_m, const int* __restrict__ lm2k, const double* __restrict__ gu,
                            const double* __restrict__ gn, const double* __restrict__ q, double* __restrict__ surf_bar,
                            double* __restrict__ out) {
  const int lm = blockIdx.x * blockDim.x + threadIdx.x;
  if (lm >= nlm) return;
  const int l = lm_l[lm], m = lm_m[lm];
  const double cm = (m == 0) ? 1.0 : 2.0;
  const double qr = q[2 * lm] * cm / sc, qi = (m == 0) ? 0.0 : q[2 * lm + 1] * cm / sc;
  const double gd = gn[l] - gu[l];
  out[2 * lm] = gd * qr / cm;
  out[2 * lm + 1] = gd * qi / cm;
  if (l == 0) return;
  const int k = lm2k[lm];
  surf_bar[(size_t)0 * nk + k] -= qr;
  surf_bar[(size_t)1 * nk + k] -= qi;
  surf_bar[(size_t)2 * nk + k] -= qr / g;
  surf_bar[(size_t)3 * nk + k] -= qi / g;
}

// s / c_m (the closing load's sigma_bar, ahead of the analysis transpose)
__global__ void k_lm_div_cm(int nlm, const int* __restrict__ lm_m, const double* __restrict__ in,
                            double* __restrict__ out) {
  const int lm = blockIdx.x * blockDim.x + threadIdx.x;
  if (lm >= nlm) return;
  const double cm = (lm_m[lm] == 0) ? 1.0 : 2.0;
  out[2 * lm] = in[2 * lm] / cm;
  out[2 * lm + 1] = in[2 * lm + 1] / cm;
}

// load_bar = sc w_j g (g the synthesis of sigma_bar / c_m); lam_out (= or, with
// add, +=) rho_w C load_bar; digbar += rho_i load_bar
__global__ void k_rev_load(int ng, int nphi, const double* __restrict__ g, const double* __restrict__ wts, double sc,
                           const unsigned char* __restrict__ C, int add, double* __restrict__ lam_out,
                           double* __restrict__ digbar) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ng) return;
  const double lb = sc * wts[p / nphi] * g[p];
  const double v = C[p] ? RHO_WATER * lb : 0.0;
  lam_out[p] = add ? lam_out[p] + v : v;
  digbar[p] += RHO_ICE * lb;
}

// the end of a pass: ice_now_bar = (1 - C) (digbar - (rho_i / rho_w) ice_int_bar
// w_j dlon), into the adjoints of this interval's end ice (frac) and of the
// previous interval's (1 - frac; none for the first interval of the call)
__global__ void k_rev_ice(int ng, int nphi, const unsigned char* __restrict__ C, const double* __restrict__ digbar,
                          const double* __restrict__ wts, double dlon, const double* __restrict__ scal, int with_int,
                          double frac, double* __restrict__ gi1, double* __restrict__ gi0) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ng || C[p]) return;
  double d = digbar[p];
  if (with_int) d -= (RHO_ICE / RHO_WATER) * scal[1] * wts[p / nphi] * dlon;
  gi1[p] += frac * d;
  if (gi0) gi0[p] += (1.0 - frac) * d;
}

// sum over the 3-D elements' grids (n3 fields of ng) into y, divided by w_j
// (the synthesis transpose of the lateral field's gradient)
__global__ void k_sum_fields_w(int n3, int ng, int nphi, const double* __restrict__ f, const double* __restrict__ wts,
                               double* __restrict__ y) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ng) return;
  double acc = 0.0;
  for (int e = 0; e < n3; ++e) acc += f[(size_t)e * ng + p];
  y[p] = acc / wts[p / nphi];
}

// q_bar = (c_m / sc) q, the imaginary part of m = 0 zero
__global__ void k_synthT_scale(int nlm, double sc, const int* __restrict__ lm_m, double* __restrict__ q) {
  const int lm = blockIdx.x * blockDim.x + threadIdx.x;
  if (lm >= nlm) return;
  const int m = lm_m[lm];
  const double cm = (m == 0) ? 1.0 : 2.0;
  q[2 * lm] *= cm / sc;
  q[2 * lm + 1] = (m == 0) ? 0.0 : q[2 * lm + 1] * cm / sc;
}

// ------------------------------------------------------------------ host

namespace {


// tape of the coupled forward (sea-level misfit): per accepted forward-Euler
// sub-step its interval, interpolation fraction, length and sea-level passes;
// per pass its inner iterations and ocean area, its ocean function as bytes
struct TapePass {
  int K;         // inner iterations done (0 without an ocean)
  double C_int;  // ocean area <C>
};
struct TapeSub {
  int n;        // interval
  double frac;  // where the sub-step ends in its interval (ice interpolation)
  double dt;    // length [s]
  int pass0, npass;
};
struct SleTape {
  std::vector<TapeSub> subs;
  std::vector<TapePass> passes;
  DArr<unsigned char> cb;  // the passes' ocean functions, ng bytes each
  size_t pass_cap = 0;
  double* gseg = nullptr;  // the sub-steps' longitude grids (3-D elements), gsz doubles each
  size_t gsz = 0;
  int gcap = 0;
  int interval = 0;
  size_t att_pass0 = 0;
  double att_frac = 0.0, att_dt = 0.0;
};

struct AdjWork {
  DArr<double> sig, obs, resid, lam, lam_new, dUn_bar, dVn_bar, surf_bar, qbar, w, gsig, ckpt, E, G1T;
  DArr<double> ckpt_norm, gseg, gradMdt;  // checkpoint norms, a segment's longitude grids, d J / d (M dt)
  // the toroidal channels: memory adjoints, element and nodal W adjoints, forcing adjoints, checkpoints
  DArr<double> lam_t, lam_t_new, Et, Wb, gb, ckpt_t;
  DArr<int> site;
  // sea-level misfit: interval-end ice, checkpoints (rsl and entering ice
  // beside the memory), the entry state, the reverse sweep's grid and
  // spectral work arrays, d J / d ice, the tape
  DArr<double> ice, ck_rsl, ck_hice;
  DriverSnap entry;
  DArr<double> rA, rB, digbar, ybuf, gbuf, obuf, sbuf, scal, rows, gice;
  SleTape tape;
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
  DArr<double>& saved_t;
  int cur;
  StateGuard(vg_handle* hh, DArr<double>& buf, DArr<double>& buf_t) : h(hh), saved(buf), saved_t(buf_t), cur(hh->cur) {
    const size_t S = h->d_mem[h->cur].n;
    ensure(saved, S);
    VG_CUDA(cudaMemcpyAsync(saved.p, h->d_mem[h->cur].p, S * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    if (h->tor_on) {
      ensure(saved_t, h->d_tmem[h->cur].n);
      VG_CUDA(cudaMemcpyAsync(saved_t.p, h->d_tmem[h->cur].p, h->d_tmem[h->cur].n * sizeof(double),
                              cudaMemcpyDeviceToDevice, h->stream));
    }
  }
  void restore() {
    h->cur = cur;
    VG_CUDA(cudaMemcpyAsync(h->d_mem[h->cur].p, saved.p, h->d_mem[h->cur].n * sizeof(double),
                            cudaMemcpyDeviceToDevice, h->stream));
    if (h->tor_on)
      VG_CUDA(cudaMemcpyAsync(h->d_tmem[h->cur].p, saved_t.p, h->d_tmem[h->cur].n * sizeof(double),
                              cudaMemcpyDeviceToDevice, h->stream));
    compute_mem_norm(h, h->cur);
    h->mem_norm = read_mem_norm(h, h->cur);
  }
};


// buffers and one-time attributes of a reverse sweep
void reverse_prepare(vg_handle* h, AdjWork& W) {
  const int nk = h->nk, nr = h->nr, ne = h->ne, nd = h->ndof;
  const size_t S = h->d_mem[0].n;
  ensure(W.lam, S);
  ensure(W.lam_new, S);
  ensure(W.dUn_bar, (size_t)2 * nr * nk);
  ensure(W.dVn_bar, (size_t)2 * nr * nk);
  ensure(W.surf_bar, (size_t)4 * nk);
  ensure(W.qbar, 2 * (size_t)h->grid.nlm);
  ensure(W.w, (size_t)2 * nd * nk);
  ensure(W.E, (size_t)5 * 2 * ne * nk);
  if (h->tor_on) {
    ensure(W.lam_t, h->d_tmem[0].n);
    ensure(W.lam_t_new, h->d_tmem[0].n);
    ensure(W.Et, (size_t)2 * 2 * ne * nk);
    ensure(W.Wb, (size_t)2 * nr * nk);
    ensure(W.gb, (size_t)2 * nr * nk);
    VG_CUDA(cudaMemsetAsync(W.lam_t.p, 0, W.lam_t.n * sizeof(double), h->stream));  // no terminal cost
  }
  const int nrow = 2 * nr + 1, ncol = 2 * nr;
  if (W.G1T.n != (size_t)nrow * ncol) {
    W.G1T.alloc((size_t)nrow * ncol);
    k_transpose<<<(nrow * ncol + 255) / 256, 256, 0, h->stream>>>(nrow, ncol, h->d_G1.p, W.G1T.p);
    VG_CUDA(cudaGetLastError());
  }
  static std::atomic<bool> ts_attr{false};  // set once; concurrent handles may race to it
  if (!ts_attr) {
    VG_CUDA(cudaFuncSetAttribute(k_drift_T, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(TS_WARPS * TS_WARP * sizeof(double))));
    ts_attr = true;
  }
}

// advance^T of one step of length dt: lam -> lam_new ((1 - M) lam on the 1-D
// elements, gather^T on the 3-D ones, whose grid the forward stored in
// gstore; gw d J / d (M dt) into gradMdt), the nodal drift adjoints, and
// sigma_bar += the load's share (sbar)
void advance_T(vg_handle* h, AdjWork& W, double dt, const double* gstore, double gw, double* sbar) {
  const int nk = h->nk, nr = h->nr, ne = h->ne;
  const dim3 eg((nk + 31) / 32, (ne + 7) / 8, 2), ng_((nk + 31) / 32, (nr + 7) / 8, 2);
  cudaStream_t s = h->stream;
  k_adv1d_T_elem<<<eg, dim3(32, 8), 0, s>>>(ne, nr, nk, dt, h->d_kdeg.p, h->d_Jr.p, h->d_xUn.p, h->d_xVn.p,
                                             h->d_mu.p, h->d_MkPerDt.p, h->d_active1d.p, W.lam.p, W.lam_new.p,
                                             W.E.p);
  if (h->tor_on) advance_1d_tor_T(h, dt, W.lam_t.p, W.lam_t_new.p, W.Et.p);
  if (h->lat_visc && h->ne3d > 0)
    visc3d_adjoint(h, gstore, dt, W.lam.p, W.lam_new.p, W.E.p, W.gradMdt.p, gw, h->tor_on ? W.lam_t.p : nullptr,
                   h->tor_on ? W.lam_t_new.p : nullptr, h->tor_on ? W.Et.p : nullptr);
  k_adv1d_T_node<<<ng_, dim3(32, 8), 0, s>>>(ne, nr, nk, h->d_k2lm.p, W.E.p, W.dUn_bar.p, W.dVn_bar.p, sbar);
  h->n_launch += 2;
  VG_CUDA(cudaGetLastError());
}

// drift^T: the nodal (dUn_bar, dVn_bar) and surface (surf_bar) drift
// adjoints into the memory adjoint lam_new (adds)
void drift_T(vg_handle* h, AdjWork& W) {
  const int nk = h->nk, nr = h->nr, ne = h->ne, nd = h->ndof;
  const dim3 eg((nk + 31) / 32, (ne + 7) / 8, 2);
  cudaStream_t s = h->stream;
  const size_t shm1 = (size_t)(4 * (2 * nr + 1) + 4 * 2 * nr) * sizeof(double);
  const size_t ts_smem = (size_t)TS_WARPS * TS_WARP * sizeof(double);
  k_drift_T<<<(h->ntask + TS_WARPS - 1) / TS_WARPS, 32 * TS_WARPS, ts_smem, s>>>(
      nr, nd, nk, h->d_tasks.p, h->ntask, h->d_ab.p, h->d_dc.p, W.dUn_bar.p, W.dVn_bar.p, W.surf_bar.p, W.w.p);
  k_rhs_T<<<eg, dim3(32, 8), 0, s>>>(ne, nd, nk, h->d_kdeg.p, h->d_dr.p, h->d_Krhs.p, W.w.p, W.lam_new.p);
  k_drift_T_deg1<<<1, 512, shm1, s>>>(ne, nr, nk, h->p.deg1_cm, h->d_dr1.p, h->d_null1.p, W.G1T.p, h->d_Krhs.p,
                                      W.dUn_bar.p, W.dVn_bar.p, W.surf_bar.p, W.lam_new.p);
  h->n_launch += 3;
  VG_CUDA(cudaGetLastError());
  if (h->tor_on) drift_tor_T(h, W.Et.p, W.Wb.p, W.gb.p, W.lam_t_new.p);
}

// the memory adjoints of the next step become the current ones
void swap_adjoints(vg_handle* h, AdjWork& W) {
  std::swap(W.lam.p, W.lam_new.p);
  if (h->tor_on) std::swap(W.lam_t.p, W.lam_t_new.p);
}

}  // namespace

double misfit_dev(vg_handle* h, int nsteps, double dt, const double* sigma, int nsite, const int* site,
                  const double* obs) {
  check_args(h, nsteps, dt, nsite, site);
  if (h->p.scheme != VG_SCHEME_FE) throw Error("vg_misfit: the response-level run follows the forward-Euler scheme");
  SkipOff skip(h);
  AdjWork& W = work_of(h);
  StateGuard guard(h, W.lam_new, W.lam_t_new);
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
  const int nk = h->nk, ne = h->ne;
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
  const size_t ST = h->tor_on ? h->d_tmem[0].n : 0;  // the toroidal memory beside it
  if (ST) ensure(W.ckpt_t, (size_t)nck * ST);
  auto snapshot = [&](double* st, double* nm, int c) {  // the state and its per-slot norms (the drift's gate)
    VG_CUDA(cudaMemcpyAsync(st, h->d_mem[h->cur].p, S * sizeof(double), cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(nm, h->d_mnorm.p + (size_t)h->cur * nk, nk * sizeof(double), cudaMemcpyDeviceToDevice,
                            s));
    if (ST)
      VG_CUDA(cudaMemcpyAsync(W.ckpt_t.p + (size_t)c * ST, h->d_tmem[h->cur].p, ST * sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
  };
  auto restore = [&](const double* st, const double* nm, int c) {
    VG_CUDA(cudaMemcpyAsync(h->d_mem[h->cur].p, st, S * sizeof(double), cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(h->d_mnorm.p + (size_t)h->cur * nk, nm, nk * sizeof(double), cudaMemcpyDeviceToDevice,
                            s));
    if (ST)
      VG_CUDA(cudaMemcpyAsync(h->d_tmem[h->cur].p, W.ckpt_t.p + (size_t)c * ST, ST * sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
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
    if (n % ckpt == 0)
      snapshot(W.ckpt.p + (size_t)(n / ckpt) * S, W.ckpt_norm.p + (size_t)(n / ckpt) * nk, n / ckpt);
    h->v3_gstore = (v3 && n >= last0) ? W.gseg.p + (size_t)(n - last0) * gsz : nullptr;
    fwd_step(h, W, n, nsite, dt);
  }
  h->v3_gstore = nullptr;
  const double J = sum_squares(h, W, (size_t)nsteps * nsite);
  // reverse sweep
  reverse_prepare(h, W);
  ensure(W.gsig, (size_t)nsteps * n2);
  VG_CUDA(cudaMemsetAsync(W.lam.p, 0, S * sizeof(double), s));  // no terminal cost: lam_N = 0
  VG_CUDA(cudaMemsetAsync(W.gsig.p, 0, (size_t)nsteps * n2 * sizeof(double), s));
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
      restore(W.ckpt.p + (size_t)(n / ckpt) * S, W.ckpt_norm.p + (size_t)(n / ckpt) * nk, n / ckpt);
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
    h->n_launch += 2;
    VG_CUDA(cudaGetLastError());
    advance_T(h, W, dt, v3 ? W.gseg.p + (size_t)(n - n0) * gsz : nullptr, 1.0, sbar);
    drift_T(h, W);
    swap_adjoints(h, W);
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
  if (ST)
    VG_CUDA(cudaMemcpyAsync(h->d_tmem[h->cur].p, W.ckpt_t.p, ST * sizeof(double), cudaMemcpyDeviceToDevice, s));
  compute_mem_norm(h, h->cur);
  h->mem_norm = read_mem_norm(h, h->cur);
  return J;
}


// ------------------------------------------------------------------ sea-level misfit (host)

void tape_attempt_begin(vg_handle* h, double frac, double dt) {
  SleTape* T = static_cast<SleTape*>(h->sle_tape);
  if (!T) return;
  T->att_pass0 = T->passes.size();
  T->att_frac = frac;
  T->att_dt = dt;
  if (T->gseg) {
    if ((int)T->subs.size() >= T->gcap)
      throw Error("vg_sle_misfit_grad: a checkpoint segment has more sub-steps than its grid store (the guard "
                  "rejected sub-steps); use a smaller ckpt_every");
    h->v3_gstore = T->gseg + T->subs.size() * T->gsz;
  }
}

void tape_pass(vg_handle* h, double C_int, int n_inner) {
  SleTape* T = static_cast<SleTape*>(h->sle_tape);
  if (!T) return;
  if (T->passes.size() >= T->pass_cap)
    throw Error("vg_sle_misfit_grad: a checkpoint segment has more sea-level passes than the tape holds; use a "
                "smaller ckpt_every");
  const int ng = h->grid.ng;
  k_c_bytes<<<(ng + 255) / 256, 256, 0, h->stream>>>(ng, h->d_C.p, T->cb.p + T->passes.size() * (size_t)ng);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  T->passes.push_back({C_int > 0.0 ? n_inner : 0, C_int});
}

void tape_attempt_end(vg_handle* h, bool accepted) {
  SleTape* T = static_cast<SleTape*>(h->sle_tape);
  if (!T) return;
  if (accepted)
    T->subs.push_back({T->interval, T->att_frac, T->att_dt, (int)T->att_pass0,
                       (int)(T->passes.size() - T->att_pass0)});
  else
    T->passes.resize(T->att_pass0);
  h->v3_gstore = nullptr;
}

namespace {

void sle_check(vg_handle* h, int nsteps, double dt_yr, const double* ice, int nsite, const int* site,
               const double* obs) {
  if (!ice || !obs) throw Error("vg_sle_misfit: null argument");
  if (nsteps < 1) throw Error("vg_sle_misfit: nsteps must be >= 1");
  if (!(dt_yr > 0.0)) throw Error("vg_sle_misfit: dt_yr must be > 0");
  if (nsite < 1 || !site) throw Error("vg_sle_misfit: at least one site is required");
  for (int s = 0; s < nsite; ++s)
    if (site[s] < 0 || site[s] >= h->grid.ng) throw Error("vg_sle_misfit: site index outside the Gauss grid");
  if (!h->have_reference) throw Error("vg_sle_misfit: call vg_set_reference first (solid_earth_init)");
  if (h->p.scheme != VG_SCHEME_FE) throw Error("vg_sle_misfit: the coupled misfit follows the forward-Euler scheme");
  if (h->rot_on) throw Error("vg_sle_misfit: rotational feedback is not differentiated (rotation = 0)");
}

// forward-Euler sub-steps of an interval by the Maxwell-CFL rule of the driver
int fe_substeps(const vg_handle* h, double dt_yr) {
  const vg_params& p = h->p;
  const double span = dt_yr * SEC_PER_YEAR;
  double dt_stab = h->max_rate > 0.0 ? p.cfl / h->max_rate : span;
  dt_stab = std::min(dt_stab, p.dt_max);
  if (p.dt_min > 0.0) dt_stab = std::max(dt_stab, p.dt_min);
  return std::max(1, (int)std::ceil(span / dt_stab - 1.0e-9));
}

// the interval driver's state at entry (memory, norms, sea-level fields and
// the last load spectrum, clocks and counters), put back at exit, also when
// the call fails
struct DriverGuard {
  vg_handle* h;
  DriverSnap& snap;
  bool done = false;
  DriverGuard(vg_handle* hh, DriverSnap& sn) : h(hh), snap(sn) { snap.save(h); }
  void restore() {
    done = true;
    h->sle_tape = nullptr;
    h->v3_gstore = nullptr;
    snap.restore(h);
  }
  ~DriverGuard() {
    if (!done) {
      try {
        restore();
      } catch (...) {
      }
    }
  }
};

void sle_upload(vg_handle* h, AdjWork& W, int nsteps, const double* ice, int nsite, const int* site,
                const double* obs) {
  const size_t ng = h->grid.ng;
  cudaStream_t s = h->stream;
  ensure(W.ice, (size_t)nsteps * ng);
  W.ice.upload(ice, (size_t)nsteps * ng, s);
  ensure(W.obs, (size_t)nsteps * nsite);
  W.obs.upload(obs, (size_t)nsteps * nsite, s);
  ensure(W.resid, (size_t)nsteps * nsite);
  ensure(W.site, (size_t)nsite);
  W.site.upload(site, nsite, s);
}

// interval n of the coupled forward (the driver's own update) and its site residuals
void sle_interval(vg_handle* h, AdjWork& W, int n, double dt_yr, int nsite) {
  const size_t ng = h->grid.ng;
  W.tape.interval = n;
  update_dev(h, W.ice.p + (size_t)n * ng, dt_yr);
  k_site_resid<<<(nsite + 127) / 128, 128, 0, h->stream>>>(nsite, W.site.p, h->d_rsl.p,
                                                          W.obs.p + (size_t)n * nsite, W.resid.p + (size_t)n * nsite);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// One pass's adjoint iterations (the pass's K inner iterations in reverse)
// from rb, the adjoint of the pass's final r, to the adjoint of its starting
// r (left in rb); digbar and scal[1] (ice_int_bar) accumulate, surf_bar too.
void rev_pass(vg_handle* h, AdjWork& W, const unsigned char* C, const TapePass& P, double*& rb, double*& rb2) {
  const Grid& G = h->grid;
  const int ng = G.ng, nphi = G.nphi, nlat = G.nlat, nlm = G.nlm;
  const double dlon = 2.0 * PI / (double)nphi, sc = dlon;
  cudaStream_t s = h->stream;
  const int eg = (ng + 255) / 256, lg = (nlm + 255) / 256;
  for (int k = 0; k < P.K; ++k) {
    k_rev_rows<<<nlat, 128, 0, s>>>(nphi, rb, W.rows.p);
    k_rev_scal<<<1, 32, 0, s>>>(nlat, W.rows.p, P.C_int, W.scal.p);
    k_rev_y<<<eg, 256, 0, s>>>(ng, nphi, rb, C, G.d_wts.p, dlon, W.scal.p, W.ybuf.p);
    h->n_launch += 3;
    VG_CUDA(cudaGetLastError());
    sht_analysis_dev(h, W.ybuf.p, W.obuf.p, 1);
    k_rev_apply<<<lg, 256, 0, s>>>(nlm, h->nk, h->g, sc, G.d_lm_l.p, G.d_lm_m.p, h->d_lm2k.p, h->d_gu.p, h->d_gn.p,
                                   W.obuf.p, W.surf_bar.p, W.sbuf.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
    sht_synthesis_dev(h, W.sbuf.p, W.gbuf.p, 1);
    k_rev_load<<<eg, 256, 0, s>>>(ng, nphi, W.gbuf.p, G.d_wts.p, sc, C, 0, rb2, W.digbar.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
    std::swap(rb, rb2);
  }
}

// the reverse of one accepted sub-step: lam = the memory adjoint after it,
// rb = the adjoint of its final rsl; on return lam = the adjoint before it,
// rb = the adjoint of the rsl it started from
void rev_substep(vg_handle* h, AdjWork& W, const TapeSub& sb, double dt_ref, bool warm, double*& rb,
                 double*& rb2) {
  const Grid& G = h->grid;
  const int ng = G.ng, nphi = G.nphi, nlm = G.nlm;
  const size_t n2 = 2 * (size_t)nlm;
  const double dlon = 2.0 * PI / (double)nphi, sc = dlon;
  cudaStream_t s = h->stream;
  SleTape& T = W.tape;
  const int eg = (ng + 255) / 256, lg = (nlm + 255) / 256;
  // memory advance^T: the closing load's adjoint sigma_bar (qbar) and the nodal drift adjoints
  VG_CUDA(cudaMemsetAsync(W.qbar.p, 0, n2 * sizeof(double), s));
  VG_CUDA(cudaMemsetAsync(W.surf_bar.p, 0, W.surf_bar.n * sizeof(double), s));
  const double* gst = T.gseg ? T.gseg + (size_t)(&sb - T.subs.data()) * T.gsz : nullptr;
  advance_T(h, W, sb.dt, gst, sb.dt / dt_ref, W.qbar.p);
  // closing load^T: rb += rho_w C r_bar, digbar = rho_i load_bar (last pass's C)
  VG_CUDA(cudaMemsetAsync(W.digbar.p, 0, (size_t)ng * sizeof(double), s));
  const unsigned char* Clast = T.cb.p + (size_t)(sb.pass0 + sb.npass - 1) * ng;
  k_lm_div_cm<<<lg, 256, 0, s>>>(nlm, G.d_lm_m.p, W.qbar.p, W.obuf.p);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  sht_synthesis_dev(h, W.obuf.p, W.gbuf.p, 1);
  k_rev_load<<<eg, 256, 0, s>>>(ng, nphi, W.gbuf.p, G.d_wts.p, sc, Clast, 1, rb, W.digbar.p);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  // the passes, last first
  double* gi1 = W.gice.p + (size_t)sb.n * ng;
  double* gi0 = sb.n > 0 ? W.gice.p + (size_t)(sb.n - 1) * ng : nullptr;
  for (int io = sb.npass - 1; io >= 0; --io) {
    const TapePass& P = T.passes[sb.pass0 + io];
    const unsigned char* C = T.cb.p + (size_t)(sb.pass0 + io) * ng;
    if (io != sb.npass - 1) VG_CUDA(cudaMemsetAsync(W.digbar.p, 0, (size_t)ng * sizeof(double), s));
    VG_CUDA(cudaMemsetAsync(W.scal.p, 0, 2 * sizeof(double), s));
    rev_pass(h, W, C, P, rb, rb2);
    k_rev_ice<<<eg, 256, 0, s>>>(ng, nphi, C, W.digbar.p, G.d_wts.p, dlon, W.scal.p, P.K > 0 ? 1 : 0, sb.frac, gi1,
                                 gi0);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  // the first pass started from the previous sub-step's rsl (warm start) or from zero
  if (!warm) VG_CUDA(cudaMemsetAsync(rb, 0, (size_t)ng * sizeof(double), s));
  // drift^T: the surface drift adjoints of every inner iteration and the nodal ones of the advance
  drift_T(h, W);
  swap_adjoints(h, W);
}

}  // namespace

double sle_misfit_dev(vg_handle* h, int nsteps, double dt_yr, const double* ice, int nsite, const int* site,
                      const double* obs) {
  sle_check(h, nsteps, dt_yr, ice, nsite, site, obs);
  SkipOff skip(h);
  AdjWork& W = work_of(h);
  DriverGuard guard(h, W.entry);
  sle_upload(h, W, nsteps, ice, nsite, site, obs);
  for (int n = 0; n < nsteps; ++n) sle_interval(h, W, n, dt_yr, nsite);
  const double J = sum_squares(h, W, (size_t)nsteps * nsite);
  guard.restore();
  return J;
}

double sle_misfit_grad_dev(vg_handle* h, int nsteps, double dt_yr, const double* ice, int nsite, const int* site,
                           const double* obs, int ckpt, double* grad_ice, double* grad_pert, double* grad_pert_lm) {
  sle_check(h, nsteps, dt_yr, ice, nsite, site, obs);
  if (ckpt < 1) throw Error("vg_sle_misfit_grad: ckpt_every must be >= 1");
  const bool v3 = h->lat_visc && h->ne3d > 0;
  if (v3 && h->p.visc3d_precision != VG_VISC3D_FP64)
    throw Error("vg_sle_misfit_grad: the 3-D adjoint follows the FP64 path (visc3d_precision = FP64)");
  SkipOff skip(h);
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  const size_t ng = G.ng, S = h->d_mem[0].n, nk = h->nk;
  AdjWork& W = work_of(h);
  DriverGuard guard(h, W.entry);
  sle_upload(h, W, nsteps, ice, nsite, site, obs);
  const double dt_ref = dt_yr * SEC_PER_YEAR;
  // checkpoints every ckpt intervals: memory, its per-slot norms, rsl, the
  // entering ice and the clocks
  const int nck = (nsteps + ckpt - 1) / ckpt, seg = std::min(ckpt, nsteps);
  ensure(W.ckpt, (size_t)nck * S);
  ensure(W.ckpt_norm, (size_t)nck * nk);
  ensure(W.ck_rsl, (size_t)nck * ng);
  ensure(W.ck_hice, (size_t)nck * ng);
  const size_t STt = h->tor_on ? h->d_tmem[0].n : 0;  // the toroidal memory
  if (STt) ensure(W.ckpt_t, (size_t)nck * STt);
  std::vector<double> ck_ts(nck), ck_ty(nck), ck_mn(nck);
  auto snapshot = [&](int c) {
    VG_CUDA(cudaMemcpyAsync(W.ckpt.p + (size_t)c * S, h->d_mem[h->cur].p, S * sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(W.ckpt_norm.p + (size_t)c * nk, h->d_mnorm.p + (size_t)h->cur * nk, nk * sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(W.ck_rsl.p + (size_t)c * ng, h->d_rsl.p, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(W.ck_hice.p + (size_t)c * ng, h->d_h_ice.p, ng * sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
    if (STt)
      VG_CUDA(cudaMemcpyAsync(W.ckpt_t.p + (size_t)c * STt, h->d_tmem[h->cur].p, STt * sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
    ck_ts[c] = h->time_s;
    ck_ty[c] = h->time_yr;
    ck_mn[c] = h->mem_norm;
  };
  auto restore = [&](int c) {
    VG_CUDA(cudaMemcpyAsync(h->d_mem[h->cur].p, W.ckpt.p + (size_t)c * S, S * sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(h->d_mnorm.p + (size_t)h->cur * nk, W.ckpt_norm.p + (size_t)c * nk, nk * sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(h->d_rsl.p, W.ck_rsl.p + (size_t)c * ng, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
    VG_CUDA(cudaMemcpyAsync(h->d_h_ice.p, W.ck_hice.p + (size_t)c * ng, ng * sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
    if (STt)
      VG_CUDA(cudaMemcpyAsync(h->d_tmem[h->cur].p, W.ckpt_t.p + (size_t)c * STt, STt * sizeof(double),
                              cudaMemcpyDeviceToDevice, s));
    h->time_s = ck_ts[c];
    h->time_yr = ck_ty[c];
    h->mem_norm = ck_mn[c];
  };
  // the tape of one checkpoint segment: its passes' ocean functions and, with
  // 3-D elements, its sub-steps' longitude grids
  SleTape& T = W.tape;
  const int nsub = fe_substeps(h, dt_yr);
  T.pass_cap = (size_t)seg * (nsub + 4) * std::max(1, h->p.sle_n_outer);
  if (T.cb.n < T.pass_cap * ng) T.cb.alloc(T.pass_cap * ng);
  T.gsz = v3 ? (size_t)G.nlat * 3 * h->ne3d * 6 * G.nphi : 0;
  T.gcap = v3 ? seg * nsub + 4 : 0;
  if (v3) ensure(W.gseg, (size_t)T.gcap * T.gsz);
  T.gseg = v3 ? W.gseg.p : nullptr;
  auto record_segment = [&](int c, bool with_resid) {
    T.subs.clear();
    T.passes.clear();
    h->sle_tape = &T;
    const int a = c * ckpt, b = std::min(nsteps, a + ckpt);
    for (int n = a; n < b; ++n) {
      if (with_resid) {
        sle_interval(h, W, n, dt_yr, nsite);
      } else {
        T.interval = n;
        update_dev(h, W.ice.p + (size_t)n * ng, dt_yr);
      }
    }
    h->sle_tape = nullptr;
  };
  // forward sweep: the last segment is recorded on the way
  for (int c = 0; c < nck; ++c) {
    snapshot(c);
    if (c == nck - 1) {
      record_segment(c, true);
    } else {
      for (int n = c * ckpt; n < (c + 1) * ckpt; ++n) sle_interval(h, W, n, dt_yr, nsite);
    }
  }
  const double J = sum_squares(h, W, (size_t)nsteps * nsite);
  // reverse sweep
  reverse_prepare(h, W);
  ensure(W.rA, ng);
  ensure(W.rB, ng);
  ensure(W.digbar, ng);
  ensure(W.ybuf, ng);
  ensure(W.gbuf, ng);
  ensure(W.obuf, 2 * (size_t)G.nlm);
  ensure(W.sbuf, 2 * (size_t)G.nlm);
  ensure(W.scal, 2);
  ensure(W.rows, (size_t)G.nlat);
  ensure(W.gice, (size_t)nsteps * ng);
  VG_CUDA(cudaMemsetAsync(W.lam.p, 0, S * sizeof(double), s));
  VG_CUDA(cudaMemsetAsync(W.rA.p, 0, ng * sizeof(double), s));
  VG_CUDA(cudaMemsetAsync(W.gice.p, 0, (size_t)nsteps * ng * sizeof(double), s));
  if (v3) {
    ensure(W.gradMdt, (size_t)h->ne3d * ng);
    VG_CUDA(cudaMemsetAsync(W.gradMdt.p, 0, (size_t)h->ne3d * ng * sizeof(double), s));
  }
  double* rb = W.rA.p;
  double* rb2 = W.rB.p;
  const bool warm = h->p.sle_warm_start != 0;
  for (int c = nck - 1; c >= 0; --c) {
    if (c != nck - 1) {
      restore(c);
      record_segment(c, false);
    }
    const int a = c * ckpt, b = std::min(nsteps, a + ckpt);
    int q = (int)T.subs.size() - 1;
    for (int n = b - 1; n >= a; --n) {
      k_site_scatter<<<1, 32, 0, s>>>(nsite, W.site.p, W.resid.p + (size_t)n * nsite, rb);
      ++h->n_launch;
      VG_CUDA(cudaGetLastError());
      for (; q >= 0 && T.subs[q].n == n; --q) rev_substep(h, W, T.subs[q], dt_ref, warm, rb, rb2);
    }
    if (q != -1) throw Error("vg_sle_misfit_grad: the recorded sub-steps do not match the segment's intervals");
  }
  if (grad_ice) W.gice.download(grad_ice, (size_t)nsteps * ng, s);
  if (v3 && (grad_pert || grad_pert_lm)) {
    const size_t n3 = (size_t)h->ne3d * ng;
    k_grad_pert<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(n3, -std::log(10.0) * dt_ref, h->d_MkPerDt3.p,
                                                            W.gradMdt.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  if (grad_pert) {
    int e3 = 0;
    for (int e = 0; e < h->ne; ++e) {
      if (v3 && e3 < h->ne3d && h->e3d_h[e3] == e) {
        VG_CUDA(cudaMemcpyAsync(grad_pert + (size_t)e * ng, W.gradMdt.p + (size_t)e3 * ng, ng * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
        ++e3;
      } else {
        std::fill(grad_pert + (size_t)e * ng, grad_pert + (size_t)(e + 1) * ng, 0.0);
      }
    }
  }
  if (grad_pert_lm) {
    // the lateral field shared by the 3-D elements as a spectrum: d J / d q =
    // Synth^T(sum over the elements of d J / d pert) = (c_m / sc) A(. / w_j)
    const size_t n2 = 2 * (size_t)G.nlm;
    if (v3) {
      k_sum_fields_w<<<(unsigned)((ng + 255) / 256), 256, 0, s>>>(h->ne3d, (int)ng, G.nphi, W.gradMdt.p, G.d_wts.p,
                                                                  W.ybuf.p);
      sht_analysis_dev(h, W.ybuf.p, W.obuf.p, 1);
      k_synthT_scale<<<(G.nlm + 255) / 256, 256, 0, s>>>(G.nlm, 2.0 * PI / (double)G.nphi, G.d_lm_m.p, W.obuf.p);
      h->n_launch += 2;
      VG_CUDA(cudaGetLastError());
      W.obuf.download(grad_pert_lm, n2, s);
    } else {
      std::fill(grad_pert_lm, grad_pert_lm + n2, 0.0);
    }
  }
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
                              const int* site, const double* obs, int ckpt_every, double* J, double* grad_sigma,
                              double* grad_pert) {
  if (!h) return 1;
  try {
    if (!sigma_lm || !obs || !J) throw vg::Error("vg_misfit_grad: null argument");
    *J = vg::misfit_grad_dev(h, nsteps, dt_s, sigma_lm, nsite, site, obs, ckpt_every, grad_sigma, grad_pert);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}

extern "C" int vg_sle_misfit(vg_handle* h, int nsteps, double dt_yr, const double* ice, int nsite, const int* site,
                             const double* obs, double* J) {
  if (!h) return 1;
  try {
    if (!J) throw vg::Error("vg_sle_misfit: null argument");
    *J = vg::sle_misfit_dev(h, nsteps, dt_yr, ice, nsite, site, obs);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}

extern "C" int vg_sle_misfit_grad(vg_handle* h, int nsteps, double dt_yr, const double* ice, int nsite,
                                  const int* site, const double* obs, int ckpt_every, double* J, double* grad_ice,
                                  double* grad_pert, double* grad_pert_lm) {
  if (!h) return 1;
  try {
    if (!J) throw vg::Error("vg_sle_misfit_grad: null argument");
    *J = vg::sle_misfit_grad_dev(h, nsteps, dt_yr, ice, nsite, site, obs, ckpt_every, grad_ice, grad_pert,
                                 grad_pert_lm);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}
