// Field-driver kernels of the 1-D (spectral) path: the per-(l,m) drift solve
// with the reference's skip gate, the affine apply, and the forward-Euler
// memory advance with the per-slot memory norm that the next drift gate and
// the stepper's guard read (src/vilma_response.f90:679-864, 944-992;
// src/vilma_viscoelastic.f90:329-589).
//
// Drift solve (degrees >= 2), two kernels:
//   k_drift_rhs    one thread per (slot, re/im, node): the dissipative forcing
//                  -int tau:d eps at the node's U and V dofs from its two
//                  elements, equilibrated (b = Dr f). Streams the memory state
//                  with full parallelism.
//   k_drift_solve  one thread per (slot, re/im): the pivoted band sweeps of
//                  dgbtrs with the active window in registers (7 values in the
//                  L sweep, kl = 6; 13 in the U sweep, kv = 12). Only the L-sweep
//                  output y goes through memory (L2-resident scratch).
// Degree 1 (bordered, dense): a mat-vec with the precomputed response block G1.
#include <cstdio>
#include <cstring>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

struct DriftArgs {
  const double* mem;                  // current state buffer
  const double* mnorm;                // per-slot norms of the current buffer
  const unsigned long long* maxbits;  // global max of the current buffer
  double skip_tol;
  const double* r;
  const double *sa, *sb, *sc, *nrmc;
  const double *ab, *dr, *dc, *rdiag;
  const int* ipiv;
  const int* kdeg;
  double* bh;  // equilibrated RHS (2, 2*nr, nk)
  double* ys;  // L-sweep output (2, nd, nk)
  double *dUn, *dVn, *drift;
  int ne, nr, nd, nk;
  const double *dr1, *null1, *G1;
  int deg1_cm;
  const double* K;     // dissipative-forcing coefficients (lmax+1, ne, 48)
  const int4* tasks;   // sweep tasks (degree, first slot, slots)
  int ntask;
};

// Element forcing of one (slot, re/im) at two of its test dofs, from the
// precomputed linear map K (floc_t = sum_{s,m} K[t][s][m] mem_s[m]).
__device__ __forceinline__ void element_floc2(const DriftArgs& A, int l, int k, int ri, int e, int t0, int t1,
                                              double& f0, double& f1) {
  const double* Kp = A.K + ((size_t)l * A.ne + e) * 48;
  double a0 = 0.0, a1 = 0.0;
#pragma unroll
  for (int s3 = 0; s3 < 3; ++s3)
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const double v = A.mem[mem_idx(s3, ri, e, m, k, A.ne, A.nk)];
      a0 += __ldg(&Kp[(t0 * 3 + s3) * 4 + m]) * v;
      a1 += __ldg(&Kp[(t1 * 3 + s3) * 4 + m]) * v;
    }
  f0 = a0;
  f1 = a1;
}

__device__ __forceinline__ double skip_threshold(const DriftArgs& A) {
  return A.skip_tol * __longlong_as_double((long long)*A.maxbits);
}

// One element's contribution to the four test dofs (U_e, U_e+1, V_e, V_e+1):
// 2-point radial Gauss quadrature of sum_lam norm_lam tau^lam d eps^lam
// (src/vilma_viscoelastic.f90:441-480).
__device__ __forceinline__ void element_floc(const DriftArgs& A, int l, int k, int ri, int e, double floc[4]) {
  const double xg = 0.5773502691896257;
  const double* sa = A.sa + l * 16;
  const double* sb = A.sb + l * 16;
  const double* sc = A.sc + l * 16;
  const double* nrm = A.nrmc + l * 4;
  double rk = A.r[e], rk1 = A.r[e + 1], h = rk1 - rk;
  double Am[4], Bm[4], Cm[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    Am[m] = A.mem[mem_idx(0, ri, e, m, k, A.ne, A.nk)];
    Bm[m] = A.mem[mem_idx(1, ri, e, m, k, A.ne, A.nk)];
    Cm[m] = A.mem[mem_idx(2, ri, e, m, k, A.ne, A.nk)];
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) floc[t] = 0.0;
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
        double deps = __ldg(&sa[t * 4 + m]) / h + __ldg(&sb[t * 4 + m]) * psik / ra + __ldg(&sc[t * 4 + m]) * psik1 / ra;
        D = D + __ldg(&nrm[m]) * tauV[m] * deps;
      }
      floc[t] = floc[t] - D * ra * ra * h * 0.5;
    }
  }
}

// b(U_node) = dr * (floc1(e = node-1) + floc0(e = node)), likewise V with floc3/floc2:
// the reference's accumulation order (element e adds to nodes e, e+1 in turn).
__global__ void __launch_bounds__(128) k_drift_rhs(DriftArgs A) {
  int k = blockIdx.x * 32 + threadIdx.x, node = blockIdx.y * 4 + threadIdx.y, ri = blockIdx.z;
  if (k >= A.nk || node >= A.nr) return;
  if (A.mnorm[k] <= skip_threshold(A)) return;
  int l = A.kdeg[k];
  double fU = 0.0, fV = 0.0, a, b2;
  if (node >= 1) {  // element node-1: its second node's U, V (test dofs 1, 3)
    element_floc2(A, l, k, ri, node - 1, 1, 3, a, b2);
    fU = a;
    fV = b2;
  }
  if (node < A.ne) {  // element node: its first node's U, V (test dofs 0, 2)
    element_floc2(A, l, k, ri, node, 0, 2, a, b2);
    fU = fU + a;
    fV = fV + b2;
  }
  const double* dr = (l == 1) ? A.dr1 : A.dr + (size_t)(l - 2) * A.nd;
  double* b = A.bh + ((size_t)ri * 2 * A.nr + 2 * node) * A.nk + k;
  b[0] = __ldg(&dr[4 * node]) * fU;
  b[A.nk] = __ldg(&dr[4 * node + 1]) * fV;
}

// ---- shared-memory staging of the sweeps (cp.async, double-buffered) ----
constexpr int SW_CH = 32;                            // band columns (sweep steps) per chunk
constexpr int SW_BAND = 2 * SW_CH * VG_LDAB;         // two band chunks
constexpr int SW_AUX = 2 * SW_CH * 32;               // two chunks of per-lane values (b or y)
constexpr int SW_WARP = SW_BAND + SW_AUX;            // doubles of shared memory per warp
constexpr int SW_WARPS = 4;                          // warps (tasks) per block

__device__ __forceinline__ void cp8(double* s, const double* g) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// band records of columns [c0, c0 + SW_CH) of one degree; zero outside [0, nd)
__device__ __forceinline__ void stage_band(double* dst, const double* ab, int c0, int nd, int lane) {
  for (int t = lane; t < SW_CH * VG_LDAB; t += 32) {
    int col = c0 + t / VG_LDAB;
    if (col >= 0 && col < nd)
      cp8(dst + t, ab + (size_t)col * VG_LDAB + (t % VG_LDAB));
    else
      dst[t] = 0.0;
  }
}

// Drift sweeps, one warp per task: up to 16 slots of one degree x (re, im).
// The degree's band columns stream through shared memory in chunks of 32 so
// that every load on the recurrence is a shared-memory load; the per-lane
// entering values (RHS in the L sweep, y in the U sweep) are staged the same
// way one chunk ahead.
__global__ void __launch_bounds__(128) k_drift_solve(DriftArgs A) {
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tix = blockIdx.x * SW_WARPS + warp;
  if (tix >= A.ntask) return;  // whole warp
  const int4 T = A.tasks[tix];
  const int l = T.x, k0 = T.y, nsl = T.z;
  const int sl = lane & 15, ri = lane >> 4;
  const bool valid = sl < nsl;
  const int k = k0 + (valid ? sl : 0);
  const int nr = A.nr, nd = A.nd;
  const size_t nk = A.nk;
  double* dUn = A.dUn + (size_t)ri * nr * nk + k;
  double* dVn = A.dVn + (size_t)ri * nr * nk + k;
  const bool active = valid && !(A.mnorm[k] <= skip_threshold(A));
  if (valid && !active) {  // negligible memory => zero drift
    for (int node = 0; node < nr; ++node) {
      dUn[node * nk] = 0.0;
      dVn[node * nk] = 0.0;
    }
    A.drift[(0 + ri) * nk + k] = 0.0;
    A.drift[(2 + ri) * nk + k] = 0.0;
    A.drift[(4 + ri) * nk + k] = 0.0;
  }
  if (!__any_sync(0xffffffffu, active)) return;
  double* sband = smem + (size_t)warp * SW_WARP;
  double* saux = sband + SW_BAND;
  const double* ab = A.ab + (size_t)(l - 2) * VG_LDAB * nd;
  const double* dc = A.dc + (size_t)(l - 2) * nd;
  const double* b = A.bh + ((size_t)ri * 2 * nr) * nk + k;  // b[(2 node + {0,1}) nk]
  double* y = A.ys + (size_t)ri * nd * nk + k;
  // entering RHS values of chunk c: U, V of nodes 8c+2 .. 8c+9, slot (2 kbi + uv)
  auto stage_b = [&](double* dst, int c) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      int node = 8 * c + (q >> 1) + 2;
      if (node < nr)
        cp8(dst + q * 32 + lane, b + (size_t)(2 * node + (q & 1)) * nk);
      else
        dst[q * 32 + lane] = 0.0;
    }
  };
  // ---- L sweep (P and L): window w0..w6 = x(j .. j+6) ----
  const int nchf = (nd - 1 + SW_CH - 1) / SW_CH;  // steps j = 0 .. nd-2
  stage_band(sband, ab, 0, nd, lane);
  stage_b(saux, 0);
  cp_commit();
  double w0 = b[0], w1 = b[nk], w2 = 0.0, w3 = 0.0, w4 = b[2 * nk], w5 = b[3 * nk], w6;
  for (int c = 0; c < nchf; ++c) {
    const int cur = c & 1;
    if (c + 1 < nchf) {
      stage_band(sband + (cur ^ 1) * SW_CH * VG_LDAB, ab, SW_CH * (c + 1), nd, lane);
      stage_b(saux + (cur ^ 1) * SW_CH * 32, c + 1);
      cp_commit();
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncwarp();
    const double* bandc = sband + cur * SW_CH * VG_LDAB;
    const double* bin = saux + cur * SW_CH * 32;
#pragma unroll 4
    for (int jj = 0; jj < SW_CH; ++jj) {
      const int j = SW_CH * c + jj, t = jj & 3;
      if (j > nd - 2) break;
      // dof j + 6 enters: F_{kb+1}, P_{kb+1} (no forcing), U_{kb+2}, V_{kb+2}
      w6 = (t < 2) ? 0.0 : bin[(2 * (jj >> 2) + (t - 2)) * 32 + lane];
      const double* col = bandc + jj * VG_LDAB;
      // row interchange j <-> j + jp: every lane of the warp solves with the
      // same degree's factor, so the branch is warp-uniform and a step
      // without interchange costs one compare
      const int jp = (int)col[20];
      if (jp != 0) {
        const double x0 = w0;
        switch (jp) {
          case 1: w0 = w1; w1 = x0; break;
          case 2: w0 = w2; w2 = x0; break;
          case 3: w0 = w3; w3 = x0; break;
          case 4: w0 = w4; w4 = x0; break;
          case 5: w0 = w5; w5 = x0; break;
          case 6: w0 = w6; w6 = x0; break;
          default: break;  // offsets lie in 0 .. kl = 6 by construction
        }
      }
      if (valid) y[(size_t)j * nk] = w0;
      w1 -= col[13] * w0;
      w2 -= col[14] * w0;
      w3 -= col[15] * w0;
      w4 -= col[16] * w0;
      w5 -= col[17] * w0;
      w6 -= col[18] * w0;
      w0 = w1;
      w1 = w2;
      w2 = w3;
      w3 = w4;
      w4 = w5;
      w5 = w6;
    }
    __syncwarp();  // the buffer just read is refilled by the next prefetch
  }
  if (valid) y[(size_t)(nd - 1) * nk] = w0;
  __threadfence_block();  // y stores before this lane's own cp.async reads of them
  // ---- U sweep: window v0..v12 = x(j-12 .. j), j descending ----
  // entering y(j - 13) of chunk c (steps j = J0-31 .. J0, J0 = nd-1-32c) at slot j - (J0 - 31)
  auto stage_y = [&](double* dst, int c) {
    const int jlo = nd - 1 - SW_CH * c - (SW_CH - 1);
#pragma unroll 4
    for (int q = 0; q < SW_CH; ++q) {
      int src = jlo + q - 13;
      if (src >= 0 && valid)
        cp8(dst + q * 32 + lane, y + (size_t)src * nk);
      else
        dst[q * 32 + lane] = 0.0;
    }
  };
  const int nchb = (nd + SW_CH - 1) / SW_CH;
  stage_band(sband, ab, nd - SW_CH, nd, lane);
  stage_y(saux, 0);
  cp_commit();
  double v0, v1, v2, v3, v4, v5, v6, v7, v8, v9, v10, v11, v12;
#define YAT(i) (((i) >= 0 && valid) ? y[(size_t)(i) * nk] : 0.0)
  v0 = YAT(nd - 13);
  v1 = YAT(nd - 12);
  v2 = YAT(nd - 11);
  v3 = YAT(nd - 10);
  v4 = YAT(nd - 9);
  v5 = YAT(nd - 8);
  v6 = YAT(nd - 7);
  v7 = YAT(nd - 6);
  v8 = YAT(nd - 5);
  v9 = YAT(nd - 4);
  v10 = YAT(nd - 3);
  v11 = YAT(nd - 2);
  v12 = YAT(nd - 1);
#undef YAT
  const int us = 4 * (nr - 1);
  for (int c = 0; c < nchb; ++c) {
    const int cur = c & 1, J0 = nd - 1 - SW_CH * c, jlo = J0 - (SW_CH - 1);
    if (c + 1 < nchb) {
      stage_band(sband + (cur ^ 1) * SW_CH * VG_LDAB, ab, jlo - SW_CH, nd, lane);
      stage_y(saux + (cur ^ 1) * SW_CH * 32, c + 1);
      cp_commit();
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncwarp();
    const double* bandc = sband + cur * SW_CH * VG_LDAB;
    const double* yin = saux + cur * SW_CH * 32;
#pragma unroll 4
    for (int jj = SW_CH - 1; jj >= 0; --jj) {
      const int j = jlo + jj;
      if (j < 0) break;
      const double* col = bandc + jj * VG_LDAB;
      const double xj = v12 * col[19];
      const int node = j >> 2, typ = j & 3;
      if (active) {
        if (typ == 0) dUn[node * nk] = __ldg(&dc[j]) * xj;
        if (typ == 1) dVn[node * nk] = __ldg(&dc[j]) * xj;
        if (j >= us) {
          if (typ == 0) A.drift[(0 + ri) * nk + k] = dc[j] * xj;
          if (typ == 2) A.drift[(2 + ri) * nk + k] = dc[j] * xj;
          if (typ == 1) A.drift[(4 + ri) * nk + k] = dc[j] * xj;
        }
      }
      v11 -= col[11] * xj;
      v10 -= col[10] * xj;
      v9 -= col[9] * xj;
      v8 -= col[8] * xj;
      v7 -= col[7] * xj;
      v6 -= col[6] * xj;
      v5 -= col[5] * xj;
      v4 -= col[4] * xj;
      v3 -= col[3] * xj;
      v2 -= col[2] * xj;
      v1 -= col[1] * xj;
      v0 -= col[0] * xj;
      v12 = v11;
      v11 = v10;
      v10 = v9;
      v9 = v8;
      v8 = v7;
      v7 = v6;
      v6 = v5;
      v5 = v4;
      v4 = v3;
      v3 = v2;
      v2 = v1;
      v1 = v0;
      v0 = yin[jj * 32 + lane];
    }
    __syncwarp();
  }
}

// Degree-1 drift (slots k = 0, 1; 4 right-hand sides): x = G1 b, then the
// CM-frame projection with the stored null mode (src/vilma_response.f90:770-779).
__global__ void __launch_bounds__(512) k_drift_deg1(DriftArgs A) {
  extern __shared__ double sh[];
  const int nr = A.nr, ncol = 2 * nr, nrow = 2 * nr + 1;
  const size_t nk = A.nk;
  double* f = sh;             // [4][ncol]
  double* x = sh + 4 * ncol;  // [4][nrow]
  __shared__ int s_act[2];
  __shared__ double s_c[4];
  const double thr = skip_threshold(A);
  if (threadIdx.x < 2) s_act[threadIdx.x] = !(A.mnorm[threadIdx.x] <= thr);
  __syncthreads();
  for (int t = threadIdx.x; t < 4 * ncol; t += blockDim.x) {
    int q = t / ncol, c = t % ncol, kk = q >> 1, ri = q & 1;
    f[t] = s_act[kk] ? A.bh[((size_t)ri * 2 * nr + c) * nk + kk] : 0.0;
  }
  __syncthreads();
  // x = G1 f: a warp per row, lanes over the columns (coalesced rows of G1),
  // the four right-hand sides at once
  {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = wid; r < nrow; r += nw) {
      const double* G = A.G1 + (size_t)r * ncol;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      for (int c = lane; c < ncol; c += 32) {
        const double g = __ldg(&G[c]);
        a0 += g * f[c];
        a1 += g * f[ncol + c];
        a2 += g * f[2 * ncol + c];
        a3 += g * f[3 * ncol + c];
      }
      for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        a3 += __shfl_xor_sync(0xffffffffu, a3, o);
      }
      if (lane == 0) {
        x[r] = a0;
        x[nrow + r] = a1;
        x[2 * nrow + r] = a2;
        x[3 * nrow + r] = a3;
      }
    }
  }
  __syncthreads();
  const int fs = 4 * (nr - 1) + 2;
  const double fa_n = A.null1[fs];
  const bool proj = A.deg1_cm && fa_n != 0.0;
  if (proj) {
    if (threadIdx.x < 4) s_c[threadIdx.x] = -x[threadIdx.x * nrow + 2 * nr] / fa_n;
    __syncthreads();
    for (int t = threadIdx.x; t < 4 * nrow; t += blockDim.x) {
      int q = t / nrow, r = t % nrow;
      int dof = (r < 2 * nr) ? 4 * (r >> 1) + (r & 1) : fs;
      x[t] = x[t] + s_c[q] * A.null1[dof];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < 4 * nr; t += blockDim.x) {
    int q = t / nr, node = t % nr, kk = q >> 1, ri = q & 1;
    bool act = s_act[kk];
    A.dUn[((size_t)ri * nr + node) * nk + kk] = act ? x[q * nrow + 2 * node] : 0.0;
    A.dVn[((size_t)ri * nr + node) * nk + kk] = act ? x[q * nrow + 2 * node + 1] : 0.0;
  }
  if (threadIdx.x < 4) {
    int q = threadIdx.x, kk = q >> 1, ri = q & 1;
    bool act = s_act[kk];
    A.drift[(0 + ri) * nk + kk] = act ? x[q * nrow + 2 * (nr - 1)] : 0.0;
    // N_1 == 0 in the "cf" frame (src/vilma_response.f90:779)
    A.drift[(2 + ri) * nk + kk] = (act && A.deg1_cm) ? x[q * nrow + 2 * nr] : 0.0;
    A.drift[(4 + ri) * nk + kk] = act ? x[q * nrow + 2 * (nr - 1) + 1] : 0.0;
  }
}

void launch_drift_on(vg_handle* h, int buf, double* dUn, double* dVn, cudaStream_t s0, cudaStream_t s1) {
  DriftArgs A;
  A.mem = h->d_mem[buf].p;
  A.mnorm = h->d_mnorm.p + (size_t)buf * h->nk;
  A.maxbits = h->d_maxbits.p + buf;
  A.skip_tol = h->p.skip_tol;
  A.r = h->d_r.p;
  A.sa = h->d_sa.p;
  A.sb = h->d_sb.p;
  A.sc = h->d_sc.p;
  A.nrmc = h->d_nrmc.p;
  A.ab = h->d_ab.p;
  A.dr = h->d_dr.p;
  A.dc = h->d_dc.p;
  A.rdiag = h->d_rdiag.p;
  A.ipiv = h->d_ipiv.p;
  A.kdeg = h->d_kdeg.p;
  A.bh = h->d_bh.p;
  A.ys = h->d_xs.p;
  A.dUn = dUn ? dUn : h->d_dUn.p;
  A.dVn = dVn ? dVn : h->d_dVn.p;
  A.drift = h->d_drift.p;
  A.ne = h->ne;
  A.nr = h->nr;
  A.nd = h->ndof;
  A.nk = h->nk;
  A.dr1 = h->d_dr1.p;
  A.null1 = h->d_null1.p;
  A.G1 = h->d_G1.p;
  A.deg1_cm = h->p.deg1_cm;
  A.K = h->d_Krhs.p;
  A.tasks = h->d_tasks.p;
  A.ntask = h->ntask;
  dim3 rgrid((h->nk + 31) / 32, (h->nr + 3) / 4, 2);
  k_drift_rhs<<<rgrid, dim3(32, 4), 0, s0>>>(A);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  const size_t sw_smem = (size_t)SW_WARPS * SW_WARP * sizeof(double);
  static std::atomic<bool> sw_attr{false};  // set once; concurrent handles may race to it
  if (!sw_attr) {
    VG_CUDA(cudaFuncSetAttribute(k_drift_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw_smem));
    sw_attr = true;
  }
  // degree 1 (slots 0, 1: reads their forcing, writes their drift) beside the
  // band sweeps (slots >= 2), on the handle's second stream
  VG_CUDA(cudaEventRecord(h->ev_fork, s0));
  VG_CUDA(cudaStreamWaitEvent(s1, h->ev_fork, 0));
  size_t shm = (size_t)(4 * 2 * h->nr + 4 * (2 * h->nr + 1)) * sizeof(double);
  k_drift_deg1<<<1, 512, shm, s1>>>(A);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  VG_CUDA(cudaEventRecord(h->ev_join, s1));
  k_drift_solve<<<(h->ntask + SW_WARPS - 1) / SW_WARPS, 32 * SW_WARPS, sw_smem, s0>>>(A);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  VG_CUDA(cudaStreamWaitEvent(s0, h->ev_join, 0));
}


void launch_drift(vg_handle* h, int buf, double* dUn, double* dVn, double* dWn) {
  PhaseScope ps(h, VG_PH_DRIFT);
  if (buf < 0) buf = h->cur;
  launch_drift_on(h, buf, dUn, dVn, h->stream, h->aux);
  if (h->tor_on) launch_drift_tor(h, buf, dWn);  // its own forcing, its own operator
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
                                                    h->d_gn.p, h->d_drift.p, d_sigma, d_u, d_n);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// Forward-Euler memory advance (src/vilma_viscoelastic.f90:577-584) of the
// spectrally advanced elements, out of place (cur -> nxt): one thread per
// (slot, element, re/im). Each thread also folds |new memory| of its element
// into the per-slot norm.
__global__ void __launch_bounds__(256) k_advance_1d(const double* __restrict__ mem, double* __restrict__ nxt, int ne,
                                                    int nr, int nk, double dt, const double* __restrict__ sigma,
                                                    const int* __restrict__ kdeg, const int* __restrict__ k2lm,
                                                    const double* __restrict__ Jrv, const double* __restrict__ xUn,
                                                    const double* __restrict__ xVn, const double* __restrict__ dUn,
                                                    const double* __restrict__ dVn, const double* __restrict__ mu,
                                                    const double* __restrict__ MkPerDt,
                                                    const char* __restrict__ active, double* __restrict__ mnorm,
                                                    int trap) {
  // 3-D elements (active[e] == 0) are advanced, and their maxima folded into
  // mnorm, by the pseudo-spectral pass's scatter
  const int k = blockIdx.x * 32 + threadIdx.x, e = blockIdx.y * 8 + threadIdx.y, ri = blockIdx.z;
  double amax = 0.0;
  if (k < nk && e < ne) {
    if (active[e]) {
      const int l = kdeg[k], lm = k2lm[k];
      const double s = sigma[2 * lm + ri];
      const double* xu = xUn + (size_t)l * nr;
      const double* xv = xVn + (size_t)l * nr;
      const double U0 = s * __ldg(&xu[e]) + dUn[((size_t)ri * nr + e) * nk + k];
      const double V0 = s * __ldg(&xv[e]) + dVn[((size_t)ri * nr + e) * nk + k];
      const double U1 = s * __ldg(&xu[e + 1]) + dUn[((size_t)ri * nr + e + 1) * nk + k];
      const double V1 = s * __ldg(&xv[e + 1]) + dVn[((size_t)ri * nr + e + 1) * nk + k];
      double a[4], b[4], c[4];
      strain_coeffs(U0, U1, V0, V1, Jrv[l], a, b, c);
      const double Me = MkPerDt[e] * dt;
      // forward Euler: (1 - M) tau - 2 mu M eps; trapezoidal with eps the mean of
      // eps_n and eps_{n+1}: [(1 - M/2) tau_n - 2 mu M eps] / (1 + M/2)
      // (src/vilma_viscoelastic.f90:556-569, 577-584)
      double om = 1.0 - Me, two_muM = 2.0 * mu[e] * Me;
      if (trap) {
        const double denom = 1.0 + 0.5 * Me;
        om = (1.0 - 0.5 * Me) / denom;
        two_muM = 2.0 * (mu[e] * Me / denom);
      }
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

// global max of the per-slot norms of one buffer
__global__ void k_norm_max(const double* __restrict__ mnorm, int nk, unsigned long long* __restrict__ maxbits) {
  __shared__ double red[1024];
  double v = 0.0;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) v = nanmax(v, mnorm[k]);
  v = block_max(v, red);
  if (threadIdx.x == 0) *maxbits = (unsigned long long)__double_as_longlong(v);
}

// Memory advance of one step, current buffer -> the other one: the 3-D
// elements through the pseudo-spectral pass (its scatter folds their maxima
// into the per-slot norms), the others spectrally (k_advance_1d). The two
// write disjoint elements of the next buffer and fold maxima (order-free)
// into the same norms, so without the toroidal channel the spectral advance
// runs on the handle's second stream beside the 3-D pass; with phase timers on
// they run one after the other so that each phase times its own kernels.
void advance_memory(vg_handle* h, const double* d_sigma, double dt, const double* dUn, const double* dVn, bool trap,
                    const double* dWn) {
  const int nxt = 1 - h->cur;
  double* mn = h->d_mnorm.p + (size_t)nxt * h->nk;
  VG_CUDA(cudaMemsetAsync(mn, 0, h->nk * sizeof(double), h->stream));
  const bool v3 = h->lat_visc && h->ne3d > 0;
  const bool side = v3 && !h->tor_on && !h->prof.on;
  auto spectral = [&](cudaStream_t s) {
    PhaseScope ps(h, VG_PH_ADVANCE_1D);
    dim3 grid((h->nk + 31) / 32, (h->ne + 7) / 8, 2);
    k_advance_1d<<<grid, dim3(32, 8), 0, s>>>(h->d_mem[h->cur].p, h->d_mem[nxt].p, h->ne, h->nr, h->nk, dt, d_sigma,
                                              h->d_kdeg.p, h->d_k2lm.p, h->d_Jr.p, h->d_xUn.p, h->d_xVn.p,
                                              dUn ? dUn : h->d_dUn.p, dVn ? dVn : h->d_dVn.p, h->d_mu.p,
                                              h->d_MkPerDt.p, h->d_active1d.p, mn, trap ? 1 : 0);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
    if (h->tor_on) launch_advance_1d_tor(h, dt, dWn, trap, mn);  // W is pure drift: no sigma x_Wn term
  };
  if (side) {
    VG_CUDA(cudaEventRecord(h->ev_fork, h->stream));
    VG_CUDA(cudaStreamWaitEvent(h->aux, h->ev_fork, 0));
    spectral(h->aux);
    VG_CUDA(cudaEventRecord(h->ev_join, h->aux));
    visc3d_advance(h, d_sigma, dt, dUn, dVn, trap, dWn);
    VG_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
  } else {
    if (v3) visc3d_advance(h, d_sigma, dt, dUn, dVn, trap, dWn);
    spectral(h->stream);
  }
  k_norm_max<<<1, 1024, 0, h->stream>>>(mn, h->nk, h->d_maxbits.p + nxt);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// per-slot norm and global max of one buffer (after vg_set_state / reset)
__global__ void k_mem_norm(const double* __restrict__ mem, int ne, int nk, double* __restrict__ mnorm) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  double amax = 0.0;
  for (int q = 0; q < 6 * ne * 4; ++q) amax = nanmax(amax, fabs(mem[(size_t)q * nk + k]));
  mnorm[k] = amax;
}

void compute_mem_norm(vg_handle* h, int buf) {
  double* mn = h->d_mnorm.p + (size_t)buf * h->nk;
  k_mem_norm<<<(h->nk + 255) / 256, 256, 0, h->stream>>>(h->d_mem[buf].p, h->ne, h->nk, mn);
  VG_CUDA(cudaGetLastError());
  if (h->tor_on) mem_norm_tor(h, buf, mn);
  k_norm_max<<<1, 1024, 0, h->stream>>>(mn, h->nk, h->d_maxbits.p + buf);
  VG_CUDA(cudaGetLastError());
}

double read_mem_norm(vg_handle* h, int buf) {
  unsigned long long bits[3] = {0, 0, 0};
  VG_CUDA(cudaMemcpyAsync(bits, h->d_maxbits.p, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
  VG_CUDA(cudaStreamSynchronize(h->stream));
  if (bits[2] != 0) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "tensor-core stage wait timed out (status bits 0x%llx); results are invalid",
                  bits[2]);
    throw Error(msg);
  }
  double v;
  std::memcpy(&v, &bits[buf], sizeof(v));
  return v;
}

}  // namespace vg
