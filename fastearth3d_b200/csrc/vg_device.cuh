// Device helpers shared by the kernels of several translation units.
#pragma once
#include <cuda_runtime.h>

namespace vg {

// index of memory element (s, ri, e, lam, k) in one state buffer
__device__ __forceinline__ size_t mem_idx(int s, int ri, int e, int lam, int k, int ne, int nk) {
  return ((size_t)((s * 2 + ri) * ne + e) * 4 + lam) * nk + k;
}

// index of toroidal memory element (s, ri, e, lam, k), lam 0 = lambda 3, 1 = lambda 4
__device__ __forceinline__ size_t tmem_idx(int s, int ri, int e, int lam, int k, int ne, int nk) {
  return ((size_t)((s * 2 + ri) * ne + e) * 2 + lam) * nk + k;
}

// src/vilma_viscoelastic.f90:373-390 strain_coeffs_tor: element strain (a, b, c)
// for lam = 3, 4 from nodal W; Z4 has no harmonic below degree 2.
__device__ __forceinline__ void strain_coeffs_tor(double w1, double w2, double Jr, double a[2], double b[2],
                                                  double c[2]) {
  a[0] = -w1 + w2;
  b[0] = -w1;
  c[0] = -w2;
  a[1] = 0.0;
  b[1] = w1;
  c[1] = w2;
  if (Jr <= 2.0) {
    b[1] = 0.0;
    c[1] = 0.0;
  }
}

// max that propagates NaN, so a non-finite state never hides from the guard
__device__ __forceinline__ double nanmax(double a, double b) { return (a != a || b != b) ? (a + b) : fmax(a, b); }

__device__ __forceinline__ void atomic_max_bits(unsigned long long* dst, double v) {
  // non-negative doubles (and NaN, whose bits sort above +inf) order like their bit patterns
  atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

// src/vilma_viscoelastic.f90:329-359 strain_coeffs: element strain (a, b, c) for
// lam = 1, 2, 5, 6 from nodal U, V; Z6 has no harmonic below degree 2.
__device__ __forceinline__ void strain_coeffs(double u1, double u2, double v1, double v2, double Jr, double a[4],
                                              double b[4], double c[4]) {
  a[0] = -u1 + u2;
  b[0] = 0.0;
  c[0] = 0.0;
  a[1] = -v1 + v2;
  b[1] = u1 - v1;
  c[1] = u2 - v2;
  a[2] = 0.0;
  b[2] = -u1 / Jr + 0.5 * v1;
  c[2] = -u2 / Jr + 0.5 * v2;
  a[3] = 0.0;
  b[3] = 0.5 * v1;
  c[3] = 0.5 * v2;
  if (Jr <= 2.0) {
    b[3] = 0.0;
    c[3] = 0.0;
  }
}

// Degree-1 bordered system, dense band storage with kl = ku = nd, solved for
// up to 4 right-hand sides held in shared memory (xsh[nrhs][ns]); dgbtrs order,
// CTA-parallel inner loops. Column-major band storage ab[(col - 1) * ldab + (row - 1)].
__device__ __forceinline__ void deg1_solve_cta(const double* __restrict__ ab, int ldab, int ns, int kl, int kv,
                                               const int* __restrict__ ipiv, double* xsh, int nrhs) {
  for (int j = 1; j <= ns - 1; ++j) {
    int lm = min(kl, ns - j);
    int l = ipiv[j - 1] + 1;
    if ((int)threadIdx.x < nrhs && l != j) {
      double* x = xsh + threadIdx.x * ns;
      double t = x[l - 1];
      x[l - 1] = x[j - 1];
      x[j - 1] = t;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < lm * nrhs; t += blockDim.x) {
      int i = 1 + t / nrhs, rr = t % nrhs;
      double* x = xsh + rr * ns;
      x[j + i - 1] -= ab[(size_t)(j - 1) * ldab + (kv + i)] * x[j - 1];
    }
    __syncthreads();
  }
  for (int j = ns; j >= 1; --j) {
    if ((int)threadIdx.x < nrhs) {
      double* x = xsh + threadIdx.x * ns;
      x[j - 1] = x[j - 1] / ab[(size_t)(j - 1) * ldab + kv];
    }
    __syncthreads();
    int lm = min(kv, j - 1);
    for (int t = threadIdx.x; t < lm * nrhs; t += blockDim.x) {
      int i = 1 + t / nrhs, rr = t % nrhs;
      double* x = xsh + rr * ns;
      x[j - i - 1] -= ab[(size_t)(j - 1) * ldab + (kv - i)] * x[j - 1];
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------------
// Longitude transforms of one latitude row, CTA-cooperative, twiddles from
// tables cos/sin(2 pi t / nphi). The real-field convention of the Gauss-grid
// transforms (src/vilma_sht.f90:11-15): f_i = Re G_0 + 2 Re sum_{m>0} G_m e^{i m phi_i},
// and F_m = (2 pi / nphi) sum_i f_i e^{-i m phi_i}.

// row (smem, nphi) -> F[m] = (re, im) at F + 2*m*stride, m < M
__device__ __forceinline__ void row_fourier_analysis(const double* row, int nphi, int M, const double* __restrict__ cs,
                                                     const double* __restrict__ sn, double* F, size_t stride) {
  const double sc = 2.0 * 3.14159265358979323846 / (double)nphi;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    double re = 0.0, im = 0.0;
    int t = 0;
    for (int i = 0; i < nphi; ++i) {
      double f = row[i];
      re += f * __ldg(&cs[t]);
      im -= f * __ldg(&sn[t]);
      t += m;
      if (t >= nphi) t -= nphi;
    }
    F[2 * (size_t)m * stride] = re * sc;
    F[2 * (size_t)m * stride + 1] = im * sc;
  }
}

// G (smem, M complex interleaved) -> f_i for i < nphi (called per thread for its i)
__device__ __forceinline__ double row_fourier_synth_at(const double* G, int M, int i, int nphi,
                                                       const double* __restrict__ cs, const double* __restrict__ sn) {
  double acc = 0.0;
  int t = i;
  for (int m = 1; m < M; ++m) {
    acc += G[2 * m] * __ldg(&cs[t]) - G[2 * m + 1] * __ldg(&sn[t]);
    t += i;
    if (t >= nphi) t -= nphi;
  }
  return G[0] + 2.0 * acc;
}

// CTA reductions (fixed order: deterministic for a fixed block size)
__device__ __forceinline__ double block_sum(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}
// The same reductions through warp shuffles (two block barriers instead of
// one per tree level); blockDim a multiple of 32, every thread gets the
// result; the warp partials are added in warp order.
__device__ __forceinline__ double block_sum_w(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int nw = blockDim.x >> 5;
  __syncthreads();  // the previous call's readers are done with red
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = red[0];
  for (int w = 1; w < nw; ++w) r += red[w];
  return r;
}
__device__ __forceinline__ double block_max_w(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = red[0];
  for (int w = 1; w < nw; ++w) r = nanmax(r, red[w]);
  return r;
}
__device__ __forceinline__ double block_max(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] = nanmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}

// dgbtrs-style solve with the factor of band_factor_dev (column-major band
// storage, leading dimension ldab), right-hand side with element stride st
__host__ __device__ __forceinline__ void band_solve_strided(const double* __restrict__ ab, int ldab, int n, int kl, int kv,
                                                   const int* __restrict__ ipiv, double* x, size_t st) {
#define AB(row1, col1) ab[(size_t)((col1)-1) * ldab + ((row1)-1)]
  for (int j = 1; j <= n - 1; ++j) {
    int lm = min(kl, n - j);
    int l = ipiv[j - 1] + 1;
    if (l != j) {
      double t = x[(size_t)(l - 1) * st];
      x[(size_t)(l - 1) * st] = x[(size_t)(j - 1) * st];
      x[(size_t)(j - 1) * st] = t;
    }
    double t = x[(size_t)(j - 1) * st];
    for (int i = 1; i <= lm; ++i) x[(size_t)(j + i - 1) * st] -= AB(kv + 1 + i, j) * t;
  }
  for (int j = n; j >= 1; --j) {
    double xj = x[(size_t)(j - 1) * st] / AB(kv + 1, j);
    x[(size_t)(j - 1) * st] = xj;
    int lm = min(kv, j - 1);
    for (int i = 1; i <= lm; ++i) x[(size_t)(j - i - 1) * st] -= AB(kv + 1 - i, j) * xj;
  }
#undef AB
}

// The same solve as band_solve_strided (unit stride), operation for operation
// and in the same order, for compile-time bandwidths: the sweep's active
// window of the right-hand side is held in registers (forward: x[k .. k + KL],
// the row interchange a select within it; backward: x[k - KV .. k]), so that
// each element is read once before its sweep and written once after it
// instead of going through memory at every update, and the next step's
// operands (pivot, band column, the entering element) are loaded one step
// ahead, so their latency overlaps the current step's arithmetic. For one
// thread per right-hand side, whose sweeps are otherwise a chain of dependent
// memory round trips.
template <int KL, int KV>
__host__ __device__ __forceinline__ void band_solve_window(const double* __restrict__ ab, int ldab, int n,
                                                  const int* __restrict__ ipiv, double* __restrict__ x) {
  double w[KL + 1];  // w[i] = x[k + i]
#pragma unroll
  for (int i = 0; i <= KL; ++i) w[i] = i < n ? x[i] : 0.0;
  // operands of step k: the interchange offset, AB(KV + 1 + i, k + 1) for
  // i = 1 .. KL, and x[k + 1 + KL], the element that enters after the step
  int ip = 0;
  double cn[KL + 1];
  double xn = (KL + 1 < n) ? x[KL + 1] : 0.0;
  if (n > 1) {
    ip = ipiv[0];
#pragma unroll
    for (int i = 1; i <= KL; ++i) cn[i] = ab[KV + i];
  }
  for (int k = 0; k < n - 1; ++k) {
    const int d = ip - k;  // the interchange partner row k + d, 0 <= d <= KL
    double cc[KL + 1];
#pragma unroll
    for (int i = 1; i <= KL; ++i) cc[i] = cn[i];
    const double xe = xn;
    if (k + 1 < n - 1) {
      ip = ipiv[k + 1];
      const double* col = ab + (size_t)(k + 1) * ldab + KV;
#pragma unroll
      for (int i = 1; i <= KL; ++i) cn[i] = col[i];
    }
    xn = (k + 2 + KL < n) ? x[k + 2 + KL] : 0.0;
#pragma unroll
    for (int i = 1; i <= KL; ++i)
      if (d == i) {
        const double s = w[0];
        w[0] = w[i];
        w[i] = s;
      }
    const double t = w[0];
    const int lm = min(KL, n - 1 - k);
#pragma unroll
    for (int i = 1; i <= KL; ++i)
      if (i <= lm) w[i] -= cc[i] * t;
    x[k] = w[0];
#pragma unroll
    for (int i = 0; i < KL; ++i) w[i] = w[i + 1];
    w[KL] = xe;
  }
  if (n >= 1) x[n - 1] = w[0];
  double v[KV + 1];  // v[i] = x[k - i]
#pragma unroll
  for (int i = 0; i <= KV; ++i) v[i] = (n - 1 - i >= 0) ? x[n - 1 - i] : 0.0;
  // operands of step k: AB(KV + 1 - i, k + 1) for i = 0 .. KV and x[k - 1 - KV]
  double bn[KV + 1];
  double yn = (n - 2 - KV >= 0) ? x[n - 2 - KV] : 0.0;
  if (n >= 1) {
    const double* col = ab + (size_t)(n - 1) * ldab + KV;
#pragma unroll
    for (int i = 0; i <= KV; ++i) bn[i] = col[-i];
  }
  for (int k = n - 1; k >= 0; --k) {
    double bc[KV + 1];
#pragma unroll
    for (int i = 0; i <= KV; ++i) bc[i] = bn[i];
    const double ye = yn;
    if (k >= 1) {
      const double* col = ab + (size_t)(k - 1) * ldab + KV;
#pragma unroll
      for (int i = 0; i <= KV; ++i) bn[i] = col[-i];
    }
    yn = (k - 2 - KV >= 0) ? x[k - 2 - KV] : 0.0;
    const double xk = v[0] / bc[0];
    x[k] = xk;
    const int lm = min(KV, k);
#pragma unroll
    for (int i = 1; i <= KV; ++i)
      if (i <= lm) v[i] -= bc[i] * xk;
#pragma unroll
    for (int i = 0; i < KV; ++i) v[i] = v[i + 1];
    v[KV] = ye;
  }
}

}  // namespace vg
