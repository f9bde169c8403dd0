// The trapezoidal (Crank-Nicolson) memory scheme, scheme = "trap"
// (src/vilma_viscoelastic.f90:556-569; src/vilma_response.f90:1321-1663;
// src/vilma_sle.f90:218-365; src/vilma_timestep.f90:229-307).
//
//   tau_{n+1} = [(1 - M/2) tau_n - mu M (eps_n + eps_{n+1})] / (1 + M/2)
//
// is the forward-Euler update with the strain replaced by the mean of the
// step's two ends and the factors (1 - M, 2 mu M) by ((1 - M/2) / (1 + M/2),
// 2 mu M / (1 + M/2)); strain and the 3-D synthesis are linear, so the
// forward-Euler kernels run it on the averaged load sigma and drift (dUn +
// edUn) / 2 (1-D elements: k_advance_1d, 3-D elements: the pseudo-spectral
// advance with the pointwise factor M / (1 + M/2)). Each endpoint pass
// advances from tau_n (the current buffer) into the other buffer, re-solves
// the endpoint drift edUn from it, and measures the change of the surface
// drift dUa against the previous pass; the sea-level solve repeats passes
// until that change is below couple_tol (at least two passes). The
// step-doubling controller (one coarse step against two half steps, error
// ||tau_fine - tau_coarse||_inf / 3 against atol + rtol ||tau_fine||_inf)
// keeps its snapshots in two extra state buffers.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

// sigma and nodal drift averaged over the step's two ends (sigma_n = sigma_{n+1}
// before the start-of-step load is known, src/vilma_response.f90:1553-1558)
__global__ void k_trap_avg(int n2lm, int nd2, const double* __restrict__ sig_n, const double* __restrict__ sig1,
                           int primed, double* __restrict__ sig_avg, const double* __restrict__ dUn,
                           const double* __restrict__ edUn, double* __restrict__ dUa, const double* __restrict__ dVn,
                           const double* __restrict__ edVn, double* __restrict__ dVa) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n2lm) sig_avg[t] = primed ? 0.5 * (sig_n[t] + sig1[t]) : sig1[t];
  if (t < nd2) {
    dUa[t] = 0.5 * (dUn[t] + edUn[t]);
    dVa[t] = 0.5 * (dVn[t] + edVn[t]);
  }
}

// maxima of non-negative values (NaN propagates: its bits order above inf)
__device__ __forceinline__ void warp_max_to(unsigned long long* dst, double v) {
  for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

// coarse / fine error of the step-doubling estimate (response_coarse_fine_error,
// src/vilma_response.f90:1760-1781): red[0] = max |f - c|, red[1] = max |f|
__global__ void k_trap_cf(size_t n, const double* __restrict__ f, const double* __restrict__ c,
                          unsigned long long* __restrict__ red) {
  double e = 0.0, t = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    e = nanmax(e, fabs(f[i] - c[i]));
    t = nanmax(t, fabs(f[i]));
  }
  warp_max_to(red, e);
  warp_max_to(red + 1, t);
}

// change of the surface drift since the previous pass (drift_change,
// src/vilma_response.f90:1499-1512): red[2] = max |dUa - prev|, red[3] = max |dUa|
__global__ void k_trap_dchange(int nk, const double* __restrict__ drift, const double* __restrict__ prev,
                               unsigned long long* __restrict__ red) {
  double c = 0.0, s = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x) {
    const double re = drift[k], im = drift[nk + k];
    c = nanmax(c, hypot(re - prev[k], im - prev[nk + k]));
    s = nanmax(s, hypot(re, im));
  }
  warp_max_to(red + 2, c);
  warp_max_to(red + 3, s);
}

void trap_setup(vg_handle* h) {
  const size_t nd2 = (size_t)2 * h->nr * h->nk, n2 = (size_t)2 * h->grid.nlm, S = h->d_mem[0].n;
  for (DArr<double>* a : {&h->d_edUn, &h->d_edVn, &h->d_dU_avg, &h->d_dV_avg}) a->alloc(nd2);
  for (DArr<double>* a : {&h->d_sigma_n, &h->d_sigma_next, &h->d_sigma_avg, &h->d_sigma_n_s}) a->alloc(n2);
  h->d_dUa_prev.alloc((size_t)2 * h->nk);
  h->d_mem_s.alloc(S);
  h->d_mem_c.alloc(S);
  h->d_trap_red.alloc(4);
}

static void d2d(double* dst, const double* src, size_t n, cudaStream_t s) {
  VG_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

// ve_response_prepare_endpoint (src/vilma_response.f90:1598-1616): tau_n stays
// in the current buffer; the endpoint drift starts from the entering drift
void trap_prepare(vg_handle* h) {
  const size_t nd2 = (size_t)2 * h->nr * h->nk;
  d2d(h->d_edUn.p, h->d_dUn.p, nd2, h->stream);
  d2d(h->d_edVn.p, h->d_dVn.p, nd2, h->stream);
  d2d(h->d_dUa_prev.p, h->d_drift.p, (size_t)2 * h->nk, h->stream);  // keep_drift
  if (h->tor_on) {
    d2d(h->d_edWn.p, h->d_dWn.p, nd2, h->stream);
    d2d(h->d_dWa_prev.p, h->d_dWa.p, (size_t)2 * h->nk, h->stream);
  }
  h->couple_pass = 0;
}

// mean of the entering and endpoint W drift
__global__ void k_trap_avg_w(int n, const double* __restrict__ dWn, const double* __restrict__ edWn,
                             double* __restrict__ dWavg) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dWavg[t] = 0.5 * (dWn[t] + edWn[t]);
}

// ve_response_advance_endpoint (src/vilma_response.f90:1618-1646) with the
// converged load in d_sigma; returns couple_done
bool trap_endpoint_pass(vg_handle* h, double dt) {
  cudaStream_t s = h->stream;
  const int n2lm = 2 * h->grid.nlm, nd2 = 2 * h->nr * h->nk;
  const int n = std::max(n2lm, nd2);
  k_trap_avg<<<(n + 255) / 256, 256, 0, s>>>(n2lm, nd2, h->d_sigma_n.p, h->d_sigma.p, h->sigma_primed ? 1 : 0,
                                            h->d_sigma_avg.p, h->d_dUn.p, h->d_edUn.p, h->d_dU_avg.p, h->d_dVn.p,
                                            h->d_edVn.p, h->d_dV_avg.p);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  if (h->tor_on) {
    k_trap_avg_w<<<(nd2 + 255) / 256, 256, 0, s>>>(nd2, h->d_dWn.p, h->d_edWn.p, h->d_dW_avg.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  const double* dWavg = h->tor_on ? h->d_dW_avg.p : nullptr;
  advance_memory(h, h->d_sigma_avg.p, dt, h->d_dU_avg.p, h->d_dV_avg.p, true, dWavg);
  d2d(h->d_sigma_next.p, h->d_sigma.p, (size_t)n2lm, s);
  launch_drift(h, 1 - h->cur, h->d_edUn.p, h->d_edVn.p, h->tor_on ? h->d_edWn.p : nullptr);  // solve_endpoint_drift
  ++h->couple_pass;
  VG_CUDA(cudaMemsetAsync(h->d_trap_red.p + 2, 0, 2 * sizeof(unsigned long long), s));
  k_trap_dchange<<<(h->nk + 255) / 256, 256, 0, s>>>(h->nk, h->d_drift.p, h->d_dUa_prev.p, h->d_trap_red.p);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  if (h->tor_on) {  // W(a) joins U(a) in the convergence signal (drift_change, :1499-1512)
    k_trap_dchange<<<(h->nk + 255) / 256, 256, 0, s>>>(h->nk, h->d_dWa.p, h->d_dWa_prev.p, h->d_trap_red.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  unsigned long long bits[2];
  VG_CUDA(cudaMemcpyAsync(bits, h->d_trap_red.p + 2, sizeof(bits), cudaMemcpyDeviceToHost, s));
  d2d(h->d_dUa_prev.p, h->d_drift.p, (size_t)2 * h->nk, s);  // keep_drift
  if (h->tor_on) d2d(h->d_dWa_prev.p, h->d_dWa.p, (size_t)2 * h->nk, s);
  VG_CUDA(cudaStreamSynchronize(s));
  double cnorm, snorm;
  std::memcpy(&cnorm, &bits[0], sizeof(double));
  std::memcpy(&snorm, &bits[1], sizeof(double));
  return h->couple_pass >= 2 && cnorm <= h->p.couple_tol * std::max(snorm, TINY);
}

// ve_response_finalize_step (src/vilma_response.f90:1653-1663): the advanced
// buffer becomes the memory, sigma_{n+1} the next step's sigma_n
void trap_finalize(vg_handle* h, double dt) {
  d2d(h->d_sigma_n.p, h->d_sigma_next.p, (size_t)2 * h->grid.nlm, h->stream);
  h->sigma_primed = true;
  h->cur = 1 - h->cur;
  h->time_s += dt;
  h->couple_iters_last = h->couple_pass;
}

// response_save_state / response_restore_state / response_stash_coarse
// (src/vilma_response.f90:1695-1758): memory, time, sigma_n
void trap_save(vg_handle* h) {
  d2d(h->d_mem_s.p, h->d_mem[h->cur].p, h->d_mem_s.n, h->stream);
  if (h->tor_on) d2d(h->d_tmem_s.p, h->d_tmem[h->cur].p, h->d_tmem_s.n, h->stream);
  d2d(h->d_sigma_n_s.p, h->d_sigma_n.p, (size_t)2 * h->grid.nlm, h->stream);
  h->time_s_saved = h->time_s;
  h->sigma_primed_s = h->sigma_primed;
}
void trap_restore(vg_handle* h) {
  d2d(h->d_mem[h->cur].p, h->d_mem_s.p, h->d_mem_s.n, h->stream);
  if (h->tor_on) d2d(h->d_tmem[h->cur].p, h->d_tmem_s.p, h->d_tmem_s.n, h->stream);
  d2d(h->d_sigma_n.p, h->d_sigma_n_s.p, (size_t)2 * h->grid.nlm, h->stream);
  h->time_s = h->time_s_saved;
  h->sigma_primed = h->sigma_primed_s;
  compute_mem_norm(h, h->cur);  // the drift's skip gate reads the buffer's norms
}
void trap_stash_coarse(vg_handle* h) {
  d2d(h->d_mem_c.p, h->d_mem[h->cur].p, h->d_mem_c.n, h->stream);
  if (h->tor_on) d2d(h->d_tmem_c.p, h->d_tmem[h->cur].p, h->d_tmem_c.n, h->stream);
}

void trap_coarse_fine_error(vg_handle* h, double& err_inf, double& tau_inf) {
  cudaStream_t s = h->stream;
  VG_CUDA(cudaMemsetAsync(h->d_trap_red.p, 0, 2 * sizeof(unsigned long long), s));
  k_trap_cf<<<1184, 256, 0, s>>>(h->d_mem_c.n, h->d_mem[h->cur].p, h->d_mem_c.p, h->d_trap_red.p);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  if (h->tor_on) {
    k_trap_cf<<<1184, 256, 0, s>>>(h->d_tmem_c.n, h->d_tmem[h->cur].p, h->d_tmem_c.p, h->d_trap_red.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  unsigned long long bits[2];
  VG_CUDA(cudaMemcpyAsync(bits, h->d_trap_red.p, sizeof(bits), cudaMemcpyDeviceToHost, s));
  VG_CUDA(cudaStreamSynchronize(s));
  std::memcpy(&err_inf, &bits[0], sizeof(double));
  std::memcpy(&tau_inf, &bits[1], sizeof(double));
}

// response_prime_sigma: the start-of-step load from a report-only solve
void trap_prime(vg_handle* h) {
  d2d(h->d_sigma_n.p, h->d_sigma.p, (size_t)2 * h->grid.nlm, h->stream);
  h->sigma_primed = true;
}

}  // namespace vg
