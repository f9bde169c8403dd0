// C-ABI entry points (include/vilma_gpu.h). Every call returns an int status;
// failures are caught here and their message is kept for vg_last_error. No
// exit or abort inside the library.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "vg_internal.cuh"

using vg::DArr;
using vg::Error;

static thread_local std::string g_last_error;

template <class F>
static int guarded(vg_handle* h, F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& ex) {
    if (h)
      h->err = ex.what();
    else
      g_last_error = ex.what();
    return 1;
  }
}

static void need(vg_handle* h, bool cond, const char* msg) {
  (void)h;
  if (!cond) throw Error(msg);
}

namespace vg {
void raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<const void*, size_t> limit;
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = limit[kernel];
  if (bytes <= cur) return;
  VG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
}

PhaseScope::PhaseScope(vg_handle* hh, int p) : h(hh), ph(p) {
  if (!h->prof.on) return;
  cudaEvent_t e;
  VG_CUDA(cudaEventCreate(&e));
  VG_CUDA(cudaEventRecord(e, h->stream));
  h->prof.ev[ph].push_back(e);
}
PhaseScope::~PhaseScope() {
  if (!h->prof.on) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, h->stream);
  h->prof.ev[ph].push_back(e);
  h->prof.calls[ph]++;
}
void prof_collect(vg_handle* h) {
  VG_CUDA(cudaStreamSynchronize(h->stream));
  for (int ph = 0; ph < VG_NPHASE; ++ph) {
    auto& v = h->prof.ev[ph];
    for (size_t i = 0; i + 1 < v.size(); i += 2) {
      float ms = 0.f;
      VG_CUDA(cudaEventElapsedTime(&ms, v[i], v[i + 1]));
      h->prof.ms[ph] += ms;
    }
    for (cudaEvent_t e : v) cudaEventDestroy(e);
    v.clear();
  }
}
}  // namespace vg

extern "C" {

int vg_params_default(vg_params* p) {
  if (!p) return 1;
  std::memset(p, 0, sizeof(*p));
  const double km = 1e3;
  p->lmax = 16;
  p->nlat = 17;
  p->nphi = 34;
  p->n_layer = 4;
  p->r_earth = 6371.0 * km;
  const double rb[4] = {6301.0 * km, 5701.0 * km, 3480.0 * km, 0.0};
  const double rt[4] = {6371.0 * km, 6301.0 * km, 5701.0 * km, 3480.0 * km};
  const double rho[4] = {3300.0, 3450.0, 4900.0, 10900.0};
  const double mu[4] = {0.7e11, 0.9e11, 2.0e11, 0.0};
  const double eta[4] = {1e300, 5e20, 2e21, 0.0};
  const int rh[4] = {VG_RHEOL_ELASTIC, VG_RHEOL_MAXWELL, VG_RHEOL_MAXWELL, VG_RHEOL_FLUID};
  for (int i = 0; i < 4; ++i) {
    p->r_bot[i] = rb[i];
    p->r_top[i] = rt[i];
    p->rho[i] = rho[i];
    p->mu[i] = mu[i];
    p->eta[i] = eta[i];
    p->rheology[i] = rh[i];
  }
  p->scheme = VG_SCHEME_FE;
  p->deg1_cm = 1;
  p->skip_tol = 1e-4;
  p->visc3d_tol = 1e-3;
  p->dt_init = 0.0;
  p->cfl = 1.0;
  p->guard_growth = 1e3;
  p->dt_min = 0.0;
  p->dt_max = 1.7976931348623157e308;
  p->sle_n_outer = 3;
  p->sle_n_inner = 20;
  p->sle_tol = 1e-7;
  p->sle_fixed_ocean = 0;
  p->sle_subgrid = 1;
  p->sle_warm_start = 1;
  p->rotation = 0;
  p->visc3d_precision = VG_VISC3D_FP64;
  p->rtol = 1e-4;
  p->atol = 1e-3;
  p->safety = 0.9;
  p->grow_max = 5.0;
  p->shrink_min = 0.2;
  p->sle_max_mem_iter = 20;
  p->couple_tol = 1e-6;
  return 0;
}

int vg_create(const vg_params* p, vg_handle** out) {
  if (!p || !out) {
    g_last_error = "vg_create: null argument";
    return 1;
  }
  *out = nullptr;
  vg_handle* h = new vg_handle();
  h->p = *p;
  int rc = guarded(nullptr, [&] {
    int ndev = 0;
    VG_CUDA(cudaGetDevice(&h->device));
    VG_CUDA(cudaGetDeviceCount(&ndev));
    VG_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    VG_CUDA(cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking));
    VG_CUDA(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    VG_CUDA(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    VG_CUDA(cudaStreamCreateWithFlags(&h->aux2, cudaStreamNonBlocking));
    VG_CUDA(cudaEventCreateWithFlags(&h->ev_dfork, cudaEventDisableTiming));
    VG_CUDA(cudaEventCreateWithFlags(&h->ev_djoin, cudaEventDisableTiming));
    vg::setup_handle(h);
    if (h->p.rotation) vg::rotation_setup(h);
    if (h->p.scheme == VG_SCHEME_TRAP) vg::trap_setup(h);
    vg::compute_mem_norm(h, 0);
    h->mem_norm = vg::read_mem_norm(h, 0);
  });
  if (rc) {
    vg_destroy(h);
    return rc;
  }
  *out = h;
  return 0;
}

int vg_destroy(vg_handle* h) {
  if (!h) return 0;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->aux) cudaStreamSynchronize(h->aux);
  if (h->aux2) cudaStreamSynchronize(h->aux2);
  if (h->h_sc) cudaFreeHost(h->h_sc);
  cudaStream_t s = h->stream, a = h->aux, a2 = h->aux2;
  cudaEvent_t ev[4] = {h->ev_fork, h->ev_join, h->ev_dfork, h->ev_djoin};
  delete h;
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
  if (a2) cudaStreamDestroy(a2);
  if (a) cudaStreamDestroy(a);
  if (s) cudaStreamDestroy(s);
  return 0;
}

const char* vg_last_error(const vg_handle* h) { return h ? h->err.c_str() : g_last_error.c_str(); }

int vg_set_reference(vg_handle* h, const double* z_bed_eq, const double* h_ice_eq, const double* h_ice_init) {
  return guarded(h, [&] {
    need(h, z_bed_eq && h_ice_eq, "vg_set_reference: z_bed_eq and h_ice_eq are required");
    const int ng = h->grid.ng;
    cudaStream_t s = h->stream;
    h->d_z_bed_eq.upload(z_bed_eq, ng, s);
    h->d_h_ice_eq.upload(h_ice_eq, ng, s);
    h->d_h_ice.upload(h_ice_init ? h_ice_init : h_ice_eq, ng, s);
    VG_CUDA(cudaMemsetAsync(h->d_rsl.p, 0, ng * sizeof(double), s));
    VG_CUDA(cudaMemcpyAsync(h->d_zbed.p, z_bed_eq, ng * sizeof(double), cudaMemcpyHostToDevice, s));
    // C0 = ocean_function(z_bed_eq, h_ice_eq); C = C0 (src/vilma_coupling.f90:211-212)
    VG_CUDA(cudaMemsetAsync(h->d_tmp.p, 0, ng * sizeof(double), s));
    std::vector<double> c0(ng);
    for (int i = 0; i < ng; ++i)
      c0[i] = (z_bed_eq[i] < 0.0 && vg::RHO_ICE * h_ice_eq[i] < -vg::RHO_WATER * z_bed_eq[i]) ? 1.0 : 0.0;
    h->d_C0.upload(c0.data(), ng, s);
    h->d_C.upload(c0.data(), ng, s);
    VG_CUDA(cudaStreamSynchronize(s));
    h->have_reference = true;
  });
}

int vg_enable_visc3d(vg_handle* h, const double* pert) {
  return guarded(h, [&] {
    need(h, pert != nullptr, "vg_enable_visc3d: pert is required");
    vg::visc3d_enable(h, pert);
  });
}

int vg_advance(vg_handle* h, const double* ice0, const double* ice1, double t0_yr, double t1_yr, const double* s_rot,
               double* rsl, double* C, double* sigma_lm) {
  return guarded(h, [&] {
    need(h, h->have_reference, "vg_advance: call vg_set_reference first (solid_earth_init)");
    need(h, ice0 != nullptr && ice1 != nullptr, "vg_advance: ice0 and ice1 are required");
    need(h, t1_yr >= t0_yr, "vg_advance: t1 must not precede t0");
    need(h, !(s_rot && h->rot_on), "vg_advance: with rotation = 1 the library integrates s_rot itself");
    const size_t ng = (size_t)h->grid.ng;
    cudaStream_t s = h->stream;
    h->d_h_ice.upload(ice0, ng, s);  // the entering (carried) ice
    h->d_ice1.upload(ice1, ng, s);
    h->time_yr = t0_yr;
    h->time_s = t0_yr * vg::SEC_PER_YEAR;
    if (s_rot) {
      if (h->d_srot.n != ng) h->d_srot.alloc(ng);
      h->d_srot.upload(s_rot, ng, s);
    }
    h->srot_ext = s_rot != nullptr;
    try {
      vg::update_dev(h, h->d_ice1.p, t1_yr - t0_yr);
    } catch (...) {
      h->srot_ext = false;
      throw;
    }
    h->srot_ext = false;
    if (rsl) h->d_rsl.download(rsl, ng, s);
    if (C) h->d_C.download(C, ng, s);
    if (sigma_lm) h->d_sigma.download(sigma_lm, 2 * (size_t)h->grid.nlm, s);
    VG_CUDA(cudaStreamSynchronize(s));
  });
}

int vg_enable_visc3d_from_nodes(vg_handle* h, const double* visc_node, double lid_depth, double lid_log10max,
                                double log10_cap) {
  return guarded(h, [&] {
    need(h, visc_node != nullptr, "vg_enable_visc3d_from_nodes: visc_node is required");
    const int ng = h->grid.ng, ne = h->ne, nr = h->nr;
    const double r_top = h->r[nr - 1];
    const double r_lid = lid_depth > 0.0 ? r_top - lid_depth : HUGE_VAL;  // no element above it: rule off
    std::vector<double> pert((size_t)ne * ng, 0.0);
    for (int e = 0; e < ne; ++e) {
      if (h->MkPerDt[e] == 0.0) continue;  // elastic / fluid: stay as they are
      const double logeta_ref = std::log10(h->mu[e] / h->MkPerDt[e]);
      const bool in_lid = h->r[e] >= r_lid - 1.0e-6 * r_top;  // element wholly above the lid base
      for (int g = 0; g < ng; ++g) {
        double v = 0.5 * (visc_node[(size_t)e * ng + g] + visc_node[(size_t)(e + 1) * ng + g]);  // log10-mean
        if (in_lid && v > lid_log10max) v = log10_cap;
        pert[(size_t)e * ng + g] = v - logeta_ref;
      }
    }
    vg::visc3d_enable(h, pert.data());
  });
}

int vg_update_device(vg_handle* h, const double* d_h_ice, double dt_yr) {
  return guarded(h, [&] {
    need(h, h->have_reference, "vg_update: call vg_set_reference first (solid_earth_init)");
    need(h, d_h_ice != nullptr, "vg_update: h_ice is required");
    vg::update_dev(h, d_h_ice, dt_yr);
    VG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int vg_update(vg_handle* h, const double* h_ice, double dt_yr) {
  return guarded(h, [&] {
    need(h, h->have_reference, "vg_update: call vg_set_reference first (solid_earth_init)");
    need(h, h_ice != nullptr, "vg_update: h_ice is required");
    h->d_ice1.upload(h_ice, h->grid.ng, h->stream);
    vg::update_dev(h, h->d_ice1.p, dt_yr);
    VG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int vg_update_batch(vg_handle* const* hs, int n, const double* const* ice, int ice_on_device, double dt_yr,
                    int nthreads, int* failed_index) {
  if (failed_index) *failed_index = -1;
  const int arg = guarded(nullptr, [&] {
    need(nullptr, n >= 0, "vg_update_batch: n must be >= 0");
    need(nullptr, n == 0 || (hs != nullptr && ice != nullptr), "vg_update_batch: null argument");
    std::vector<vg_handle*> seen(hs, hs + n);
    std::sort(seen.begin(), seen.end());
    for (int i = 0; i < n; ++i) {
      need(nullptr, seen[i] != nullptr, "vg_update_batch: null handle");
      need(nullptr, i == 0 || seen[i] != seen[i - 1], "vg_update_batch: a handle appears twice");
    }
  });
  if (arg != 0) return arg;
  if (n == 0) return 0;
  // costliest first (state size; 3-D elements weigh in with the transforms)
  std::vector<int> order(n);
  std::vector<double> cost(n);
  for (int i = 0; i < n; ++i) {
    order[i] = i;
    cost[i] = (double)hs[i]->nk * hs[i]->ne * (1.0 + 4.0 * hs[i]->ne3d / std::max(hs[i]->ne, 1));
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<int> rc(n, 0);
  std::atomic<int> next{0};
  auto work = [&] {
    for (int t = next++; t < n; t = next++) {
      const int i = order[t];
      vg_handle* h = hs[i];
      if (cudaSetDevice(h->device) != cudaSuccess) {
        h->err = "vg_update_batch: cudaSetDevice failed";
        rc[i] = 1;
        continue;
      }
      rc[i] = ice_on_device ? vg_update_device(h, ice[i], dt_yr) : vg_update(h, ice[i], dt_yr);
    }
  };
  const int nt = std::min(n, nthreads <= 0 ? n : nthreads);
  std::vector<std::thread> pool;
  pool.reserve(nt);
  try {
    for (int t = 0; t < nt; ++t) pool.emplace_back(work);
  } catch (const std::exception&) {
    // no more threads to be had: the calling thread takes the rest of the queue
  }
  if (pool.empty()) work();
  for (std::thread& th : pool) th.join();
  for (int i = 0; i < n; ++i)
    if (rc[i] != 0) {
      if (failed_index) *failed_index = i;
      return rc[i];
    }
  return 0;
}

int vg_get_fields(vg_handle* h, double* rsl, double* z_bed, double* C, double* sigma_lm) {
  return guarded(h, [&] {
    const int ng = h->grid.ng;
    cudaStream_t s = h->stream;
    if (rsl) h->d_rsl.download(rsl, ng, s);
    if (z_bed) h->d_zbed.download(z_bed, ng, s);
    if (C) h->d_C.download(C, ng, s);
    if (sigma_lm) h->d_sigma.download(sigma_lm, 2 * (size_t)h->grid.nlm, s);
    VG_CUDA(cudaStreamSynchronize(s));
  });
}

int vg_rsl_device(vg_handle* h, const double** d_rsl) {
  return guarded(h, [&] {
    need(h, d_rsl != nullptr, "vg_rsl_device: null argument");
    *d_rsl = h->d_rsl.p;
  });
}

int vg_get_rotation(vg_handle* h, double* m, double* love) {
  return guarded(h, [&] {
    if (!h->rot_on) throw vg::Error("vg_get_rotation: rotational feedback is off for this handle");
    double sc[2] = {0.0, 0.0};
    VG_CUDA(cudaMemcpyAsync(sc, h->d_rot_sc.p + 8, sizeof(sc), cudaMemcpyDeviceToHost, h->stream));
    VG_CUDA(cudaStreamSynchronize(h->stream));
    if (m) {
      m[0] = sc[0];
      m[1] = sc[1];
    }
    if (love) {
      love[0] = h->rot_kTe;
      love[1] = h->rot_hTe;
      love[2] = h->rot_ks_fluid;
      love[3] = h->rot_ks_flat;
    }
  });
}

int vg_get_info(vg_handle* h, vg_info* info) {
  return guarded(h, [&] {
    std::memset(info, 0, sizeof(*info));
    info->lmax = h->grid.lmax;
    info->nlat = h->grid.nlat;
    info->nphi = h->grid.nphi;
    info->nlm = h->grid.nlm;
    info->nr = h->nr;
    info->ne = h->ne;
    info->ndof = h->ndof;
    info->nk = h->nk;
    info->ne3d = h->ne3d;
    info->n_sub_last = h->n_sub_last;
    info->n_accept = h->n_accept;
    info->n_reject = h->n_reject;
    info->n_solve = h->n_solve;
    info->n_drift_solved = h->n_drift_solved;
    info->time_yr = h->time_yr;
    info->worst_mass_resid = h->worst_mass_resid;
    info->bsl = h->bsl;
    info->n_outer_last = h->n_outer_last;
    info->n_inner_last = h->n_inner_last;
    info->n_coast_flip_last = h->n_flip_last;
    info->n_launch = h->n_launch;
  });
}

int vg_stream(vg_handle* h, void** stream) {
  return guarded(h, [&] {
    need(h, stream != nullptr, "vg_stream: null argument");
    *stream = (void*)h->stream;
  });
}

int vg_set_wait_limit(vg_handle* h, double seconds) {
  return guarded(h, [&] {
    if (!(seconds >= 0.0) || seconds > 60.0) throw vg::Error("vg_set_wait_limit: seconds must be in [0, 60]");
    h->wait_ns = (unsigned long long)(seconds * 1.0e9);
  });
}

int vg_profile_enable(vg_handle* h, int on) {
  return guarded(h, [&] {
    if (h->prof.on && !on) vg::prof_collect(h);
    h->prof.on = on != 0;
  });
}

int vg_profile_read(vg_handle* h, double* ms, long long* calls) {
  return guarded(h, [&] {
    vg::prof_collect(h);
    for (int ph = 0; ph < VG_NPHASE; ++ph) {
      if (ms) ms[ph] = h->prof.ms[ph];
      if (calls) calls[ph] = h->prof.calls[ph];
      h->prof.ms[ph] = 0.0;
      h->prof.calls[ph] = 0;
    }
  });
}

int vg_response_set_dt(vg_handle* h, double dt_s) {
  return guarded(h, [&] { h->dt = dt_s; });
}

int vg_response_begin_step(vg_handle* h) {
  return guarded(h, [&] {
    vg::launch_drift(h);
    VG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int vg_response_apply(vg_handle* h, const double* sigma_lm, double* u_lm, double* n_lm) {
  return guarded(h, [&] {
    const size_t n2 = 2 * (size_t)h->grid.nlm;
    h->d_sigma.upload(sigma_lm, n2, h->stream);
    vg::launch_apply(h, h->d_sigma.p, h->d_ulm.p, h->d_ulm.p + n2);
    if (u_lm) VG_CUDA(cudaMemcpyAsync(u_lm, h->d_ulm.p, n2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (n_lm)
      VG_CUDA(cudaMemcpyAsync(n_lm, h->d_ulm.p + n2, n2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    VG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int vg_response_advance(vg_handle* h, const double* sigma_lm) {
  return guarded(h, [&] {
    const size_t n2 = 2 * (size_t)h->grid.nlm;
    h->d_sigma.upload(sigma_lm, n2, h->stream);
    vg::advance_memory(h, h->d_sigma.p, h->dt);
    h->cur = 1 - h->cur;
    h->mem_norm = vg::read_mem_norm(h, h->cur);
    h->time_s += h->dt;
  });
}

int vg_get_gains(vg_handle* h, double* gu, double* gn, double* gv) {
  return guarded(h, [&] {
    int L = h->grid.lmax + 1;
    if (gu) h->d_gu.download(gu, L, h->stream);
    if (gn) h->d_gn.download(gn, L, h->stream);
    if (gv) h->d_gv.download(gv, L, h->stream);
    VG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int vg_get_drift(vg_handle* h, double* dUa, double* dFa, double* dVa) {
  return guarded(h, [&] {
    const int nk = h->nk;
    std::vector<double> d((size_t)6 * nk);
    h->d_drift.download(d.data(), d.size(), h->stream);
    VG_CUDA(cudaStreamSynchronize(h->stream));
    double* outs[3] = {dUa, dFa, dVa};
    for (int q = 0; q < 3; ++q)
      if (outs[q])
        for (int k = 0; k < nk; ++k) {
          outs[q][2 * k] = d[(size_t)(2 * q) * nk + k];
          outs[q][2 * k + 1] = d[(size_t)(2 * q + 1) * nk + k];
        }
  });
}

// restart layout (NLAM, ne, nk) <-> device [s][ri][e][lam][k]
int vg_get_state(vg_handle* h, double* Are, double* Aim, double* Bre, double* Bim, double* Cre, double* Cim,
                 double* time_s) {
  return guarded(h, [&] {
    const int ne = h->ne, nk = h->nk;
    const size_t per = (size_t)ne * 4 * nk;
    std::vector<double> m(6 * per);
    h->d_mem[h->cur].download(m.data(), m.size(), h->stream);
    VG_CUDA(cudaStreamSynchronize(h->stream));
    double* outs[6] = {Are, Aim, Bre, Bim, Cre, Cim};  // (s, ri) = (0,0),(0,1),(1,0),...
    for (int q = 0; q < 6; ++q) {
      if (!outs[q]) continue;
      const double* src = m.data() + q * per;
      for (int e = 0; e < ne; ++e)
        for (int lam = 0; lam < 4; ++lam)
          for (int k = 0; k < nk; ++k) outs[q][((size_t)k * ne + e) * 4 + lam] = src[((size_t)e * 4 + lam) * nk + k];
    }
    if (time_s) *time_s = h->time_s;
  });
}

int vg_get_toroidal(vg_handle* h, double* t_lm) {
  return guarded(h, [&] {
    need(h, t_lm != nullptr, "vg_get_toroidal: null argument");
    const int nlm = h->grid.nlm, nk = h->nk;
    for (int i = 0; i < 2 * nlm; ++i) t_lm[i] = 0.0;
    if (!h->tor_on) return;
    std::vector<double> w((size_t)2 * nk);
    h->d_dWa.download(w.data(), w.size(), h->stream);
    VG_CUDA(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < nk; ++k) {
      t_lm[2 * h->k2lm_h[k]] = w[k];
      t_lm[2 * h->k2lm_h[k] + 1] = w[(size_t)nk + k];
    }
  });
}

// toroidal restart layout (NLAM_TOR, ne, nk) <-> device [s][ri][e][lam][k]
int vg_get_state_tor(vg_handle* h, double* Are, double* Aim, double* Bre, double* Bim, double* Cre, double* Cim,
                     int* carried) {
  return guarded(h, [&] {
    need(h, carried != nullptr, "vg_get_state_tor: null argument");
    *carried = h->tor_on ? 1 : 0;
    if (!h->tor_on) return;
    const int ne = h->ne, nk = h->nk;
    const size_t per = (size_t)ne * 2 * nk;
    std::vector<double> m(6 * per);
    h->d_tmem[h->cur].download(m.data(), m.size(), h->stream);
    VG_CUDA(cudaStreamSynchronize(h->stream));
    double* outs[6] = {Are, Aim, Bre, Bim, Cre, Cim};
    for (int q = 0; q < 6; ++q) {
      if (!outs[q]) continue;
      const double* src = m.data() + q * per;
      for (int e = 0; e < ne; ++e)
        for (int lam = 0; lam < 2; ++lam)
          for (int k = 0; k < nk; ++k) outs[q][((size_t)k * ne + e) * 2 + lam] = src[((size_t)e * 2 + lam) * nk + k];
    }
  });
}

int vg_set_state_tor(vg_handle* h, const double* Are, const double* Aim, const double* Bre, const double* Bim,
                     const double* Cre, const double* Cim) {
  return guarded(h, [&] {
    need(h, h->tor_on, "vg_set_state_tor: the toroidal channels are not carried by this handle");
    const int ne = h->ne, nk = h->nk;
    const size_t per = (size_t)ne * 2 * nk;
    std::vector<double> m(6 * per);
    const double* ins[6] = {Are, Aim, Bre, Bim, Cre, Cim};
    for (int q = 0; q < 6; ++q) {
      need(h, ins[q] != nullptr, "vg_set_state_tor: all six memory arrays are required");
      double* dst = m.data() + q * per;
      for (int e = 0; e < ne; ++e)
        for (int lam = 0; lam < 2; ++lam)
          for (int k = 0; k < nk; ++k) dst[((size_t)e * 2 + lam) * nk + k] = ins[q][((size_t)k * ne + e) * 2 + lam];
    }
    h->d_tmem[h->cur].upload(m.data(), m.size(), h->stream);
    vg::compute_mem_norm(h, h->cur);
    h->mem_norm = vg::read_mem_norm(h, h->cur);
  });
}

int vg_get_step_state(vg_handle* h, double* dt_try_yr, double* sigma_n, int* sigma_primed) {
  return guarded(h, [&] {
    if (dt_try_yr) *dt_try_yr = h->dt_try / vg::SEC_PER_YEAR;
    const bool tracked = h->sigma_primed && h->d_sigma_n.p != nullptr;
    if (sigma_primed) *sigma_primed = tracked ? 1 : 0;
    if (sigma_n) {
      const size_t n2 = 2 * (size_t)h->grid.nlm;
      if (tracked) {
        h->d_sigma_n.download(sigma_n, n2, h->stream);
        VG_CUDA(cudaStreamSynchronize(h->stream));
      } else {
        for (size_t i = 0; i < n2; ++i) sigma_n[i] = 0.0;
      }
    }
  });
}

int vg_set_step_state(vg_handle* h, double dt_try_yr, const double* sigma_n, int sigma_primed) {
  return guarded(h, [&] {
    need(h, !(sigma_primed && !sigma_n), "vg_set_step_state: a primed sigma_n is required");
    need(h, !(sigma_primed && h->p.scheme != VG_SCHEME_TRAP),
         "vg_set_step_state: sigma_n is tracked by the trapezoidal scheme only");
    h->dt_try = dt_try_yr * vg::SEC_PER_YEAR;
    h->sigma_primed = false;
    if (sigma_primed) {
      h->d_sigma_n.upload(sigma_n, 2 * (size_t)h->grid.nlm, h->stream);
      VG_CUDA(cudaStreamSynchronize(h->stream));
      h->sigma_primed = true;
    }
  });
}

int vg_set_state(vg_handle* h, const double* Are, const double* Aim, const double* Bre, const double* Bim,
                 const double* Cre, const double* Cim, double time_s) {
  return guarded(h, [&] {
    const int ne = h->ne, nk = h->nk;
    const size_t per = (size_t)ne * 4 * nk;
    std::vector<double> m(6 * per);
    const double* ins[6] = {Are, Aim, Bre, Bim, Cre, Cim};
    for (int q = 0; q < 6; ++q) {
      need(h, ins[q] != nullptr, "vg_set_state: all six memory arrays are required");
      double* dst = m.data() + q * per;
      for (int e = 0; e < ne; ++e)
        for (int lam = 0; lam < 4; ++lam)
          for (int k = 0; k < nk; ++k) dst[((size_t)e * 4 + lam) * nk + k] = ins[q][((size_t)k * ne + e) * 4 + lam];
    }
    h->d_mem[h->cur].upload(m.data(), m.size(), h->stream);
    vg::compute_mem_norm(h, h->cur);
    h->mem_norm = vg::read_mem_norm(h, h->cur);
    h->time_s = time_s;
    h->time_yr = time_s / vg::SEC_PER_YEAR;
    h->sigma_primed = false;  // trapezoidal scheme: the next update seeds sigma_n from this state
  });
}

int vg_set_fields(vg_handle* h, const double* h_ice, const double* rsl, const double* z_bed, const double* C) {
  return guarded(h, [&] {
    need(h, h->have_reference, "vg_set_fields: vg_set_reference must come first");
    const int ng = h->grid.ng;
    cudaStream_t s = h->stream;
    if (h_ice) h->d_h_ice.upload(h_ice, ng, s);
    if (rsl) h->d_rsl.upload(rsl, ng, s);
    if (z_bed) h->d_zbed.upload(z_bed, ng, s);
    if (C) h->d_C.upload(C, ng, s);
    vg::update_bsl(h);
  });
}

int vg_get_rotation_state(vg_handle* h, double* m, double* load_mem, double* tidal_mem) {
  return guarded(h, [&] {
    need(h, h->rot_on, "vg_get_rotation_state: rotational feedback is off for this handle");
    const size_t per = (size_t)6 * h->ne * 4;
    cudaStream_t s = h->stream;
    if (m) VG_CUDA(cudaMemcpyAsync(m, h->d_rot_sc.p + 8, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (load_mem) VG_CUDA(cudaMemcpyAsync(load_mem, h->d_rot_mem.p, per * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (tidal_mem)
      VG_CUDA(cudaMemcpyAsync(tidal_mem, h->d_rot_mem.p + per, per * sizeof(double), cudaMemcpyDeviceToHost, s));
    VG_CUDA(cudaStreamSynchronize(s));
  });
}

int vg_set_rotation_state(vg_handle* h, const double* m, const double* load_mem, const double* tidal_mem) {
  return guarded(h, [&] {
    need(h, h->rot_on, "vg_set_rotation_state: rotational feedback is off for this handle");
    need(h, m && load_mem && tidal_mem, "vg_set_rotation_state: m and both channel memories are required");
    const size_t per = (size_t)6 * h->ne * 4;
    cudaStream_t s = h->stream;
    VG_CUDA(cudaMemcpyAsync(h->d_rot_sc.p + 8, m, 2 * sizeof(double), cudaMemcpyHostToDevice, s));
    VG_CUDA(cudaMemcpyAsync(h->d_rot_mem.p, load_mem, per * sizeof(double), cudaMemcpyHostToDevice, s));
    VG_CUDA(cudaMemcpyAsync(h->d_rot_mem.p + per, tidal_mem, per * sizeof(double), cudaMemcpyHostToDevice, s));
    VG_CUDA(cudaStreamSynchronize(s));
  });
}

int vg_sht_analysis(vg_handle* h, const double* f, double* q_lm) {
  return guarded(h, [&] {
    const int ng = h->grid.ng;
    const size_t n2 = 2 * (size_t)h->grid.nlm;
    h->d_tmp.upload(f, ng, h->stream);
    vg::sht_analysis_dev(h, h->d_tmp.p, h->d_nlm.p, 1);
    h->d_nlm.download(q_lm, n2, h->stream);
    VG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int vg_sht_synthesis(vg_handle* h, const double* q_lm, double* f) {
  return guarded(h, [&] {
    const int ng = h->grid.ng;
    const size_t n2 = 2 * (size_t)h->grid.nlm;
    h->d_nlm.upload(q_lm, n2, h->stream);
    vg::sht_synthesis_dev(h, h->d_nlm.p, h->d_tmp.p, 1);
    h->d_tmp.download(f, ng, h->stream);
    VG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

}  // extern "C"

namespace vg {

void DriverSnap::save(vg_handle* h) {
  cudaStream_t s = h->stream;
  const size_t S = h->d_mem[0].n, nk = h->nk, ng = h->grid.ng, n2 = 2 * (size_t)h->grid.nlm;
  cur = h->cur;
  auto grab = [&](DArr<double>& dst, const double* src, size_t n) {
    if (dst.n < n) dst.alloc(n);
    VG_CUDA(cudaMemcpyAsync(dst.p, src, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  };
  grab(mem, h->d_mem[cur].p, S);
  grab(mnorm, h->d_mnorm.p + (size_t)cur * nk, nk);
  grab(rsl, h->d_rsl.p, ng);
  grab(hice, h->d_h_ice.p, ng);
  grab(C, h->d_C.p, ng);
  grab(zbed, h->d_zbed.p, ng);
  grab(sig, h->d_sigma.p, n2);
  if (h->tor_on) grab(tmem, h->d_tmem[cur].p, h->d_tmem[cur].n);
  sigma_primed = h->sigma_primed;
  dt_try = h->dt_try;
  if (h->d_sigma_n.p) grab(sig_n, h->d_sigma_n.p, h->d_sigma_n.n);
  if (h->rot_on) {
    grab(rot_sc, h->d_rot_sc.p, h->d_rot_sc.n);
    grab(rot_mem, h->d_rot_mem.p, h->d_rot_mem.n);
  }
  if (maxbits.n < 2) maxbits.alloc(2);
  VG_CUDA(cudaMemcpyAsync(maxbits.p, h->d_maxbits.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s));
  time_s = h->time_s;
  time_yr = h->time_yr;
  mem_norm = h->mem_norm;
  bsl = h->bsl;
  worst = h->worst_mass_resid;
  n_accept = h->n_accept;
  n_reject = h->n_reject;
  n_solve = h->n_solve;
  n_sub = h->n_sub_last;
  n_outer = h->n_outer_last;
  n_inner = h->n_inner_last;
  n_flip = h->n_flip_last;
}

void DriverSnap::restore(vg_handle* h) {
  cudaStream_t s = h->stream;
  const size_t S = h->d_mem[0].n, nk = h->nk, ng = h->grid.ng, n2 = 2 * (size_t)h->grid.nlm;
  h->cur = cur;
  auto put = [&](double* dst, const DArr<double>& src, size_t n) {
    VG_CUDA(cudaMemcpyAsync(dst, src.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  };
  put(h->d_mem[cur].p, mem, S);
  put(h->d_mnorm.p + (size_t)cur * nk, mnorm, nk);
  put(h->d_rsl.p, rsl, ng);
  put(h->d_h_ice.p, hice, ng);
  put(h->d_C.p, C, ng);
  put(h->d_zbed.p, zbed, ng);
  put(h->d_sigma.p, sig, n2);
  if (h->tor_on) put(h->d_tmem[cur].p, tmem, h->d_tmem[cur].n);
  h->sigma_primed = sigma_primed;
  h->dt_try = dt_try;
  if (h->d_sigma_n.p && sig_n.n >= h->d_sigma_n.n) put(h->d_sigma_n.p, sig_n, h->d_sigma_n.n);
  if (h->rot_on) {
    put(h->d_rot_sc.p, rot_sc, h->d_rot_sc.n);
    put(h->d_rot_mem.p, rot_mem, h->d_rot_mem.n);
  }
  VG_CUDA(cudaMemcpyAsync(h->d_maxbits.p, maxbits.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s));
  h->time_s = time_s;
  h->time_yr = time_yr;
  h->mem_norm = mem_norm;
  h->bsl = bsl;
  h->worst_mass_resid = worst;
  h->n_accept = n_accept;
  h->n_reject = n_reject;
  h->n_solve = n_solve;
  h->n_sub_last = n_sub;
  h->n_outer_last = n_outer;
  h->n_inner_last = n_inner;
  h->n_flip_last = n_flip;
  VG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace vg
