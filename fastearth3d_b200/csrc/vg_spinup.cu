// LGM-memory spin-up: solid_earth_spinup (src/vilma_coupling.f90:453-570).
// Seed the entering ice with a zero-length update; optionally relax first under
// the lateral mean of the 3-D viscosity (pre_spinup_1d); then, in relax_hold,
// hold h_ice_lgm over passes of SPINUP_DT0 years
// growing by SPINUP_GROW (at most SPINUP_MAXP passes, capped at t_max in total)
// until the mean bed velocity int |z_bed - z_prev| dOmega / (4 pi) / pass_dt
// falls below rate_tol [m/yr]. Each pass is an ordinary update on the device;
// the bed change is reduced per latitude row on the device and integrated on
// the host in row order with the Gauss weights (sht_grid_surface_integral).
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

constexpr double SPINUP_DT0 = 200.0;  // first relaxation interval [yr] (src/vilma_coupling.f90:65)
constexpr double SPINUP_GROW = 1.6;   // interval growth per pass (:66)
constexpr int SPINUP_MAXP = 60;       // cap on relaxation passes (:67)

// row sums of |a - b| (one CTA per latitude row)
__global__ void k_absdiff_rows(int nphi, const double* __restrict__ a, const double* __restrict__ b,
                               double* __restrict__ out) {
  __shared__ double red[128];
  const int j = blockIdx.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    const size_t p = (size_t)j * nphi + i;
    v += fabs(a[p] - b[p]);
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) out[j] = v;
}

// mean |z_bed - z_prev| over the sphere [m]
static double mean_bed_change(vg_handle* h, const double* d_prev, double* d_rows) {
  const Grid& G = h->grid;
  k_absdiff_rows<<<G.nlat, 128, 0, h->stream>>>(G.nphi, h->d_zbed.p, d_prev, d_rows);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  std::vector<double> rows(G.nlat);
  VG_CUDA(cudaMemcpyAsync(rows.data(), d_rows, G.nlat * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  VG_CUDA(cudaStreamSynchronize(h->stream));
  const double dlon = 2.0 * PI / (double)G.nphi;
  double integral = 0.0;
  for (int j = 0; j < G.nlat; ++j) integral += G.wts[j] * rows[j] * dlon;
  return integral / (4.0 * PI);
}

// relax_hold (src/vilma_coupling.f90:500-545): t_cap <= 0 runs to rest within
// the pass cap only
static void relax_hold(vg_handle* h, const double* d_ice_lgm, double t_cap, double tol, double& t_done, int& passes,
                       bool& converged) {
  const Grid& G = h->grid;
  t_done = 0.0;
  passes = 0;
  converged = false;
  DArr<double> prev, rows;
  prev.alloc(G.ng);
  rows.alloc(G.nlat);
  VG_CUDA(cudaMemcpyAsync(prev.p, h->d_zbed.p, G.ng * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  double pass_dt = SPINUP_DT0;
  for (int it = 1; it <= SPINUP_MAXP; ++it) {
    if (t_cap > 0.0) pass_dt = std::min(pass_dt, t_cap - t_done);
    if (pass_dt <= 0.0) break;
    update_dev(h, d_ice_lgm, pass_dt);
    t_done += pass_dt;
    passes = it;
    const double rate = mean_bed_change(h, prev.p, rows.p) / pass_dt;  // mean bed velocity [m/yr]
    if (rate < tol) {
      converged = true;
      break;
    }
    VG_CUDA(cudaMemcpyAsync(prev.p, h->d_zbed.p, G.ng * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    pass_dt = pass_dt * SPINUP_GROW;
  }
}

// The lateral mean of the 3-D field (src/vilma_coupling.f90:484-493): every
// genuinely 3-D element advances spectrally at mu / eta_radial * 10^-(mean
// perturbation), as a laterally uniform element does, until restored.
struct LateralMean {
  vg_handle* h;
  std::vector<double> MkPerDt;
  std::vector<char> active1d;
  int ne3d;
  double max_rate;
  explicit LateralMean(vg_handle* hh) : h(hh), MkPerDt(hh->MkPerDt), active1d(hh->active1d_h), ne3d(hh->ne3d),
                                        max_rate(hh->max_rate) {
    for (size_t ei = 0; ei < h->e3d_h.size(); ++ei) {
      const int e = h->e3d_h[ei];
      h->MkPerDt[e] = MkPerDt[e] * std::pow(10.0, -h->pert_mean3d[ei]);
      h->active1d_h[e] = 1;
    }
    h->ne3d = 0;
    h->max_rate = 0.0;
    for (double v : h->MkPerDt) h->max_rate = std::max(h->max_rate, v);
    upload();
  }
  void upload() {
    h->d_MkPerDt.upload(h->MkPerDt, h->stream);
    h->d_active1d.upload(h->active1d_h, h->stream);
    VG_CUDA(cudaStreamSynchronize(h->stream));
  }
  ~LateralMean() {  // the real 3-D field (solid_earth_enable_visc_3d); never throws
    h->MkPerDt = MkPerDt;
    h->active1d_h = active1d;
    h->ne3d = ne3d;
    h->max_rate = max_rate;
    cudaMemcpyAsync(h->d_MkPerDt.p, h->MkPerDt.data(), h->MkPerDt.size() * sizeof(double), cudaMemcpyHostToDevice,
                    h->stream);
    cudaMemcpyAsync(h->d_active1d.p, h->active1d_h.data(), h->active1d_h.size(), cudaMemcpyHostToDevice, h->stream);
    cudaStreamSynchronize(h->stream);
  }
};

void spinup_dev(vg_handle* h, const double* d_ice_lgm, double t_cap, double tol, bool pre_1d, double& t_done,
                int& passes, bool& converged, int& passes_1d) {
  t_done = 0.0;
  passes = 0;
  converged = false;
  passes_1d = 0;
  if (!pre_1d && !(t_cap > 0.0)) return;  // nothing to do (src/vilma_coupling.f90:477)
  update_dev(h, d_ice_lgm, 0.0);  // seed the entering ice = the start (LGM) ice
  if (pre_1d) {
    std::unique_ptr<LateralMean> mean;
    if (h->lat_visc && !h->e3d_h.empty()) mean.reset(new LateralMean(h));
    double t1 = 0.0;
    bool c1 = false;
    relax_hold(h, d_ice_lgm, -1.0, tol, t1, passes_1d, c1);
  }
  if (t_cap > 0.0) relax_hold(h, d_ice_lgm, t_cap, tol, t_done, passes, converged);
}

}  // namespace vg

extern "C" int vg_spinup(vg_handle* h, const double* h_ice_lgm, double t_max_yr, double rate_tol, int pre_1d,
                         double* t_done_yr, int* passes, int* converged, int* passes_1d) {
  if (!h) return 1;
  try {
    if (!h->have_reference) throw vg::Error("vg_spinup: call vg_set_reference first (solid_earth_init)");
    if (!h_ice_lgm) throw vg::Error("vg_spinup: h_ice_lgm is required");
    vg::DArr<double> d_ice;
    d_ice.alloc(h->grid.ng);
    d_ice.upload(h_ice_lgm, h->grid.ng, h->stream);
    double t = 0.0;
    int n = 0, n1 = 0;
    bool ok = false;
    vg::spinup_dev(h, d_ice.p, t_max_yr, rate_tol, pre_1d != 0, t, n, ok, n1);
    VG_CUDA(cudaStreamSynchronize(h->stream));
    if (t_done_yr) *t_done_yr = t;
    if (passes) *passes = n;
    if (converged) *converged = ok ? 1 : 0;
    if (passes_1d) *passes_1d = n1;
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}
