// Host lon-lat <-> Gauss-grid remap of the coupling layer (src/vilma_remap.f90:
// 56-166; src/vilma_coupling.f90:172-176, 355-359, 436-447, 631-641): ice (and
// the reference fields) in by first-order conservative remapping, relative sea
// level out by bilinear interpolation, on the device.
//
// Both grids are lon-lat rectangles with cell boundaries at the axis midpoints
// (the outermost half a spacing beyond the last centre, latitudes clamped to
// +/-90), so a source / target overlap on the sphere is (longitude overlap) x
// (sin-latitude overlap): the conservative map factorises into a latitude pass
// and a longitude pass, each a short sparse sum per output (stat "mean": the
// weights of each target row and column are normalised by their coverage).
// The optional mass rescale makes the Gauss quadrature integral equal the
// source area integral (remap_to_gauss, :124-133). The bilinear leg takes the
// four surrounding Gauss nodes (the outermost row poleward of it).
//   k_remap_lat    one thread per (Gauss row, source column)
//   k_remap_lon    one thread per (Gauss row, Gauss column)
//   k_remap_mass   one CTA: both integrals and the rescale factor
//   k_remap_scale  the rescale
//   k_remap_bilin  one thread per host cell; optionally z_bed = z_bed_eq - rsl
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "vg_device.cuh"
#include "vg_internal.cuh"

using vg::DArr;
using vg::Error;

struct vg_remap {
  vg_handle* h = nullptr;
  int nlon = 0, nlat_s = 0;
  // conservative: per Gauss row (north first) the source rows, per Gauss column
  // the source columns, CSR with normalised weights
  DArr<int> d_rp, d_ri, d_cp, d_ci;
  DArr<double> d_rw, d_cw;
  DArr<double> d_dz, d_dl;  // source cell extents: sin-latitude (nlat_s), longitude [rad] (nlon)
  // bilinear: per host row (Gauss rows j0, j1, weight a), per host column (i0, i1, b)
  DArr<int> d_bj, d_bi;
  DArr<double> d_ba, d_bb;
  DArr<double> d_fll, d_tmp, d_fg, d_out, d_zeq_ll, d_scale;
  std::string err;
};

namespace vg {

static std::vector<double> axis_bounds(const double* x, int n, bool clamp) {
  std::vector<double> b(n + 1);
  for (int i = 1; i < n; ++i) b[i] = 0.5 * (x[i] + x[i - 1]);
  b[0] = x[0] - 0.5 * (x[1] - x[0]);
  b[n] = x[n - 1] + 0.5 * (x[n - 1] - x[n - 2]);
  if (clamp)
    for (double& v : b) v = std::min(90.0, std::max(-90.0, v));
  return b;
}

// length (degrees) of [a0, a1) intersect [b0, b1) on the circle
static double lon_overlap(double a0, double a1, double b0, double b1) {
  double tot = 0.0;
  for (int k = -2; k <= 2; ++k) {
    const double lo = std::max(a0, b0 + 360.0 * k), hi = std::min(a1, b1 + 360.0 * k);
    if (hi > lo) tot += hi - lo;
  }
  return tot;
}

__global__ void k_remap_lat(int nlat, int nlon, const int* __restrict__ rp, const int* __restrict__ ri,
                            const double* __restrict__ rw, const double* __restrict__ f, double* __restrict__ t) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (c >= nlon || j >= nlat) return;
  double acc = 0.0;
  for (int q = rp[j]; q < rp[j + 1]; ++q) acc = fma(rw[q], f[(size_t)ri[q] * nlon + c], acc);
  t[(size_t)j * nlon + c] = acc;
}

__global__ void k_remap_lon(int nlat, int nphi, int nlon, const int* __restrict__ cp, const int* __restrict__ ci,
                            const double* __restrict__ cw, const double* __restrict__ t, double* __restrict__ g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= nphi || j >= nlat) return;
  double acc = 0.0;
  for (int q = cp[i]; q < cp[i + 1]; ++q) acc = fma(cw[q], t[(size_t)j * nlon + ci[q]], acc);
  g[(size_t)j * nphi + i] = acc;
}

// scale = (sum f dz dl / sum dz dl * 4 pi) / (2 pi / nphi sum_j w_j sum_i g), 1 when the
// Gauss integral vanishes
__global__ void k_remap_mass(int nlat_s, int nlon, const double* __restrict__ f, const double* __restrict__ dz,
                             const double* __restrict__ dl, int nlat, int nphi, const double* __restrict__ g,
                             const double* __restrict__ wts, double* __restrict__ scale) {
  __shared__ double red[1024];
  double s = 0.0, a = 0.0, gi = 0.0;
  for (int t = threadIdx.x; t < nlat_s * nlon; t += blockDim.x) {
    const double w = dz[t / nlon] * dl[t % nlon];
    s += f[t] * w;
    a += w;
  }
  for (int t = threadIdx.x; t < nlat * nphi; t += blockDim.x) gi += wts[t / nphi] * g[t];
  s = block_sum(s, red);
  a = block_sum(a, red);
  gi = block_sum(gi, red);
  if (threadIdx.x == 0) {
    const double src = s / a * 4.0 * PI, gint = gi * (2.0 * PI / (double)nphi);
    scale[0] = fabs(gint) > TINY ? src / gint : 1.0;
  }
}

__global__ void k_remap_scale(int n, const double* __restrict__ scale, double* __restrict__ g) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) g[t] *= scale[0];
}

__global__ void k_remap_bilin(int nlat_s, int nlon, int nphi, const int* __restrict__ bj, const double* __restrict__ ba,
                              const int* __restrict__ bi, const double* __restrict__ bb, const double* __restrict__ g,
                              const double* __restrict__ zeq, double* __restrict__ out, double* __restrict__ zbed) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (c >= nlon || r >= nlat_s) return;
  const int j0 = bj[2 * r], j1 = bj[2 * r + 1], i0 = bi[2 * c], i1 = bi[2 * c + 1];
  const double a = ba[r], b = bb[c];
  const double v = (1.0 - a) * ((1.0 - b) * g[(size_t)j0 * nphi + i0] + b * g[(size_t)j0 * nphi + i1]) +
                   a * ((1.0 - b) * g[(size_t)j1 * nphi + i0] + b * g[(size_t)j1 * nphi + i1]);
  out[(size_t)r * nlon + c] = v;
  if (zbed) zbed[(size_t)r * nlon + c] = zeq[(size_t)r * nlon + c] - v;
}

// conservative ll -> Gauss of the device field r->d_fll into dst (nlat, nphi), north first
static void remap_in(vg_remap* r, double* dst, bool conserve_mass) {
  vg_handle* h = r->h;
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  k_remap_lat<<<dim3((r->nlon + 127) / 128, G.nlat), 128, 0, s>>>(G.nlat, r->nlon, r->d_rp.p, r->d_ri.p, r->d_rw.p,
                                                                   r->d_fll.p, r->d_tmp.p);
  VG_CUDA(cudaGetLastError());
  k_remap_lon<<<dim3((G.nphi + 127) / 128, G.nlat), 128, 0, s>>>(G.nlat, G.nphi, r->nlon, r->d_cp.p, r->d_ci.p,
                                                                  r->d_cw.p, r->d_tmp.p, dst);
  VG_CUDA(cudaGetLastError());
  if (!conserve_mass) return;
  k_remap_mass<<<1, 1024, 0, s>>>(r->nlat_s, r->nlon, r->d_fll.p, r->d_dz.p, r->d_dl.p, G.nlat, G.nphi, dst,
                                  G.d_wts.p, r->d_scale.p);
  VG_CUDA(cudaGetLastError());
  k_remap_scale<<<(G.ng + 255) / 256, 256, 0, s>>>(G.ng, r->d_scale.p, dst);
  VG_CUDA(cudaGetLastError());
}

static void remap_out(vg_remap* r, const double* g, double* out, double* zbed) {
  vg_handle* h = r->h;
  k_remap_bilin<<<dim3((r->nlon + 127) / 128, r->nlat_s), 128, 0, h->stream>>>(
      r->nlat_s, r->nlon, h->grid.nphi, r->d_bj.p, r->d_ba.p, r->d_bi.p, r->d_bb.p, g, r->d_zeq_ll.p, out, zbed);
  VG_CUDA(cudaGetLastError());
}

// remap_init (src/vilma_remap.f90:56-99)
static void remap_build(vg_remap* r, const double* lon_src, const double* lat_src) {
  vg_handle* h = r->h;
  const Grid& G = h->grid;
  const int nlat = G.nlat, nphi = G.nphi, nlon = r->nlon, ns = r->nlat_s;
  for (int k = 1; k < ns; ++k)
    if (!(lat_src[k] > lat_src[k - 1])) throw Error("vg_remap_create: source latitudes must ascend");
  for (int k = 1; k < nlon; ++k)
    if (!(lon_src[k] > lon_src[k - 1])) throw Error("vg_remap_create: source longitudes must ascend");
  // Gauss axes, south first for the bounds
  std::vector<double> latg(nlat), long_(nphi);
  for (int j = 0; j < nlat; ++j) latg[j] = 90.0 - G.colat[nlat - 1 - j] * (180.0 / PI);
  for (int i = 0; i < nphi; ++i) long_[i] = 360.0 * (double)i / (double)nphi;
  const std::vector<double> lbs = axis_bounds(lon_src, nlon, false), pbs = axis_bounds(lat_src, ns, true);
  const std::vector<double> lbg = axis_bounds(long_.data(), nphi, false), pbg = axis_bounds(latg.data(), nlat, true);
  std::vector<double> ss(ns + 1), sg(nlat + 1);
  for (int k = 0; k <= ns; ++k) ss[k] = std::sin(pbs[k] * PI / 180.0);
  for (int k = 0; k <= nlat; ++k) sg[k] = std::sin(pbg[k] * PI / 180.0);
  // latitude pass: Gauss row jn (north first) = ascending row nlat - 1 - jn
  std::vector<int> rp(nlat + 1, 0), ri;
  std::vector<double> rw;
  for (int jn = 0; jn < nlat; ++jn) {
    const int j = nlat - 1 - jn;
    const size_t q0 = rw.size();
    double cover = 0.0;
    for (int k = 0; k < ns; ++k) {
      const double dz = std::min(sg[j + 1], ss[k + 1]) - std::max(sg[j], ss[k]);
      if (dz > 0.0) {
        ri.push_back(k);
        rw.push_back(dz);
        cover += dz;
      }
    }
    for (size_t q = q0; q < rw.size(); ++q) rw[q] /= cover;
    rp[jn + 1] = (int)rw.size();
  }
  std::vector<int> cp(nphi + 1, 0), ci;
  std::vector<double> cw;
  for (int i = 0; i < nphi; ++i) {
    const size_t q0 = cw.size();
    double cover = 0.0;
    for (int k = 0; k < nlon; ++k) {
      const double dl = lon_overlap(lbg[i], lbg[i + 1], lbs[k], lbs[k + 1]);
      if (dl > 0.0) {
        ci.push_back(k);
        cw.push_back(dl);
        cover += dl;
      }
    }
    for (size_t q = q0; q < cw.size(); ++q) cw[q] /= cover;
    cp[i + 1] = (int)cw.size();
  }
  std::vector<double> dz(ns), dl(nlon);
  for (int k = 0; k < ns; ++k) dz[k] = ss[k + 1] - ss[k];
  for (int k = 0; k < nlon; ++k) dl[k] = (lbs[k + 1] - lbs[k]) * PI / 180.0;
  // bilinear: per host row the Gauss rows (north-first indices), per host column the Gauss columns
  std::vector<int> bj(2 * ns), bi(2 * nlon);
  std::vector<double> ba(ns), bb(nlon);
  for (int k = 0; k < ns; ++k) {
    const double y = lat_src[k];
    int j0, j1;
    double a;
    if (y <= latg[0]) {
      j0 = j1 = 0;
      a = 0.0;
    } else if (y >= latg[nlat - 1]) {
      j0 = j1 = nlat - 1;
      a = 0.0;
    } else {
      j0 = (int)(std::upper_bound(latg.begin(), latg.end(), y) - latg.begin()) - 1;
      j1 = j0 + 1;
      a = (y - latg[j0]) / (latg[j1] - latg[j0]);
    }
    bj[2 * k] = nlat - 1 - j0;
    bj[2 * k + 1] = nlat - 1 - j1;
    ba[k] = a;
  }
  const double dlon = 360.0 / (double)nphi;
  for (int k = 0; k < nlon; ++k) {
    double x = std::fmod(lon_src[k], 360.0);
    if (x < 0.0) x += 360.0;
    const int i0 = ((int)std::floor(x / dlon)) % nphi;
    bi[2 * k] = i0;
    bi[2 * k + 1] = (i0 + 1) % nphi;
    bb[k] = (x - i0 * dlon) / dlon;
  }
  cudaStream_t s = h->stream;
  r->d_rp.upload(rp, s);
  r->d_ri.upload(ri, s);
  r->d_rw.upload(rw, s);
  r->d_cp.upload(cp, s);
  r->d_ci.upload(ci, s);
  r->d_cw.upload(cw, s);
  r->d_dz.upload(dz, s);
  r->d_dl.upload(dl, s);
  r->d_bj.upload(bj, s);
  r->d_bi.upload(bi, s);
  r->d_ba.upload(ba, s);
  r->d_bb.upload(bb, s);
  r->d_fll.alloc((size_t)ns * nlon);
  r->d_tmp.alloc((size_t)nlat * nlon);
  r->d_out.alloc((size_t)ns * nlon);
  r->d_fg.alloc((size_t)G.ng);
  r->d_zeq_ll.alloc((size_t)ns * nlon);
  r->d_scale.alloc(1);
  VG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace vg

template <class F>
static int rguard(vg_remap* r, F&& f) {
  if (!r) return 1;
  try {
    f();
    return 0;
  } catch (const std::exception& ex) {
    r->err = ex.what();
    if (r->h) r->h->err = ex.what();
    return 1;
  }
}

extern "C" {

int vg_remap_create(vg_handle* h, const double* lon_src, int nlon, const double* lat_src, int nlat,
                    vg_remap** out) {
  if (!h || !out) return 1;
  *out = nullptr;
  vg_remap* r = new vg_remap();
  r->h = h;
  r->nlon = nlon;
  r->nlat_s = nlat;
  try {
    if (!lon_src || !lat_src || nlon < 2 || nlat < 2) throw Error("vg_remap_create: need at least 2 x 2 source axes");
    vg::remap_build(r, lon_src, lat_src);
  } catch (const std::exception& ex) {
    h->err = ex.what();
    delete r;
    return 1;
  }
  *out = r;
  return 0;
}

int vg_remap_destroy(vg_remap* r) {
  delete r;
  return 0;
}

int vg_remap_to_gauss(vg_remap* r, const double* f_ll, double* f_gauss, int conserve_mass) {
  return rguard(r, [&] {
    if (!f_ll || !f_gauss) throw Error("vg_remap_to_gauss: null argument");
    cudaStream_t s = r->h->stream;
    r->d_fll.upload(f_ll, r->d_fll.n, s);
    vg::remap_in(r, r->d_fg.p, conserve_mass != 0);
    r->d_fg.download(f_gauss, r->d_fg.n, s);
    VG_CUDA(cudaStreamSynchronize(s));
  });
}

int vg_remap_to_ll(vg_remap* r, const double* f_gauss, double* f_ll) {
  return rguard(r, [&] {
    if (!f_ll || !f_gauss) throw Error("vg_remap_to_ll: null argument");
    cudaStream_t s = r->h->stream;
    r->d_fg.upload(f_gauss, r->d_fg.n, s);
    vg::remap_out(r, r->d_fg.p, r->d_out.p, nullptr);
    VG_CUDA(cudaMemcpyAsync(f_ll, r->d_out.p, r->d_out.n * sizeof(double), cudaMemcpyDeviceToHost, s));
    VG_CUDA(cudaStreamSynchronize(s));
  });
}

int vg_set_reference_ll(vg_remap* r, const double* z_bed_eq_ll, const double* h_ice_eq_ll,
                        const double* h_ice_init_ll) {
  return rguard(r, [&] {
    if (!z_bed_eq_ll || !h_ice_eq_ll) throw Error("vg_set_reference_ll: z_bed_eq and h_ice_eq are required");
    vg_handle* h = r->h;
    cudaStream_t s = h->stream;
    const size_t ng = (size_t)h->grid.ng, nll = r->d_fll.n;
    std::vector<double> zb(ng), hi(ng), h0;
    r->d_zeq_ll.upload(z_bed_eq_ll, nll, s);
    r->d_fll.upload(z_bed_eq_ll, nll, s);
    vg::remap_in(r, r->d_fg.p, false);  // bed: geometry
    r->d_fg.download(zb.data(), ng, s);
    r->d_fll.upload(h_ice_eq_ll, nll, s);
    vg::remap_in(r, r->d_fg.p, true);  // ice: mass
    r->d_fg.download(hi.data(), ng, s);
    if (h_ice_init_ll) {
      h0.resize(ng);
      r->d_fll.upload(h_ice_init_ll, nll, s);
      vg::remap_in(r, r->d_fg.p, true);
      r->d_fg.download(h0.data(), ng, s);
    }
    VG_CUDA(cudaStreamSynchronize(s));
    if (vg_set_reference(h, zb.data(), hi.data(), h_ice_init_ll ? h0.data() : nullptr) != 0) throw Error(h->err);
  });
}

int vg_update_ll(vg_remap* r, const double* h_ice_ll, double dt_yr, double* rsl_ll, double* z_bed_ll) {
  return rguard(r, [&] {
    if (!h_ice_ll) throw Error("vg_update_ll: h_ice is required");
    vg_handle* h = r->h;
    cudaStream_t s = h->stream;
    const size_t nll = r->d_fll.n;
    r->d_fll.upload(h_ice_ll, nll, s);
    vg::remap_in(r, r->d_fg.p, true);  // ice load on the Gauss grid (src/vilma_coupling.f90:355-359)
    if (vg_update_device(h, r->d_fg.p, dt_yr) != 0) throw Error(h->err);
    // rsl back to the host grid, z_bed on the host's own bed (solid_earth_sync_host, :438-447)
    vg::remap_out(r, h->d_rsl.p, r->d_out.p, z_bed_ll ? r->d_fll.p : nullptr);
    if (rsl_ll) VG_CUDA(cudaMemcpyAsync(rsl_ll, r->d_out.p, nll * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (z_bed_ll) VG_CUDA(cudaMemcpyAsync(z_bed_ll, r->d_fll.p, nll * sizeof(double), cudaMemcpyDeviceToHost, s));
    VG_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
