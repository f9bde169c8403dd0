// vg_sht_analysis_noalloc: the Gauss-grid analysis of vg_sht_analysis with
// caller-owned device buffers and its Fourier-coefficient scratch in a
// file-scope device array, so that a call allocates no device or host memory.
//
// The scratch is one static array per device (the module's copy of the
// symbol). Its device address is looked up on every call, with the handle's
// device current, through cudaGetSymbolAddress: the address belongs to the
// current context, so it stays right across a cudaDeviceReset or a new
// context on the same ordinal (a cached address would then point at freed
// memory). Once the module is loaded the lookup is a table search; the first
// call on a device may load the module, so make it before any stream capture.
// Nothing in the scratch has to start at zero: each call's Fourier stage
// writes every element the Legendre stage then reads. Calls that overlap in
// time on one device (other streams, other handles, other host threads) share
// the array and race; order them on one stream or synchronise between them.
#include <cstdio>

#include "vg_internal.cuh"

static __device__ __align__(256) double g_fourier_scratch[VG_NOALLOC_SCRATCH_DOUBLES];

namespace {

// device address of the scratch in the current context
double* scratch_address() {
  void* p = nullptr;
  VG_CUDA(cudaGetSymbolAddress(&p, g_fourier_scratch));
  if (!p) throw vg::Error("vg_sht_analysis_noalloc: no device address for the scratch array");
  return static_cast<double*>(p);
}

}  // namespace

extern "C" int vg_sht_analysis_noalloc(vg_handle* h, const double* d_f, double* d_q_lm, int batch) {
  if (!h) return 1;
  try {
    if (!d_f || !d_q_lm) throw vg::Error("vg_sht_analysis_noalloc: null device pointer");
    if (batch < 1) throw vg::Error("vg_sht_analysis_noalloc: batch must be >= 1");
    const vg::Grid& G = h->grid;
    const size_t need = 2 * (size_t)G.M * (size_t)G.nlat * (size_t)batch;
    if (need > (size_t)VG_NOALLOC_SCRATCH_DOUBLES) {
      char msg[200];
      std::snprintf(msg, sizeof(msg),
                    "vg_sht_analysis_noalloc: %zu doubles of scratch needed (2 * %d orders * %d latitudes * batch %d), "
                    "limit %d",
                    need, G.M, G.nlat, batch, (int)VG_NOALLOC_SCRATCH_DOUBLES);
      throw vg::Error(msg);
    }
    int dev = -1;
    VG_CUDA(cudaGetDevice(&dev));
    if (dev != h->device) throw vg::Error("vg_sht_analysis_noalloc: the handle's device is not the current device");
    double* F = scratch_address();
    vg::fourier_analysis_dev(h, d_f, batch, F);
    vg::legendre_analysis_dev(h, F, batch, d_q_lm);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}
