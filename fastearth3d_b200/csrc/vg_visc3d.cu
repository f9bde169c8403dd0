// Laterally varying viscosity: the pseudo-spectral Maxwell memory advance of
// the genuinely 3-D elements (src/vilma_response.f90:994-1053, 1171-1319).
#include <algorithm>
#include <cmath>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

void visc3d_enable(vg_handle* h, const double* pert) {
  (void)h;
  (void)pert;
  throw Error("vg_enable_visc3d: lateral viscosity is not built yet");
}

void visc3d_advance(vg_handle* h, const double* d_sigma, double dt) {
  (void)h;
  (void)d_sigma;
  (void)dt;
  throw Error("visc3d_advance: lateral viscosity is not built yet");
}

}  // namespace vg
