// Autotuner of the time step's launch shapes (no reference counterpart: the
// reference's OpenMP loops have no shapes to choose).
//
// Two knobs, both free of any effect on the results (every choice gives the
// same bits, which tests/test_gpu_autotune.py checks):
//   * the exact tensor-core stages' split of their 16 worker warps between
//     converters (FP64 rows to digit planes) and epilogue (level
//     combination, scaling, stores): 8 : 8 or 4 : 12, per stage;
//   * the CTA count of the fused sea-level loop's cooperative grid: one per
//     SM, one per Gauss row, or two per SM where they fit.
// Each candidate runs a few whole intervals of the handle's own model on the
// ice it holds, timed per phase by the handle's phase timers, from the same
// saved driver state (put back after every trial and at the end). The best
// per stage and for the loop is kept, applied to the handle and appended to a
// plain-text cache keyed by the model's sizes and the knobs tuned, which
// later handles of the same key read instead of timing.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "vg_internal.cuh"

namespace vg {
namespace {

struct Choice {
  int ncw[4] = {8, 8, 8, 8};
  int sle_ctas = 0;
};

const int PH_STAGE[4] = {VG_PH_V3_SYNTH, VG_PH_V3_LON_INV, VG_PH_V3_LON_FWD, VG_PH_V3_ANALYSIS};

std::string tune_key(const vg_handle* h, int knobs) {
  char k[220];
  std::snprintf(k, sizeof(k), "lmax=%d nlat=%d nphi=%d ne=%d ne3d=%d precision=%d toroidal=%d sle=%d knobs=%d",
                h->grid.lmax, h->grid.nlat, h->grid.nphi, h->ne, h->lat_visc ? h->ne3d : 0, h->p.visc3d_precision,
                h->tor_on ? 1 : 0, h->p.sle_fixed_ocean ? 0 : 1, knobs);
  return k;
}

// cache lines: "<key> | ncw=a,b,c,d sle_ctas=n"
bool cache_lookup(const char* path, const std::string& key, Choice& c) {
  if (!path || !*path) return false;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    const size_t bar = line.find(" | ");
    if (bar == std::string::npos || line.compare(0, bar, key) != 0 || bar != key.size()) continue;
    Choice t;
    if (std::sscanf(line.c_str() + bar + 3, "ncw=%d,%d,%d,%d sle_ctas=%d", &t.ncw[0], &t.ncw[1], &t.ncw[2],
                    &t.ncw[3], &t.sle_ctas) == 5) {
      for (int i = 0; i < 4; ++i)
        if (t.ncw[i] != 4 && t.ncw[i] != 8) return false;
      c = t;
      return true;
    }
  }
  return false;
}

void cache_store(const char* path, const std::string& key, const Choice& c) {
  if (!path || !*path) return;
  std::ofstream f(path, std::ios::app);
  if (!f) throw Error(std::string("vg_autotune: cannot write the cache file ") + path);
  f << key << " | ncw=" << c.ncw[0] << "," << c.ncw[1] << "," << c.ncw[2] << "," << c.ncw[3]
    << " sle_ctas=" << c.sle_ctas << "\n";
}

void apply(vg_handle* h, const Choice& c) {
  int cur[4];
  if (oz_get_ncw(h, cur)) oz_set_ncw(h, c.ncw);
  if (h->p.sle_ctas != c.sle_ctas) {
    h->p.sle_ctas = c.sle_ctas;
    h->sle_grid = 0;  // the fused loop's grid is sized again at its next launch
  }
}

// milliseconds per phase of `reps` intervals after one untimed interval, from the saved state
void trial(vg_handle* h, DriverSnap& snap, const double* d_ice, double dt_yr, int reps, double* ms) {
  update_dev(h, d_ice, dt_yr);
  h->prof.on = true;
  for (int r = 0; r < reps; ++r) update_dev(h, d_ice, dt_yr);
  prof_collect(h);
  h->prof.on = false;
  for (int ph = 0; ph < VG_NPHASE; ++ph) {
    ms[ph] = h->prof.ms[ph];
    h->prof.ms[ph] = 0.0;
    h->prof.calls[ph] = 0;
  }
  snap.restore(h);
}

}  // namespace

void autotune(vg_handle* h, double dt_yr, int knobs, const char* cache_path, int* from_cache) {
  if (!h->have_reference) throw Error("vg_autotune: call vg_set_reference first (solid_earth_init)");
  if (!(dt_yr > 0.0)) throw Error("vg_autotune: dt_yr must be > 0");
  if (knobs & ~(VG_TUNE_STAGES | VG_TUNE_SLE)) throw Error("vg_autotune: unknown knob bits");
  const std::string key = tune_key(h, knobs);
  Choice best;
  best.sle_ctas = h->p.sle_ctas;
  int ncw0[4];
  const bool exact = oz_get_ncw(h, ncw0);
  if (exact)
    for (int i = 0; i < 4; ++i) best.ncw[i] = ncw0[i];
  if (cache_lookup(cache_path, key, best)) {
    apply(h, best);
    if (from_cache) *from_cache = 1;
    return;
  }
  if (from_cache) *from_cache = 0;
  const bool prof_was = h->prof.on;
  if (prof_was) prof_collect(h);
  DriverSnap snap;
  snap.save(h);
  DArr<double> ice;  // the held load: the handle's current ice
  ice.alloc(h->grid.ng);
  VG_CUDA(cudaMemcpyAsync(ice.p, h->d_h_ice.p, h->grid.ng * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  const int reps = 3;
  std::vector<double> ms(VG_NPHASE);
  // exact stages: each stage's split, all four timed in one trial per split
  if (exact && (knobs & VG_TUNE_STAGES)) {
    double t_best[4] = {0, 0, 0, 0};
    const int cand[2] = {8, 4};
    for (int ci = 0; ci < 2; ++ci) {
      const int all[4] = {cand[ci], cand[ci], cand[ci], cand[ci]};
      oz_set_ncw(h, all);
      trial(h, snap, ice.p, dt_yr, reps, ms.data());
      for (int i = 0; i < 4; ++i) {
        const double t = ms[PH_STAGE[i]];
        if (ci == 0 || t < t_best[i]) {
          t_best[i] = t;
          best.ncw[i] = cand[ci];
        }
      }
    }
  }
  apply(h, best);
  // the fused sea-level loop's CTA count (only when the model has an ocean to solve for)
  if (!h->p.sle_fixed_ocean && (knobs & VG_TUNE_SLE)) {
    int dev = 0, nsm = 0;
    VG_CUDA(cudaGetDevice(&dev));
    VG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int cands[3] = {0, h->grid.nlat, 2 * nsm};  // 0: one per SM; the launch caps at what fits
    double t_best = -1.0;
    int c_best = best.sle_ctas;
    for (int c : cands) {
      Choice t = best;
      t.sle_ctas = c;
      apply(h, t);
      trial(h, snap, ice.p, dt_yr, reps, ms.data());
      const double v = ms[VG_PH_SLE];
      if (v > 0.0 && (t_best < 0.0 || v < t_best)) {
        t_best = v;
        c_best = c;
      }
    }
    best.sle_ctas = c_best;
  }
  apply(h, best);
  h->prof.on = prof_was;
  cache_store(cache_path, key, best);
}

}  // namespace vg

extern "C" int vg_autotune(vg_handle* h, double dt_yr, int knobs, const char* cache_path, int* from_cache) {
  if (!h) return 1;
  try {
    vg::autotune(h, dt_yr, knobs, cache_path, from_cache);
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}

extern "C" int vg_get_tuning(vg_handle* h, int* ncw, int* sle_ctas) {
  if (!h) return 1;
  try {
    int c[4] = {0, 0, 0, 0};
    vg::oz_get_ncw(h, c);
    if (ncw)
      for (int i = 0; i < 4; ++i) ncw[i] = c[i];
    if (sle_ctas) *sle_ctas = h->p.sle_ctas;
    return 0;
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return 1;
  }
}
