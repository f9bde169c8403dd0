// Sea-level equation on the device (src/vilma_sle.f90:124-425) and the
// explicit sub-stepping driver with its reactive guard (src/vilma_timestep.f90:
// 79-227), i.e. one solid_earth_update (src/vilma_coupling.f90:336-437) with
// every field resident in HBM. The host only takes the scalar decisions the
// reference takes (coastline, inner convergence, guard), from one small
// device-to-host read each.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

enum { RP_C = 0, RP_DIG, RP_ZETA, RP_CS, RP_DMAX, RP_SMAX, RP_FLIP, RP_MASS, RP_N };

__device__ __forceinline__ double ocean(double topo, double ice) {
  return (topo < 0.0 && RHO_ICE * ice < -RHO_WATER * topo) ? 1.0 : 0.0;
}

__global__ void k_ice_interp(int ng, double frac, const double* __restrict__ ice0, const double* __restrict__ ice1,
                             const double* __restrict__ ice_ref, double* __restrict__ ice_now,
                             double* __restrict__ dice_now) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ng) return;
  double v = ice0[i] + frac * (ice1[i] - ice0[i]);
  ice_now[i] = v;
  dice_now[i] = v - ice_ref[i];
}

// C0 = ocean_function(topo0, ice - d_ice)  (src/vilma_sle.f90:212)
__global__ void k_ocean0(int ng, const double* __restrict__ topo0, const double* __restrict__ ice,
                         const double* __restrict__ dice, double* __restrict__ C0) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ng) C0[i] = ocean(topo0[i], ice[i] - dice[i]);
}
// C = ocean_function(topo0 - rsl, ice)
__global__ void k_ocean(int ng, const double* __restrict__ topo0, const double* __restrict__ rsl,
                        const double* __restrict__ ice, double* __restrict__ C) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ng) C[i] = ocean(topo0[i] - rsl[i], ice[i]);
}

// grounded-ice increment and the per-row sums of C, dIg, topo0 (C - C0)
__global__ void k_pass_setup(int nphi, const double* __restrict__ ice, const double* __restrict__ dice,
                             const double* __restrict__ C, const double* __restrict__ C0,
                             const double* __restrict__ topo0, double* __restrict__ dig,
                             double* __restrict__ rowpart, int nlat) {
  __shared__ double red[128];
  int j = blockIdx.x;
  double sc = 0.0, sd = 0.0, sz = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    size_t p = (size_t)j * nphi + i;
    double d = ice[p] * (1.0 - C[p]) - (ice[p] - dice[p]) * (1.0 - C0[p]);
    dig[p] = d;
    sc += C[p];
    sd += d;
    sz += topo0[p] * (C[p] - C0[p]);
  }
  sc = block_sum(sc, red);
  sd = block_sum(sd, red);
  sz = block_sum(sz, red);
  if (threadIdx.x == 0) {
    rowpart[RP_C * nlat + j] = sc;
    rowpart[RP_DIG * nlat + j] = sd;
    rowpart[RP_ZETA * nlat + j] = sz;
  }
}

// Surface integral of a row-sum vector, sum_j w_j row_j 2 pi / nphi
// (src/vilma_sht.f90:184-202), summed in row order like the reference. The
// finalizer kernels run one block: every thread stages a slice of the terms
// in shared memory (one coalesced pass), then thread 0 adds them in order.
// The result is valid in thread 0.
constexpr int FIN_THREADS = 128, FIN_SEG = 1024;
__device__ double integrate_rows(const double* row, const double* w, int nlat, double dlon) {
  __shared__ double term[FIN_SEG];
  double total = 0.0;
  for (int j0 = 0; j0 < nlat; j0 += FIN_SEG) {
    const int n = min(FIN_SEG, nlat - j0);
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) term[j] = w[j0 + j] * row[j0 + j] * dlon;
    __syncthreads();
    if (threadIdx.x == 0) {  // in row order; the loads run ahead of the dependent adds
      int j = 0;
      for (; j + 8 <= n; j += 8) {
        double t[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) t[q] = term[j + q];
#pragma unroll
        for (int q = 0; q < 8; ++q) total += t[q];
      }
      for (; j < n; ++j) total += term[j];
    }
  }
  return total;
}

// the pass's ocean area, then (with an ocean) its ice and subgrid integrals
__global__ void k_finalize_pass(SleScalars* sc, const double* __restrict__ rowpart, const double* __restrict__ w,
                                int nlat, double dlon, int subgrid) {
  __shared__ double s_c;
  const double c = integrate_rows(rowpart + RP_C * nlat, w, nlat, dlon);  // valid in thread 0
  if (threadIdx.x == 0) {
    sc->C_int = c;
    s_c = c;
  }
  __syncthreads();
  if (!(s_c > 0.0)) return;  // no ocean: the pass ends here (src/vilma_sle.f90:273-274)
  const double d = integrate_rows(rowpart + RP_DIG * nlat, w, nlat, dlon);
  const double z = subgrid ? integrate_rows(rowpart + RP_ZETA * nlat, w, nlat, dlon) : 0.0;
  if (threadIdx.x == 0) {
    sc->ice_int = -(RHO_ICE / RHO_WATER) * d;
    sc->zeta_int = z;
  }
}
__global__ void k_wcorr(const SleScalars* sc, int ng, int subgrid, const double* __restrict__ topo0,
                        const double* __restrict__ C, const double* __restrict__ C0, double* __restrict__ wcorr) {
  if (!(sc->C_int > 0.0)) return;  // no ocean
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ng) wcorr[i] = subgrid ? -RHO_WATER * topo0[i] * (C[i] - C0[i]) : 0.0;
}

// total surface load (assemble_load, src/vilma_sle.f90:387-403) and its longitude transform
__global__ void k_load_fourier(int nphi, int nlat, int M, const double* __restrict__ dig,
                               const double* __restrict__ C, const double* __restrict__ rsl,
                               const double* __restrict__ wcorr, const double* __restrict__ cs,
                               const double* __restrict__ sn, double* __restrict__ F) {
  extern __shared__ double row[];
  int j = blockIdx.x;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    size_t p = (size_t)j * nphi + i;
    row[i] = RHO_ICE * dig[p] + RHO_WATER * (C[p] * rsl[p]) + wcorr[p];
  }
  __syncthreads();
  row_fourier_analysis(row, nphi, M, cs, sn, F + (size_t)j * 2, nlat);
}

// u and N rows from their Legendre sums, Sraw = N - u (+ s_rot), row sum of C Sraw
__global__ void k_synth_sraw(int nphi, int nlat, int M, const double* __restrict__ G, const double* __restrict__ cs,
                             const double* __restrict__ sn, const double* __restrict__ C,
                             const double* __restrict__ srot, double* __restrict__ Sraw,
                             double* __restrict__ rowpart) {
  extern __shared__ double sh[];  // Gu[M][2], Gn[M][2]
  __shared__ double red[128];
  int j = blockIdx.x;
  double* Gu = sh;
  double* Gn = sh + 2 * M;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    Gu[2 * m] = G[((size_t)m * nlat + j) * 2];
    Gu[2 * m + 1] = G[((size_t)m * nlat + j) * 2 + 1];
    Gn[2 * m] = G[(((size_t)M + m) * nlat + j) * 2];
    Gn[2 * m + 1] = G[(((size_t)M + m) * nlat + j) * 2 + 1];
  }
  __syncthreads();
  double acc = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    size_t p = (size_t)j * nphi + i;
    double u = row_fourier_synth_at(Gu, M, i, nphi, cs, sn);
    double N = row_fourier_synth_at(Gn, M, i, nphi, cs, sn);
    double s = N - u;
    if (srot) s = s + srot[p];
    Sraw[p] = s;
    acc += C[p] * s;
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) rowpart[RP_CS * nlat + j] = acc;
}

__global__ void k_dphi(SleScalars* sc, const double* __restrict__ rowpart, const double* __restrict__ w, int nlat,
                       double dlon) {
  const double Cs = integrate_rows(rowpart + RP_CS * nlat, w, nlat, dlon);
  if (threadIdx.x == 0) {
    sc->Cs_int = Cs;
    sc->dphi = (sc->ice_int - Cs + sc->zeta_int) / sc->C_int;
  }
}

__global__ void k_rsl_update(int nphi, const SleScalars* __restrict__ sc, const double* __restrict__ Sraw,
                             const double* __restrict__ C, double* __restrict__ rsl, double* __restrict__ rowpart,
                             int nlat) {
  __shared__ double red[128];
  int j = blockIdx.x;
  double dphi = sc->dphi, dmax = 0.0, smax = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    size_t p = (size_t)j * nphi + i;
    double rn = Sraw[p] + dphi;
    dmax = nanmax(dmax, fabs(C[p] * (rn - rsl[p])));
    rsl[p] = rn;
    smax = nanmax(smax, fabs(C[p] * rn));
  }
  dmax = block_max(dmax, red);
  smax = block_max(smax, red);
  if (threadIdx.x == 0) {
    rowpart[RP_DMAX * nlat + j] = dmax;
    rowpart[RP_SMAX * nlat + j] = smax;
  }
}

__global__ void k_conv(SleScalars* sc, const double* __restrict__ rowpart, int nlat) {
  __shared__ double red[FIN_THREADS];
  double dmax = 0.0, smax = 0.0;
  for (int j = threadIdx.x; j < nlat; j += blockDim.x) {
    dmax = nanmax(dmax, rowpart[RP_DMAX * nlat + j]);
    smax = nanmax(smax, rowpart[RP_SMAX * nlat + j]);
  }
  dmax = block_max(dmax, red);
  smax = block_max(smax, red);
  if (threadIdx.x == 0) {
    sc->dmax = dmax;
    sc->smax = smax;
  }
}

// migrated coastline and the number of cells that changed state
__global__ void k_coast(int nphi, const double* __restrict__ topo0, const double* __restrict__ rsl,
                        const double* __restrict__ ice, const double* __restrict__ C, double* __restrict__ Cn,
                        double* __restrict__ rowpart, int nlat) {
  __shared__ double red[128];
  int j = blockIdx.x;
  double cnt = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    size_t p = (size_t)j * nphi + i;
    double c = ocean(topo0[p] - rsl[p], ice[p]);
    Cn[p] = c;
    cnt += (c != C[p]) ? 1.0 : 0.0;
  }
  cnt = block_sum(cnt, red);
  if (threadIdx.x == 0) rowpart[RP_FLIP * nlat + j] = cnt;
}
__global__ void k_flips(SleScalars* sc, const double* __restrict__ rowpart, int nlat) {
  __shared__ double red[FIN_THREADS];
  double t = 0.0;  // integer-valued row counts: exact in any order
  for (int j = threadIdx.x; j < nlat; j += blockDim.x) t += rowpart[RP_FLIP * nlat + j];
  t = block_sum(t, red);
  if (threadIdx.x == 0) sc->flips = (int)t;
}

// row sums of a * b (b may be null: sum of a), into rowpart slot
__global__ void k_rowsum(int nphi, const double* __restrict__ a, const double* __restrict__ b,
                         double* __restrict__ out) {
  __shared__ double red[128];
  int j = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    size_t p = (size_t)j * nphi + i;
    s += b ? a[p] * b[p] : a[p];
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[j] = s;
}
__global__ void k_mass(SleScalars* sc, const double* __restrict__ rowpart, const double* __restrict__ w, int nlat,
                       double dlon) {
  const double m = integrate_rows(rowpart + RP_MASS * nlat, w, nlat, dlon);
  if (threadIdx.x == 0) sc->mass_Cs = m - sc->zeta_int;
}

// z_bed = z_bed_eq - rsl (src/vilma_coupling.f90:428)
__global__ void k_zbed(int ng, const double* __restrict__ zeq, const double* __restrict__ rsl,
                       double* __restrict__ zb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ng) zb[i] = zeq[i] - rsl[i];
}
// row sums of C and of h_ice (1 - C) - h_ice_eq (1 - C0), for update_bsl
__global__ void k_bsl_rows(int nphi, const double* __restrict__ hi, const double* __restrict__ hq,
                           const double* __restrict__ C, const double* __restrict__ C0, double* __restrict__ rowpart,
                           int nlat) {
  __shared__ double red[128];
  int j = blockIdx.x;
  double sc = 0.0, st = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    size_t p = (size_t)j * nphi + i;
    sc += C[p];
    st += hi[p] * (1.0 - C[p]) - hq[p] * (1.0 - C0[p]);
  }
  sc = block_sum(sc, red);
  st = block_sum(st, red);
  if (threadIdx.x == 0) {
    rowpart[RP_C * nlat + j] = sc;
    rowpart[RP_DIG * nlat + j] = st;
  }
}

// ------------------------------------------------------------------ fused inner loop
// The inner load fixed point of sle_solve (src/vilma_sle.f90:280-340) as one
// cooperative persistent kernel: one CTA per SM, the convergence test on the
// device, so no host round trip per iteration. Four grid barriers an
// iteration:
//   L  total load of each row and its longitude analysis (the CTA that owns
//      the row; for the next iteration it runs right after U, on the rows the
//      CTA has just updated)
//   A  Legendre analysis + apply, warp per lm                 | barrier
//   S  Legendre synthesis of u and N, thread per (b, m, j)    | barrier
//   R  longitude synthesis, Sraw = N - u (+ s_rot), row sums  | barrier
//   U  mass-conserving dphi (every CTA, rows summed in order by one thread,
//      so all CTAs agree), rsl update, row maxima, then L     | barrier
//   convergence (every CTA from the row maxima, the same decision everywhere)
// The longitude transforms split the half periods (phi + pi flips odd m) and
// spread each output's sum over several threads, so no thread runs a loop of
// more than about nphi / 6 terms.
constexpr int SLE_LCH = 16;  // degrees per Legendre synthesis chunk

struct InnerArgs {
  int nphi, nlat, M, nlm, nk, lmax, n_inner;
  double tol, dlon, g;
  const double *dig, *C, *wcorr, *cs, *sn, *plm, *wts, *gu, *gn, *drift, *srot;
  const int *lm_m, *lm_l, *lm2k, *mbeg;
  const int2* chunk;  // Legendre synthesis chunks: (m, first l - m), at most SLE_LCH degrees each
  const int* cbeg;    // first chunk of each order (M + 1)
  int nchunk;
  double *rsl, *F, *sigma, *ulm, *Gp, *Sraw, *rowpart;
  SleScalars* sc;
  unsigned int* bar;  // count, generation, error
  unsigned long long wait_ns;  // bound on a grid barrier's wait (the handle's wait limit, 2 s by default)
};

__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Sense-counting grid barrier with a bounded wait. Returns false (in every
// thread of the CTA) if it timed out or another CTA reported a timeout.
__device__ bool grid_barrier(unsigned int* bar, unsigned int& gen, unsigned long long wait_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned int* vgen = bar + 1;
    __threadfence();
    const unsigned int arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      bar[0] = 0u;
      __threadfence();
      atomicExch(bar + 1, gen + 1u);
    } else {
      const unsigned long long t0 = gtimer_ns();
      while (*vgen == gen) {
        if (gtimer_ns() - t0 > wait_ns) {
          atomicExch(bar + 2, 1u);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (*(volatile unsigned int*)(bar + 2)) ok = 0;
    s_ok = ok;
  }
  ++gen;
  __syncthreads();
  return s_ok != 0;
}

// L for row j: the total surface load and its longitude analysis into F
// (F_m = 2 pi / nphi sum_i f_i e^{-i m phi_i}; even m read f_i + f_{i+half},
// odd m f_i - f_{i+half}); tpm threads per order, partial sums in part[2][nthr]
__device__ __forceinline__ void sle_row_load(const InnerArgs& A, int j, double* sm, double* part) {
  const int tid = threadIdx.x, nthr = blockDim.x, nphi = A.nphi, M = A.M, half = nphi / 2;
  const double sc_f = 2.0 * PI / (double)nphi;
  __syncthreads();
  for (int i = tid; i < nphi; i += nthr) {
    const size_t p = (size_t)j * nphi + i;
    sm[i] = RHO_ICE * A.dig[p] + RHO_WATER * (A.C[p] * A.rsl[p]) + A.wcorr[p];
  }
  __syncthreads();
  const int tpm = max(1, min(8, nthr / M));
  for (int base = 0; base < M * tpm; base += nthr) {
    const int u = base + tid, m = u / tpm, q = u % tpm;
    const bool act = u < M * tpm;
    double re = 0.0, im = 0.0;
    if (act) {
      const double sg = (m & 1) ? -1.0 : 1.0;
      const int step = (m * tpm) % nphi;
      int t = (m * q) % nphi;
      for (int i = q; i < half; i += tpm) {
        const double v = sm[i] + sg * sm[i + half];
        re += v * __ldg(&A.cs[t]);
        im -= v * __ldg(&A.sn[t]);
        t += step;
        if (t >= nphi) t -= nphi;
      }
    }
    part[tid] = re;
    part[nthr + tid] = im;
    __syncthreads();
    if (act && q == 0) {
      double r = 0.0, s2 = 0.0;
      for (int c = 0; c < tpm; ++c) {
        r += part[tid + c];
        s2 += part[nthr + tid + c];
      }
      A.F[((size_t)m * A.nlat + j) * 2] = r * sc_f;
      A.F[((size_t)m * A.nlat + j) * 2 + 1] = s2 * sc_f;
    }
    __syncthreads();
  }
}

// a grid barrier gave up: record it where the host reads the loop's scalars
__device__ __forceinline__ void bar_fail(const InnerArgs& A) {
  if (threadIdx.x == 0) A.sc->bar_error = 1;
}

__global__ void __launch_bounds__(512) k_sle_inner(InnerArgs A) {
  extern __shared__ double sm[];  // max(nphi, 4 M + 4 nchunk) doubles
  __shared__ double red[512];
  __shared__ double part[4 * 512];
  __shared__ double s_val;
  __shared__ int s_stop;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5, nw = nthr >> 5;
  const int nphi = A.nphi, nlat = A.nlat, M = A.M, nlm = A.nlm, half = nphi / 2;
  unsigned int gen = 0;
  if (!(A.sc->C_int > 0.0)) return;  // no ocean: nothing to redistribute (every CTA reads the same value)
  // L of the first iteration
  for (int j = blockIdx.x; j < nlat; j += gridDim.x) sle_row_load(A, j, sm, part);
  if (!grid_barrier(A.bar, gen, A.wait_ns)) return bar_fail(A);
  for (int it = 1; it <= A.n_inner; ++it) {
    // A. Legendre analysis (warp per lm, four lm of a warp at once) and the
    //    affine response u, N
    for (int lm0 = blockIdx.x * nw + wid; lm0 < nlm; lm0 += 4 * gridDim.x * nw) {
      constexpr int U4 = 4;
      double re[U4], im[U4];
      int lmv[U4];
      const double* Fm[U4];
      const double* P[U4];
#pragma unroll
      for (int u = 0; u < U4; ++u) {
        lmv[u] = lm0 + u * gridDim.x * nw;
        const int lmc = min(lmv[u], nlm - 1);  // past the end: a valid row, result unused
        Fm[u] = A.F + ((size_t)A.lm_m[lmc] * nlat) * 2;
        P[u] = A.plm + (size_t)lmc * nlat;
        re[u] = 0.0;
        im[u] = 0.0;
      }
      for (int j = lane; j < nlat; j += 32) {
        const double w = A.wts[j];
#pragma unroll
        for (int u = 0; u < U4; ++u) {
          const double wp = w * P[u][j];
          re[u] += wp * Fm[u][2 * j];
          im[u] += wp * Fm[u][2 * j + 1];
        }
      }
#pragma unroll
      for (int u = 0; u < U4; ++u)
        for (int o = 16; o > 0; o >>= 1) {
          re[u] += __shfl_down_sync(0xffffffffu, re[u], o);
          im[u] += __shfl_down_sync(0xffffffffu, im[u], o);
        }
      // lanes 0..3 write lm u (the sums are in lane 0; broadcast them)
#pragma unroll
      for (int u = 0; u < U4; ++u) {
        re[u] = __shfl_sync(0xffffffffu, re[u], 0);
        im[u] = __shfl_sync(0xffffffffu, im[u], 0);
      }
      if (lane < U4) {
        double r = re[0], i2 = im[0];
#pragma unroll
        for (int u = 1; u < U4; ++u)
          if (lane == u) {
            r = re[u];
            i2 = im[u];
          }
        const int lm = lmv[lane];
        if (lm < nlm) {
          A.sigma[2 * lm] = r;
          A.sigma[2 * lm + 1] = i2;
          const int l = A.lm_l[lm];
          double* uu = A.ulm;
          double* n = A.ulm + 2 * (size_t)nlm;
          if (l == 0) {
            uu[2 * lm] = A.gu[0] * r;
            uu[2 * lm + 1] = A.gu[0] * i2;
            n[2 * lm] = A.gn[0] * r;
            n[2 * lm + 1] = A.gn[0] * i2;
          } else {
            const int k = A.lm2k[lm];
            uu[2 * lm] = A.gu[l] * r + A.drift[(size_t)0 * A.nk + k];
            uu[2 * lm + 1] = A.gu[l] * i2 + A.drift[(size_t)1 * A.nk + k];
            n[2 * lm] = A.gn[l] * r - A.drift[(size_t)2 * A.nk + k] / A.g;
            n[2 * lm + 1] = A.gn[l] * i2 - A.drift[(size_t)3 * A.nk + k] / A.g;
          }
        }
      }
    }
    if (!grid_barrier(A.bar, gen, A.wait_ns)) return bar_fail(A);
    // S. Legendre synthesis of u and N in chunks of at most SLE_LCH degrees: a
    //    thread per (chunk, j), partial sums Gp[j][chunk][u re, u im, N re, N im]
    //    (one 32-byte sector per thread; a row's partials contiguous)
    for (int t = blockIdx.x * nthr + tid; t < A.nchunk * nlat; t += gridDim.x * nthr) {
      const int c = t / nlat, j = t % nlat;
      const int2 ch = A.chunk[c];
      const int n = min(SLE_LCH, A.lmax - ch.x + 1 - ch.y);
      const int lm = A.mbeg[ch.x] + ch.y;
      const double* pc = A.plm + (size_t)lm * nlat + j;
      const double* qu = A.ulm + 2 * (size_t)lm;
      const double* qn = A.ulm + 2 * ((size_t)nlm + lm);
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll 4
      for (int q = 0; q < n; ++q) {
        const double p = pc[(size_t)q * nlat];
        a0 += qu[2 * q] * p;
        a1 += qu[2 * q + 1] * p;
        a2 += qn[2 * q] * p;
        a3 += qn[2 * q + 1] * p;
      }
      double* o = A.Gp + ((size_t)j * A.nchunk + c) * 4;
      o[0] = a0;
      o[1] = a1;
      o[2] = a2;
      o[3] = a3;
    }
    if (!grid_barrier(A.bar, gen, A.wait_ns)) return bar_fail(A);
    // R. longitude synthesis (g(i) = G_0 + 2 sum_m Re G_m e^{i m phi_i}, even and
    //    odd m apart, tpi threads per longitude pair (i, i + half)),
    //    Sraw = N - u (+ s_rot), row sums of C Sraw
    for (int j = blockIdx.x; j < nlat; j += gridDim.x) {
      double* Gu = sm;
      double* Gn = sm + 2 * M;
      double* gp = sm + 4 * M;  // the row's partial sums, staged
      __syncthreads();
      for (int t = tid; t < 4 * A.nchunk; t += nthr) gp[t] = A.Gp[(size_t)j * A.nchunk * 4 + t];
      __syncthreads();
      for (int m = tid; m < M; m += nthr) {  // the order's chunks summed in order
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        for (int c = A.cbeg[m]; c < A.cbeg[m + 1]; ++c) {
          const double* o = gp + 4 * c;
          a0 += o[0];
          a1 += o[1];
          a2 += o[2];
          a3 += o[3];
        }
        Gu[2 * m] = a0;
        Gu[2 * m + 1] = a1;
        Gn[2 * m] = a2;
        Gn[2 * m + 1] = a3;
      }
      __syncthreads();
      const int tpi = max(1, min(8, nthr / half));
      double acc = 0.0;
      for (int base = 0; base < half * tpi; base += nthr) {
        const int u = base + tid, i = u / tpi, q = u % tpi;
        const bool act = u < half * tpi;
        double ue = 0.0, uo = 0.0, ne = 0.0, no = 0.0;
        if (act) {
          int t = (i * (1 + q)) % nphi;
          const int step = (i * tpi) % nphi;
          for (int m = 1 + q; m < M; m += tpi) {
            const double c = __ldg(&A.cs[t]), sn = __ldg(&A.sn[t]);
            const double vu = Gu[2 * m] * c - Gu[2 * m + 1] * sn;
            const double vn = Gn[2 * m] * c - Gn[2 * m + 1] * sn;
            if (m & 1) {
              uo += vu;
              no += vn;
            } else {
              ue += vu;
              ne += vn;
            }
            t += step;
            if (t >= nphi) t -= nphi;
          }
        }
        part[tid] = ue;
        part[nthr + tid] = uo;
        part[2 * nthr + tid] = ne;
        part[3 * nthr + tid] = no;
        __syncthreads();
        if (act && q == 0) {
          double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
          for (int c = 0; c < tpi; ++c) {
            a0 += part[tid + c];
            a1 += part[nthr + tid + c];
            a2 += part[2 * nthr + tid + c];
            a3 += part[3 * nthr + tid + c];
          }
          const double u1 = Gu[0] + 2.0 * (a0 + a1), u2 = Gu[0] + 2.0 * (a0 - a1);
          const double n1 = Gn[0] + 2.0 * (a2 + a3), n2 = Gn[0] + 2.0 * (a2 - a3);
          const size_t p1 = (size_t)j * nphi + i, p2 = p1 + half;
          double s1 = n1 - u1, s2 = n2 - u2;
          if (A.srot) {
            s1 = s1 + A.srot[p1];
            s2 = s2 + A.srot[p2];
          }
          A.Sraw[p1] = s1;
          A.Sraw[p2] = s2;
          acc += A.C[p1] * s1 + A.C[p2] * s2;
        }
        __syncthreads();
      }
      acc = block_sum(acc, red);
      if (tid == 0) A.rowpart[RP_CS * nlat + j] = acc;
    }
    if (!grid_barrier(A.bar, gen, A.wait_ns)) return bar_fail(A);
    // U. dphi in every CTA (rows in order by thread 0: the same value everywhere)
    {
      const double Cs = integrate_rows(A.rowpart + RP_CS * nlat, A.wts, nlat, A.dlon);
      if (tid == 0) {
        const double dphi = (A.sc->ice_int - Cs + A.sc->zeta_int) / A.sc->C_int;
        s_val = dphi;
        if (blockIdx.x == 0) {
          A.sc->Cs_int = Cs;
          A.sc->dphi = dphi;
        }
      }
      __syncthreads();
    }
    const double dphi = s_val;
    for (int j = blockIdx.x; j < nlat; j += gridDim.x) {
      double dmax = 0.0, smax = 0.0;
      for (int i = tid; i < nphi; i += nthr) {
        const size_t p = (size_t)j * nphi + i;
        const double rn = A.Sraw[p] + dphi;
        dmax = nanmax(dmax, fabs(A.C[p] * (rn - A.rsl[p])));
        A.rsl[p] = rn;
        smax = nanmax(smax, fabs(A.C[p] * rn));
      }
      dmax = block_max_w(dmax, red);
      smax = block_max_w(smax, red);
      if (tid == 0) {
        A.rowpart[RP_DMAX * nlat + j] = dmax;
        A.rowpart[RP_SMAX * nlat + j] = smax;
      }
      sle_row_load(A, j, sm, part);  // L of the next iteration (unused if this one converged)
    }
    if (!grid_barrier(A.bar, gen, A.wait_ns)) return bar_fail(A);
    // convergence (src/vilma_sle.f90:330-338), the same decision in every CTA
    {
      double dmax = 0.0, smax = 0.0;
      for (int j = tid; j < nlat; j += nthr) {
        dmax = nanmax(dmax, A.rowpart[RP_DMAX * nlat + j]);
        smax = nanmax(smax, A.rowpart[RP_SMAX * nlat + j]);
      }
      dmax = block_max_w(dmax, red);
      smax = block_max_w(smax, red);
      if (tid == 0) {
        s_stop = (dmax <= A.tol * fmax(smax, TINY)) ? 1 : 0;
        if (blockIdx.x == 0) {
          A.sc->dmax = dmax;
          A.sc->smax = smax;
          A.sc->n_inner = it;
        }
      }
      __syncthreads();
      if (s_stop) break;
    }
  }
}

// dynamic shared memory of the fused loop: the row (nphi) or, in R, the
// Fourier sums (4 M) and the row's staged partial sums (4 chunks)
static size_t sle_inner_smem(const vg_handle* h) {
  const Grid& G = h->grid;
  int nch = 0;
  for (int m = 0; m < G.M; ++m) nch += (G.lmax - m + SLE_LCH) / SLE_LCH;
  return (size_t)std::max(G.nphi, 4 * G.M + 4 * nch) * sizeof(double);
}

static void launch_inner_loop(vg_handle* h) {
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  if (h->sle_grid == 0) {
    int dev = 0, nsm = 0, per_sm = 0;
    VG_CUDA(cudaGetDevice(&dev));
    VG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const size_t shm = sle_inner_smem(h);
    raise_smem_limit((const void*)k_sle_inner, shm);
    VG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sle_inner, 512, shm));
    if (per_sm < 1) throw Error("sle_solve: the fused inner loop does not fit on an SM");
    h->sle_grid = h->p.sle_ctas > 0 ? std::min(h->p.sle_ctas, nsm * per_sm) : nsm;
    h->d_gbar.alloc(4);
    std::vector<int2> chunk;
    std::vector<int> cbeg(G.M + 1);
    for (int m = 0; m < G.M; ++m) {
      cbeg[m] = (int)chunk.size();
      for (int l0 = 0; l0 < G.lmax - m + 1; l0 += SLE_LCH) chunk.push_back(make_int2(m, l0));
    }
    cbeg[G.M] = (int)chunk.size();
    h->sle_nchunk = (int)chunk.size();
    h->d_sle_chunk.upload(chunk, s);
    h->d_sle_cbeg.upload(cbeg, s);
    h->d_sle_Gp.alloc((size_t)h->sle_nchunk * G.nlat * 4);
  }
  InnerArgs A;
  A.nphi = G.nphi;
  A.nlat = G.nlat;
  A.M = G.M;
  A.nlm = G.nlm;
  A.nk = h->nk;
  A.lmax = G.lmax;
  A.n_inner = h->p.sle_n_inner;
  A.tol = h->p.sle_tol;
  A.dlon = 2.0 * PI / (double)G.nphi;
  A.g = h->g;
  A.dig = h->d_dig.p;
  A.C = h->d_C.p;
  A.wcorr = h->d_wcorr.p;
  A.cs = G.d_cos.p;
  A.sn = G.d_sin.p;
  A.plm = G.d_plm.p;
  A.wts = G.d_wts.p;
  A.gu = h->d_gu.p;
  A.gn = h->d_gn.p;
  A.drift = h->d_drift.p;
  A.srot = (h->rot_on || h->srot_ext) ? h->d_srot.p : nullptr;
  A.lm_m = G.d_lm_m.p;
  A.lm_l = G.d_lm_l.p;
  A.lm2k = h->d_lm2k.p;
  A.mbeg = G.d_mbeg.p;
  A.rsl = h->d_rsl.p;
  A.F = h->d_F.p;
  A.sigma = h->d_sigma.p;
  A.ulm = h->d_ulm.p;
  A.chunk = h->d_sle_chunk.p;
  A.cbeg = h->d_sle_cbeg.p;
  A.nchunk = h->sle_nchunk;
  A.Gp = h->d_sle_Gp.p;
  A.Sraw = h->d_Sraw.p;
  A.rowpart = h->d_rowpart.p;
  A.sc = h->d_sc_.p;
  A.bar = h->d_gbar.p;
  A.wait_ns = h->wait_ns;
  VG_CUDA(cudaMemsetAsync(h->d_gbar.p, 0, 4 * sizeof(unsigned int), s));
  const size_t shm = sle_inner_smem(h);
  void* args[] = {&A};
  VG_CUDA(cudaLaunchCooperativeKernel((const void*)k_sle_inner, dim3(h->sle_grid), dim3(512), args, shm, s));
  ++h->n_launch;
}

static void read_scalars(vg_handle* h) {
  VG_CUDA(cudaMemcpyAsync(h->h_sc, h->d_sc_.p, sizeof(SleScalars), cudaMemcpyDeviceToHost, h->stream));
  VG_CUDA(cudaStreamSynchronize(h->stream));
}

void sync_scalars(vg_handle* h) { read_scalars(h); }


// One sea-level solve with the memory advance at its end (FE: a single
// co-convergence pass), src/vilma_sle.f90:124-405. Writes the advanced memory
// into the other state buffer; the caller decides to keep or drop it.
void sle_solve_dev(vg_handle* h, double dt, bool report_only) {
  const Grid& G = h->grid;
  const int ng = G.ng, nlat = G.nlat, nphi = G.nphi, M = G.M, nlm = G.nlm;
  const double dlon = 2.0 * PI / (double)nphi;
  cudaStream_t s = h->stream;
  const vg_params& p = h->p;
  SleScalars* sc = h->d_sc_.p;
  double* rp = h->d_rowpart.p;
  const int eb = 256, eg = (ng + eb - 1) / eb;
  if (!p.sle_warm_start) VG_CUDA(cudaMemsetAsync(h->d_rsl.p, 0, ng * sizeof(double), s));
  VG_CUDA(cudaMemsetAsync(h->d_wcorr.p, 0, ng * sizeof(double), s));
  VG_CUDA(cudaMemsetAsync(sc, 0, sizeof(SleScalars), s));
  const bool trap = p.scheme == VG_SCHEME_TRAP && !report_only;
  // response_begin_step. Forward Euler without the toroidal channel: the drift
  // (its degree 1 beside the band sweeps) runs on the second stream while this
  // stream sets up the first pass (ocean function, row integrals: none of the
  // drift's buffers), and is joined before the fused loop reads it.
  bool drift_pending = !trap && !h->tor_on && !h->prof.on;
  if (drift_pending) {
    VG_CUDA(cudaEventRecord(h->ev_dfork, s));
    VG_CUDA(cudaStreamWaitEvent(h->aux, h->ev_dfork, 0));
    launch_drift_on(h, h->cur, nullptr, nullptr, h->aux, h->aux2);
    VG_CUDA(cudaEventRecord(h->ev_djoin, h->aux));
  } else {
    launch_drift(h);
  }
  auto join_drift = [&]() {
    if (drift_pending) VG_CUDA(cudaStreamWaitEvent(s, h->ev_djoin, 0));
    drift_pending = false;
  };
  k_ocean0<<<eg, eb, 0, s>>>(ng, h->d_z_bed_eq.p, h->d_ice_now.p, h->d_dice_now.p, h->d_C0.p); ++h->n_launch;
  // the sea-level <-> memory co-convergence (src/vilma_sle.f90:218-365): one
  // pass for forward Euler; trapezoid endpoint passes until the surface drift
  // settles for the trapezoidal scheme
  if (trap) trap_prepare(h);
  const int n_mem = trap ? std::max(1, p.sle_max_mem_iter) : 1;
  h->n_inner_last = 0;
  h->n_flip_last = 0;
  for (int im = 1; im <= n_mem; ++im) {
  for (int io = 1; io <= p.sle_n_outer; ++io) {
    if (p.sle_fixed_ocean) {
      if (io == 1) VG_CUDA(cudaMemcpyAsync(h->d_C.p, h->d_C0.p, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
    } else if (io == 1) {
      k_ocean<<<eg, eb, 0, s>>>(ng, h->d_z_bed_eq.p, h->d_rsl.p, h->d_ice_now.p, h->d_C.p); ++h->n_launch;
    } else {
      VG_CUDA(cudaMemcpyAsync(h->d_C.p, h->d_C_next.p, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    k_pass_setup<<<nlat, 128, 0, s>>>(nphi, h->d_ice_now.p, h->d_dice_now.p, h->d_C.p, h->d_C0.p, h->d_z_bed_eq.p,
                                      h->d_dig.p, rp, nlat); ++h->n_launch;
    // no host round trip before the inner loop: with no ocean (C_int <= 0) the
    // kernels below return at once and the pass ends after the one read
    k_finalize_pass<<<1, FIN_THREADS, 0, s>>>(sc, rp, G.d_wts.p, nlat, dlon, p.sle_subgrid); ++h->n_launch;
    k_wcorr<<<eg, eb, 0, s>>>(sc, ng, p.sle_subgrid, h->d_z_bed_eq.p, h->d_C.p, h->d_C0.p, h->d_wcorr.p);
    ++h->n_launch;
    join_drift();
    {
      PhaseScope ps(h, VG_PH_SLE);
      launch_inner_loop(h);
    }
    if (!p.sle_fixed_ocean) {  // the coastline test of this pass, read with the loop's scalars
      k_coast<<<nlat, 128, 0, s>>>(nphi, h->d_z_bed_eq.p, h->d_rsl.p, h->d_ice_now.p, h->d_C.p, h->d_C_next.p,
                                   rp, nlat); ++h->n_launch;
      k_flips<<<1, FIN_THREADS, 0, s>>>(sc, rp, nlat); ++h->n_launch;
    }
    read_scalars(h);
    if (h->sle_tape) tape_pass(h, h->h_sc->C_int, h->h_sc->n_inner);
    if (h->h_sc->C_int <= 0.0) break;  // no ocean: nothing to redistribute
    if (h->h_sc->bar_error) throw Error("sle_solve: grid barrier of the fused inner loop timed out");
    h->n_inner_last = h->h_sc->n_inner;
    h->n_outer_last = io;
    if (p.sle_fixed_ocean) break;
    h->n_flip_last = h->h_sc->flips;
    if (h->h_sc->flips == 0) break;
  }
  join_drift();  // (already joined unless the pass loop was empty)
  // closing load, its analysis, and the memory advance (src/vilma_sle.f90:353-358)
  k_load_fourier<<<nlat, 128, nphi * sizeof(double), s>>>(nphi, nlat, M, h->d_dig.p, h->d_C.p, h->d_rsl.p,
                                                          h->d_wcorr.p, G.d_cos.p, G.d_sin.p, h->d_F.p); ++h->n_launch;
  legendre_analysis_dev(h, h->d_F.p, 1, h->d_sigma.p);
  if (report_only) break;
  if (!trap) {
    advance_memory(h, h->d_sigma.p, dt);
    break;
  }
  if (trap_endpoint_pass(h, dt)) break;
  }
  if (trap) trap_finalize(h, dt);
  k_rowsum<<<nlat, 128, 0, s>>>(nphi, h->d_C.p, h->d_rsl.p, rp + RP_MASS * nlat); ++h->n_launch;
  k_mass<<<1, FIN_THREADS, 0, s>>>(sc, rp, G.d_wts.p, nlat, dlon); ++h->n_launch;
}

// solid_earth_update without rotation; d_ice1 is the interval-end ice on the device
void update_dev(vg_handle* h, const double* d_ice1, double dt_yr) {
  const Grid& G = h->grid;
  const int ng = G.ng;
  cudaStream_t s = h->stream;
  const vg_params& p = h->p;
  const double dt = dt_yr * SEC_PER_YEAR;
  const double t0 = h->time_yr * SEC_PER_YEAR, t1 = t0 + dt, span = t1 - t0;
  const int eb = 256, eg = (ng + eb - 1) / eb;
  h->worst_mass_resid = 0.0;
  // rotational feedback: drift frozen at the interval start, s_rot held across
  // the interval from the entering polar motion (src/vilma_coupling.f90:399-405)
  if (h->rot_on) {
    rotation_begin(h);
    rotation_s_rot(h);
  }
  auto mass_resid_read = [&]() {  // from scalars already read
    double ice_int = h->h_sc->ice_int, Cs = h->h_sc->mass_Cs;
    return std::fabs(ice_int) > 0.0 ? std::fabs(Cs - ice_int) / std::fabs(ice_int) : std::fabs(Cs);
  };
  auto mass_resid = [&]() {
    read_scalars(h);
    return mass_resid_read();
  };
  if (span <= 0.0) {
    k_ice_interp<<<eg, eb, 0, s>>>(ng, 0.0, h->d_h_ice.p, h->d_h_ice.p, h->d_h_ice_eq.p, h->d_ice_now.p,
                                   h->d_dice_now.p); ++h->n_launch;
    sle_solve_dev(h, 0.0, true);
    h->worst_mass_resid = mass_resid();
  } else if (p.scheme == VG_SCHEME_TRAP) {
    // implicit branch (src/vilma_timestep.f90:229-307): step doubling around
    // each trial step, accept / reject against rtol, atol; dt_try carried
    // across intervals
    auto solve_at = [&](double t_eval, double dts) {
      k_ice_interp<<<eg, eb, 0, s>>>(ng, (t_eval - t0) / span, h->d_h_ice.p, d_ice1, h->d_h_ice_eq.p,
                                     h->d_ice_now.p, h->d_dice_now.p); ++h->n_launch;
      VG_CUDA(cudaGetLastError());
      h->n_solve++;
      sle_solve_dev(h, dts, false);
      h->worst_mass_resid = std::max(h->worst_mass_resid, mass_resid());
    };
    if (!h->sigma_primed) {  // seed sigma_n: a report-only solve at t0 (:234-241)
      k_ice_interp<<<eg, eb, 0, s>>>(ng, 0.0, h->d_h_ice.p, h->d_h_ice.p, h->d_h_ice_eq.p, h->d_ice_now.p,
                                     h->d_dice_now.p); ++h->n_launch;
      sle_solve_dev(h, 0.0, true);
      trap_prime(h);
    }
    const double ricfac = 3.0, expo = 1.0 / 3.0;  // order 2: 2^p - 1, 1 / (p + 1)
    if (h->dt_try <= 0.0) h->dt_try = span;
    double t = t0;
    int n_acc = 0;
    while (true) {
      if (t >= t1 - 1.0e-9 * span) break;
      const double dts = std::min(h->dt_try, t1 - t);
      const bool at_floor = p.dt_min > 0.0 && dts <= p.dt_min * (1.0 + 1.0e-9);
      VG_CUDA(cudaMemcpyAsync(h->d_rsl_n.p, h->d_rsl.p, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
      trap_save(h);
      solve_at(t + dts, dts);  // coarse
      trap_stash_coarse(h);
      trap_restore(h);
      VG_CUDA(cudaMemcpyAsync(h->d_rsl.p, h->d_rsl_n.p, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
      solve_at(t + 0.5 * dts, 0.5 * dts);  // fine
      solve_at(t + dts, 0.5 * dts);
      double err_inf = 0.0, tau_inf = 0.0;
      trap_coarse_fine_error(h, err_inf, tau_inf);
      const double errsc = (err_inf / ricfac) / (p.atol + p.rtol * tau_inf);
      if (!(errsc <= HUGE_))
        throw Error("vilma_timestep: implicit local-error estimate went non-finite (viscosity too stiff, or the "
                    "state has already diverged)");
      const bool accept = errsc <= 1.0 || at_floor;
      if (accept) {
        t = t + dts;
        h->n_accept++;
        ++n_acc;
        if (at_floor && errsc > 1.0) h->n_floor++;
      } else {
        trap_restore(h);
        VG_CUDA(cudaMemcpyAsync(h->d_rsl.p, h->d_rsl_n.p, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
        h->n_reject++;
      }
      double fac = errsc <= 0.0 ? p.grow_max : p.safety * std::pow(errsc, -expo);
      fac = std::min(p.grow_max, std::max(p.shrink_min, fac));
      h->dt_try = std::min(p.dt_max, std::max(p.dt_min, dts * fac));
      if (h->dt_try <= 1.0e-12 * span)
        throw Error("vilma_timestep: implicit adaptive step collapsed (tolerance unreachable)");
    }
    h->n_sub_last = n_acc;
    h->mem_norm = read_mem_norm(h, h->cur);
  } else {
    double rate = h->max_rate;
    double dt_stab = rate > 0.0 ? p.cfl / rate : span;
    dt_stab = std::min(dt_stab, p.dt_max);
    if (p.dt_min > 0.0) dt_stab = std::max(dt_stab, p.dt_min);
    int n_sub = std::max(1, (int)std::ceil(span / dt_stab - 1.0e-9));
    h->n_sub_last = n_sub;
    double dtc = span / (double)n_sub, t = t0;
    double tau_run = h->mem_norm;
    while (true) {
      if (t >= t1 - 1.0e-9 * span) break;
      dtc = std::min(dtc, t1 - t);
      VG_CUDA(cudaMemcpyAsync(h->d_rsl_n.p, h->d_rsl.p, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
      double tau0 = h->mem_norm;
      double frac = (t + dtc - t0) / span;
      k_ice_interp<<<eg, eb, 0, s>>>(ng, frac, h->d_h_ice.p, d_ice1, h->d_h_ice_eq.p, h->d_ice_now.p,
                                     h->d_dice_now.p); ++h->n_launch;
      VG_CUDA(cudaGetLastError());
      h->n_solve++;
      if (h->sle_tape) tape_attempt_begin(h, frac, dtc);
      sle_solve_dev(h, dtc, false);
      int nxt = 1 - h->cur;
      VG_CUDA(cudaMemcpyAsync(h->h_sc, h->d_sc_.p, sizeof(SleScalars), cudaMemcpyDeviceToHost, s));
      double err_inf = read_mem_norm(h, nxt);  // synchronises: the scalars are in as well
      h->worst_mass_resid = std::max(h->worst_mass_resid, mass_resid_read());
      bool finite = err_inf <= HUGE_;
      double scale = std::max(tau0, tau_run);
      bool accept = scale <= 0.0 ? finite : (finite && err_inf <= p.guard_growth * scale);
      if (h->sle_tape) tape_attempt_end(h, accept);
      if (accept) {
        h->cur = nxt;
        h->mem_norm = err_inf;
        h->time_s += dtc;
        tau_run = std::max(tau_run, err_inf);
        t = t + dtc;
        h->n_accept++;
        dtc = std::min(span / (double)n_sub, 2.0 * dtc);
      } else {
        VG_CUDA(cudaMemcpyAsync(h->d_rsl.p, h->d_rsl_n.p, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
        h->n_reject++;
        dtc = 0.5 * dtc;
        if (dtc <= 1.0e-12 * span)
          throw Error("vilma_timestep: explicit guard sub-step collapsed (viscosity too stiff for FE)");
      }
    }
  }
  // polar motion to the interval end under the converged load (:411-421)
  if (h->rot_on) rotation_advance(h, h->d_sigma.p, span);
  VG_CUDA(cudaMemcpyAsync(h->d_h_ice.p, d_ice1, ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
  k_zbed<<<eg, eb, 0, s>>>(ng, h->d_z_bed_eq.p, h->d_rsl.p, h->d_zbed.p); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  h->time_yr += dt_yr;
  update_bsl(h);
}

// src/vilma_coupling.f90:572-597 update_bsl
void update_bsl(vg_handle* h) {
  const Grid& G = h->grid;
  const int nlat = G.nlat, nphi = G.nphi;
  cudaStream_t s = h->stream;
  double* rp = h->d_rowpart.p;
  k_bsl_rows<<<nlat, 128, 0, s>>>(nphi, h->d_h_ice.p, h->d_h_ice_eq.p, h->d_C.p, h->d_C0.p, rp, nlat); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  std::vector<double> rows((size_t)RP_N * nlat);
  VG_CUDA(cudaMemcpyAsync(rows.data(), rp, rows.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  VG_CUDA(cudaStreamSynchronize(s));
  double dlon = 2.0 * PI / (double)nphi, c_int = 0.0, t_int = 0.0;
  for (int j = 0; j < nlat; ++j) {
    c_int += G.wts[j] * rows[RP_C * nlat + j] * dlon;
    t_int += G.wts[j] * rows[RP_DIG * nlat + j] * dlon;
  }
  h->bsl = c_int > 0.0 ? -(RHO_ICE / RHO_WATER) * t_int / c_int : 0.0;
}

}  // namespace vg
