// Scalar spherical-harmonic transforms on the Gauss grid, batched over fields
// (sht_grid_synthesis / sht_grid_analysis, src/vilma_sht.f90:204-226). The
// Legendre stage is a per-m contraction over the latitude (analysis) or degree
// (synthesis) index against the device table plm[lm][j].
//   F  layout: F[((b*M + m)*nlat + j)*2 + {re,im}]
//   q  layout: q[(b*nlm + lm)*2 + {re,im}]
#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

__global__ void k_fourier_analysis(const double* __restrict__ f, int nphi, int nlat, int M,
                                   const double* __restrict__ cs, const double* __restrict__ sn,
                                   double* __restrict__ F) {
  extern __shared__ double row[];
  int j = blockIdx.x, b = blockIdx.y;
  const double* src = f + ((size_t)b * nlat + j) * nphi;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) row[i] = src[i];
  __syncthreads();
  row_fourier_analysis(row, nphi, M, cs, sn, F + (((size_t)b * M) * nlat + j) * 2, nlat);
}

// one warp per (lm, b): q = sum_j w_j plm[lm][j] F[m][j]
__global__ void k_legendre_analysis(const double* __restrict__ F, int nlat, int M, int nlm, int batch,
                                    const int* __restrict__ lm_m, const double* __restrict__ plm,
                                    const double* __restrict__ wts, double* __restrict__ q) {
  int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (gw >= nlm * batch) return;
  int lm = gw % nlm, b = gw / nlm, m = lm_m[lm];
  const double* Fm = F + (((size_t)b * M + m) * nlat) * 2;
  const double* P = plm + (size_t)lm * nlat;
  double re = 0.0, im = 0.0;
  for (int j = lane; j < nlat; j += 32) {
    double wp = wts[j] * P[j];
    re += wp * Fm[2 * j];
    im += wp * Fm[2 * j + 1];
  }
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  if (lane == 0) {
    q[((size_t)b * nlm + lm) * 2] = re;
    q[((size_t)b * nlm + lm) * 2 + 1] = im;
  }
}

// one thread per (j, m, b): G = sum_l q_lm plm[lm][j]
__global__ void k_legendre_synth(const double* __restrict__ q, int lmax, int nlat, int M, int nlm,
                                 const int* __restrict__ mbeg, const double* __restrict__ plm,
                                 double* __restrict__ G) {
  int j = blockIdx.x * blockDim.x + threadIdx.x, m = blockIdx.y, b = blockIdx.z;
  if (j >= nlat) return;
  int lm0 = mbeg[m];
  const double* qb = q + (size_t)b * nlm * 2;
  double re = 0.0, im = 0.0;
  for (int l = m; l <= lmax; ++l) {
    double p = plm[(size_t)(lm0 + l - m) * nlat + j];
    re += qb[2 * (lm0 + l - m)] * p;
    im += qb[2 * (lm0 + l - m) + 1] * p;
  }
  G[(((size_t)b * M + m) * nlat + j) * 2] = re;
  G[(((size_t)b * M + m) * nlat + j) * 2 + 1] = im;
}

__global__ void k_fourier_synth(const double* __restrict__ G, int nphi, int nlat, int M,
                                const double* __restrict__ cs, const double* __restrict__ sn,
                                double* __restrict__ f) {
  extern __shared__ double Gs[];  // M complex
  int j = blockIdx.x, b = blockIdx.y;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    Gs[2 * m] = G[(((size_t)b * M + m) * nlat + j) * 2];
    Gs[2 * m + 1] = G[(((size_t)b * M + m) * nlat + j) * 2 + 1];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nphi; i += blockDim.x)
    f[((size_t)b * nlat + j) * nphi + i] = row_fourier_synth_at(Gs, M, i, nphi, cs, sn);
}

void fourier_analysis_dev(vg_handle* h, const double* d_f, int batch, double* d_F) {
  const Grid& G = h->grid;
  dim3 grid(G.nlat, batch);
  k_fourier_analysis<<<grid, 128, G.nphi * sizeof(double), h->stream>>>(d_f, G.nphi, G.nlat, G.M, G.d_cos.p,
                                                                         G.d_sin.p, d_F); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}
void legendre_analysis_dev(vg_handle* h, const double* d_F, int batch, double* d_q) {
  const Grid& G = h->grid;
  long long warps = (long long)G.nlm * batch;
  k_legendre_analysis<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, h->stream>>>(
      d_F, G.nlat, G.M, G.nlm, batch, G.d_lm_m.p, G.d_plm.p, G.d_wts.p, d_q); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}
void legendre_synth_dev(vg_handle* h, const double* d_q, int batch, double* d_G) {
  const Grid& G = h->grid;
  dim3 grid((G.nlat + 63) / 64, G.M, batch);
  k_legendre_synth<<<grid, 64, 0, h->stream>>>(d_q, G.lmax, G.nlat, G.M, G.nlm, G.d_mbeg.p, G.d_plm.p, d_G); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}
void fourier_synth_dev(vg_handle* h, const double* d_G, int batch, double* d_f) {
  const Grid& G = h->grid;
  dim3 grid(G.nlat, batch);
  k_fourier_synth<<<grid, 128, 2 * G.M * sizeof(double), h->stream>>>(d_G, G.nphi, G.nlat, G.M, G.d_cos.p,
                                                                       G.d_sin.p, d_f); ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

void sht_analysis_dev(vg_handle* h, const double* d_f, double* d_q, int batch) {
  fourier_analysis_dev(h, d_f, batch, h->d_F.p);
  legendre_analysis_dev(h, h->d_F.p, batch, d_q);
}
void sht_synthesis_dev(vg_handle* h, const double* d_q, double* d_f, int batch) {
  legendre_synth_dev(h, d_q, batch, h->d_Gs.p);
  fourier_synth_dev(h, h->d_Gs.p, batch, d_f);
}

}  // namespace vg
