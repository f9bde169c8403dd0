// Laterally varying viscosity: the pseudo-spectral Maxwell memory advance of
// the genuinely 3-D elements (response_enable_lateral_visc and
// advance_memory_3d, src/vilma_response.f90:994-1053, 1171-1319; the dyadic
// tensor transforms of src/vilma_tensor_sh.f90:168-387).
//
// All 3-D elements and their three radial shape coefficients are batched as
// nf = 3 * ne3d tensor fields f = (element, shape). Per sub-step:
//   gather    X[k][ch][f][ri] = memory + 2 mu strain (the combined synthesis
//             input of tau + 2 mu eps), channel 3 pre-scaled by -l(l+1)
//   synth     per order m, six products over l: P.X0, D.X1, P.X1, P.X2, G.X3,
//             H.X3 -> S[m][j][p][f][ri] (Fourier coefficients at latitude j)
//   lon       per latitude: dyadic Fourier coefficients (rr, rt, rp, tt, pp, tp),
//             inverse DFT to the grid, times -M(theta, phi), forward DFT, the
//             six analysis inputs (RR, RT, m/sin RP, TT+PP, TT-PP, TP)
//   analysis  per order m, the quadrature adjoints: wP, wD, wP, wP, wG, wH
//   scatter   channel normalisations (1, 1/J, -1/(2J), 1/n6) and the increment
//             c += Delta into the next state buffer
// With the toroidal channels carried (lambda 3, 4 as channels 4, 5) the
// gather adds two channels, the synthesis four products (P.X4, D.X4, G.X5,
// H.X5: rt -= i (m/sin) P.X4, rp += D.X4, Z4 = G e_tp - H (e_tt - e_pp)), the
// longitude pass four analysis inputs (RP, m/sin RT, TP, TT - PP) and the
// analysis four quadratures (wD, wP, wG, wH), normalised by 1/J and 1/n4 with
// n4 = n6 / 4 (src/vilma_tensor_sh.f90:168-203, 231-242, 270-322, 360-387).
// G and H are the spin-2 kernels of Z6 written through P and dP/dtheta:
//   G = -2 cot dP - l(l+1) P + 2 m^2/sin^2 P,   H = (m/sin)(dP - cot P)
// so that Sg = sum c G e^{im phi} and Sh = i sum c H e^{im phi}
// (the grid identities of src/vilma_tensor_sh.f90:244-266).
#include <algorithm>
#include <cmath>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

// ------------------------------------------------------------------ tables

// spin-2 synthesis kernels and the quadrature-weighted analysis kernels, [lm][j]
__global__ void k_visc3d_tables(int nlm, int nlat, const int* __restrict__ lm_l, const int* __restrict__ lm_m,
                                const double* __restrict__ plm, const double* __restrict__ dplm,
                                const double* __restrict__ wts, const double* __restrict__ cott,
                                const double* __restrict__ invsin, double* __restrict__ G, double* __restrict__ H,
                                double* __restrict__ wP, double* __restrict__ wD, double* __restrict__ wG,
                                double* __restrict__ wH) {
  int j = blockIdx.x * blockDim.x + threadIdx.x, lm = blockIdx.y;
  if (j >= nlat || lm >= nlm) return;
  double l = lm_l[lm], m = lm_m[lm];
  size_t o = (size_t)lm * nlat + j;
  double P = plm[o], D = dplm[o], ct = cott[j], is = invsin[j], w = wts[j];
  double g = -2.0 * ct * D - l * (l + 1.0) * P + 2.0 * m * m * is * is * P;
  double hh = m * is * (D - ct * P);
  G[o] = g;
  H[o] = hh;
  wP[o] = w * P;
  wD[o] = w * D;
  wG[o] = w * g;
  wH[o] = w * hh;
}

// spin-2 norm per degree: n6(l) = 4 pi sum_j w_j (G^2 + 4 H^2) at the sectoral
// order m = l — the quadrature value of the synthesis-then-adjoint calibration
// of src/vilma_tensor_sh.f90:99-133 (which also uses m = l).
__global__ void k_visc3d_n6(int lmax, int nlat, const int* __restrict__ mbeg, const double* __restrict__ G,
                            const double* __restrict__ H, const double* __restrict__ wts, double* __restrict__ n6) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l > lmax) return;
  if (l < 2) {
    n6[l] = 0.0;
    return;
  }
  int lm = mbeg[l];  // (l, m = l)
  double s = 0.0;
  for (int j = 0; j < nlat; ++j) {
    double g = G[(size_t)lm * nlat + j], hh = H[(size_t)lm * nlat + j];
    s += wts[j] * (g * g + 4.0 * hh * hh);
  }
  n6[l] = 4.0 * PI * s;
}

// ------------------------------------------------------------------ gather

struct V3Args {
  const double* mem;
  double* nxt;
  const double* tmem;  // toroidal memory (tor), current and next buffer
  double* tnxt;
  const double* dWn;   // nodal W drift [ri][node][k] (tor)
  int tor;
  const double* sigma;
  const int *kdeg, *k2lm, *e3d;
  const double *Jr, *xUn, *xVn, *dUn, *dVn, *mu;
  int ne, nr, nk, ne3d, nf, ncf;  // ncf = 2 nf
  double* mnext = nullptr;        // per-slot norms of the next buffer (the scatter folds its maxima in)
  // exact tensor-core path: the largest |X| per (channel, column) over all
  // slots, as double bits (the synthesis operand rows' scale groups)
  unsigned long long* gmax = nullptr;
  int lm_rows = 0;  // exact tensor-core path: X rows in lm order (k2lm) instead of slot order
};

// one thread per (slot k, 3-D element): strain of both histories, 24 values,
// written as X[k][ch][f][ri] (FP64, or FP32 for the tensor-core stages)
// Blocks of 32 slots x 8 3-D elements. The memory and drift are read along
// the slot index (coalesced); the operand rows X[k][ch][f][ri] are written
// through a shared tile [ch][f in block][slot] so that each (slot, channel)
// row's 6 x 8 entries go out as one contiguous run.
constexpr int V3_TK = 32, V3_TE = 8, V3_TC = 6 * V3_TE, V3_TP = V3_TK + 1;  // tile: columns per row, padded slots

template <class T, int NC>
__global__ void __launch_bounds__(256) k_v3_gather(V3Args A, T* __restrict__ X) {
  extern __shared__ unsigned char v3_sm[];
  T* tile = reinterpret_cast<T*>(v3_sm);  // [NC ch][V3_TC][V3_TP]
  const int kx = threadIdx.x, ey = threadIdx.y;
  const int k0 = blockIdx.x * V3_TK, e0 = blockIdx.y * V3_TE;
  const int k = k0 + kx, ei = e0 + ey;
  if (k < A.nk && ei < A.ne3d) {
    const int e = A.e3d[ei], l = A.kdeg[k], lm = A.k2lm[k];
    const double Jr = A.Jr[l], twoMu = 2.0 * A.mu[e];
    const double* xu = A.xUn + (size_t)l * A.nr;
    const double* xv = A.xVn + (size_t)l * A.nr;
    for (int ri = 0; ri < 2; ++ri) {
      const double s = A.sigma[2 * lm + ri];
      const double U0 = s * xu[e] + A.dUn[((size_t)ri * A.nr + e) * A.nk + k];
      const double U1 = s * xu[e + 1] + A.dUn[((size_t)ri * A.nr + e + 1) * A.nk + k];
      const double V0 = s * xv[e] + A.dVn[((size_t)ri * A.nr + e) * A.nk + k];
      const double V1 = s * xv[e + 1] + A.dVn[((size_t)ri * A.nr + e + 1) * A.nk + k];
      double eps[3][4];
      strain_coeffs(U0, U1, V0, V1, Jr, eps[0], eps[1], eps[2]);
#pragma unroll
      for (int s3 = 0; s3 < 3; ++s3)
#pragma unroll
        for (int lam = 0; lam < 4; ++lam) {
          double v = A.mem[mem_idx(s3, ri, e, lam, k, A.ne, A.nk)] + twoMu * eps[s3][lam];
          if (lam == 2) v = -Jr * v;  // trace channel enters the synthesis as -l(l+1) c
          tile[((size_t)lam * V3_TC + ey * 6 + s3 * 2 + ri) * V3_TP + kx] = (T)v;
        }
      if (NC == 6) {  // lambda 3, 4: memory + 2 mu strain of the W drift (no load term)
        const double W0 = A.dWn[((size_t)ri * A.nr + e) * A.nk + k];
        const double W1 = A.dWn[((size_t)ri * A.nr + e + 1) * A.nk + k];
        double et[3][2];
        strain_coeffs_tor(W0, W1, Jr, et[0], et[1], et[2]);
#pragma unroll
        for (int s3 = 0; s3 < 3; ++s3)
#pragma unroll
          for (int lam = 0; lam < 2; ++lam) {
            const double v = A.tmem[tmem_idx(s3, ri, e, lam, k, A.ne, A.nk)] + twoMu * et[s3][lam];
            tile[((size_t)(4 + lam) * V3_TC + ey * 6 + s3 * 2 + ri) * V3_TP + kx] = (T)v;
          }
      }
    }
  }
  __syncthreads();
  const int nkb = min(V3_TK, A.nk - k0), w = 6 * min(V3_TE, A.ne3d - e0);
  if (A.gmax) {  // per (channel, column) of this block: the largest |value| over its slots
    for (int t = threadIdx.y * V3_TK + threadIdx.x; t < NC * w; t += V3_TK * V3_TE) {
      const int lam = t / w, cc = t % w;
      double mx = 0.0;
      for (int kl = 0; kl < nkb; ++kl) mx = fmax(mx, fabs((double)tile[((size_t)lam * V3_TC + cc) * V3_TP + kl]));
      atomic_max_bits(A.gmax + (size_t)lam * A.ncf + 6 * e0 + cc, mx);
    }
  }
  for (int t = threadIdx.y * V3_TK + threadIdx.x; t < nkb * NC * w; t += V3_TK * V3_TE) {
    const int kl = t / (NC * w), rem = t % (NC * w), lam = rem / w, c = rem % w;
    const size_t xr = A.lm_rows ? (size_t)A.k2lm[k0 + kl] : (size_t)(k0 + kl);
    X[(xr * NC + lam) * A.ncf + 6 * e0 + c] = tile[((size_t)lam * V3_TC + c) * V3_TP + kl];
  }
}

template <class T, int NC = 4>
constexpr size_t v3_gather_smem() {
  return (size_t)NC * V3_TC * V3_TP * sizeof(T);
}

// ------------------------------------------------------------------ GEMMs

// Per-order batched FP64 products (the Legendre stage of the tensor transforms).
//   mode 0 (synthesis): C[j][n] = sum_{kk < K_m} T_p[mbeg + kk][j] * X[row(m + kk, m)][col_p + n]
//                       -> S[((m * nlat + j) * np + p) * ncf + n]
//   mode 1 (analysis):  C[i][n] = sum_{j} T_p[mbeg + i][j] * S[((m * nlat + j) * np + p) * ncf + n]
//                       -> R[(row(m + i, m) * np + p) * ncf + n]
// row(l, m) = kbeg[l] + m for l >= 1, the zero row nk for l = 0.
struct GemmArgs {
  int mode, lmax, nlat, nk, ncf;
  int nin;  // synthesis input channels per slot row (4 or 6: the gathered channels; np: per product)
  int np;   // products: 6 (spheroidal) or 10 (with the toroidal channels)
  const int *mbeg, *kbeg;
  const double* T[10];  // per product: table [lm][j]
  int chan[10];         // synthesis: input channel per product
  const double* in;
  double* out;
};

constexpr int GB_M = 64, GB_N = 64, GB_K = 8;

__device__ __forceinline__ int slot_row(const int* kbeg, int l, int m, int nk) { return l >= 1 ? kbeg[l] + m : nk; }

__global__ void __launch_bounds__(256) k_v3_gemm(GemmArgs A) {
  __shared__ double As[GB_K][GB_M + 1];
  __shared__ double Bs[GB_K][GB_N];
  const int m = blockIdx.z / A.np, p = blockIdx.z % A.np;
  const int Km = A.lmax - m + 1;
  const int rows = (A.mode == 0) ? A.nlat : Km;
  const int kdim = (A.mode == 0) ? Km : A.nlat;
  const int r0 = blockIdx.y * GB_M, n0 = blockIdx.x * GB_N;
  if (r0 >= rows) return;
  const double* T = A.T[p];
  const int mb = A.mbeg[m];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads, 4 x 4 outputs each
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int k0 = 0; k0 < kdim; k0 += GB_K) {
    // A tile (rows r0.., k k0..): synthesis T[mb + kk][j = r]; analysis T[mb + r][j = kk]
    for (int t = threadIdx.x; t < GB_K * GB_M; t += 256) {
      int kk = t / GB_M, r = t % GB_M;
      int gr = r0 + r, gk = k0 + kk;
      double v = 0.0;
      if (gr < rows && gk < kdim)
        v = (A.mode == 0) ? T[(size_t)(mb + gk) * A.nlat + gr] : T[(size_t)(mb + gr) * A.nlat + gk];
      As[kk][r] = v;
    }
    for (int t = threadIdx.x; t < GB_K * GB_N; t += 256) {
      int kk = t / GB_N, n = t % GB_N;
      int gk = k0 + kk, gn = n0 + n;
      double v = 0.0;
      if (gk < kdim && gn < A.ncf) {
        if (A.mode == 0) {
          int row = slot_row(A.kbeg, m + gk, m, A.nk);
          v = A.in[(size_t)row * A.nin * A.ncf + (size_t)A.chan[p] * A.ncf + gn];
        } else {
          v = A.in[(((size_t)m * A.nlat + gk) * A.np + p) * A.ncf + gn];
        }
      }
      Bs[kk][n] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GB_K; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[kk][ty + 16 * q];
        b[q] = Bs[kk][tx + 16 * q];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[q][u] += a[q] * b[u];
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int gr = r0 + ty + 16 * q;
    if (gr >= rows) continue;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      int gn = n0 + tx + 16 * u;
      if (gn >= A.ncf) continue;
      if (A.mode == 0)
        A.out[(((size_t)m * A.nlat + gr) * A.np + p) * A.ncf + gn] = acc[q][u];
      else
        A.out[((size_t)slot_row(A.kbeg, m + gr, m, A.nk) * A.np + p) * A.ncf + gn] = acc[q][u];
    }
  }
}

// ------------------------------------------------------------------ longitude

// The longitude transforms of the FP64 path as register-tiled real DFT
// contractions over dense twiddle tables, split by the parity of m
// (phi_{i + half} = phi_i + pi flips the odd orders):
//   synthesis  E(r, i) = sum_{m even} A(r, 2m) cos(m phi_i) - A(r, 2m+1) sin(m phi_i),
//              O(r, i) the same over odd m; g(i) = E + O, g(i + half) = E - O
//   analysis   F(r, m) = sum_{i < half} X_p(r, i) (cos, -sin)(m phi_i) with
//              X_0 = g(i) + g(i + half) for even m, X_1 = g(i) - g(i + half) for odd m
// A thread owns the six dyadic components (rows) of one field at LON_TC
// longitudes or orders, spaced so that a warp's twiddle loads are contiguous.
// Tables: tw[2m + ri][ncg TC] = (cos, -sin)(m phi_i) (zero past half and M),
// twt[p][i][Mq][2] = (cos, -sin)(m phi_i) at m = p + 2 mq (zero past M).
constexpr int LON_TC = 3;

struct LonTables {
  const double* tw;
  const double* twt;
  int M, M2, half, ncg, nmg0, nmg1, Mq;
};

static LonTables lon_tables(const vg_handle* h) {
  const Grid& G = h->grid;
  LonTables T;
  T.tw = h->d_lon_tw.p;
  T.twt = h->d_lon_twt.p;
  T.M = G.M;
  T.M2 = (G.M + 1) & ~1;
  T.half = G.nphi / 2;
  T.ncg = (T.half + LON_TC - 1) / LON_TC;
  T.nmg0 = ((G.M + 1) / 2 + LON_TC - 1) / LON_TC;
  T.nmg1 = (G.M / 2 + LON_TC - 1) / LON_TC;
  T.Mq = std::max(T.nmg0, T.nmg1) * LON_TC;
  return T;
}

static void lon_tables_build(vg_handle* h) {
  const Grid& G = h->grid;
  const LonTables T = lon_tables(h);
  const int nphi = G.nphi, wT = T.ncg * LON_TC;
  std::vector<double> cs(nphi), sn(nphi);
  for (int t = 0; t < nphi; ++t) {  // the grid's twiddles cos/sin(2 pi t / nphi)
    cs[t] = std::cos(2.0 * PI * (double)t / (double)nphi);
    sn[t] = std::sin(2.0 * PI * (double)t / (double)nphi);
  }
  std::vector<double> tw((size_t)2 * T.M2 * wT, 0.0), twt((size_t)2 * T.half * T.Mq * 2, 0.0);
  for (int m = 0; m < G.M; ++m)
    for (int i = 0; i < T.half; ++i) {
      const int t = (int)(((long long)m * i) % nphi);
      tw[(size_t)(2 * m) * wT + i] = cs[t];
      tw[(size_t)(2 * m + 1) * wT + i] = -sn[t];
      const int p = m & 1, mq = m >> 1;
      twt[(((size_t)p * T.half + i) * T.Mq + mq) * 2] = cs[t];
      twt[(((size_t)p * T.half + i) * T.Mq + mq) * 2 + 1] = -sn[t];
    }
  h->d_lon_tw.upload(tw, h->stream);
  h->d_lon_twt.upload(twt, h->stream);
}

__device__ __forceinline__ void lon_cp16(void* dst, const void* src) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void lon_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void lon_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// synthesis tiles over A (shared, [6 nfl][2 M2], row 6 fl + c): for each
// (field fl, longitude i < half) calls epi(fl, i, g(i), g(i + half)) with the
// six components' values
template <class Epi>
__device__ __forceinline__ void lon_synth(const double* __restrict__ A, int nfl, const LonTables& T, Epi epi) {
  const int wA = 2 * T.M2, wT = T.ncg * LON_TC, ntile = nfl * T.ncg;
  for (int tile = threadIdx.x; tile < ntile; tile += blockDim.x) {
    const int fl = tile / T.ncg, cg = tile % T.ncg;
    const double* a = A + (size_t)fl * 6 * wA;
    double e[6][LON_TC], o[6][LON_TC];
#pragma unroll
    for (int c = 0; c < 6; ++c)
#pragma unroll
      for (int t = 0; t < LON_TC; ++t) e[c][t] = o[c][t] = 0.0;
    const double* tp = T.tw + cg;
    for (int m = 0; m < T.M2; m += 2) {
      double tr[LON_TC], ti[LON_TC], ur[LON_TC], ui[LON_TC];
#pragma unroll
      for (int t = 0; t < LON_TC; ++t) {
        tr[t] = __ldg(tp + (size_t)(2 * m) * wT + t * T.ncg);
        ti[t] = __ldg(tp + (size_t)(2 * m + 1) * wT + t * T.ncg);
        ur[t] = __ldg(tp + (size_t)(2 * m + 2) * wT + t * T.ncg);
        ui[t] = __ldg(tp + (size_t)(2 * m + 3) * wT + t * T.ncg);
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const double2 v = *reinterpret_cast<const double2*>(a + (size_t)c * wA + 2 * m);
        const double2 u = *reinterpret_cast<const double2*>(a + (size_t)c * wA + 2 * m + 2);
#pragma unroll
        for (int t = 0; t < LON_TC; ++t) {
          e[c][t] = fma(v.x, tr[t], fma(v.y, ti[t], e[c][t]));
          o[c][t] = fma(u.x, ur[t], fma(u.y, ui[t], o[c][t]));
        }
      }
    }
#pragma unroll
    for (int t = 0; t < LON_TC; ++t) {
      const int i = cg + T.ncg * t;
      if (i >= T.half) continue;
      double g1[6], g2[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        g1[c] = e[c][t] + o[c][t];
        g2[c] = e[c][t] - o[c][t];
      }
      epi(fl, i, g1, g2);
    }
  }
}

// analysis tiles over X (shared, [6 nfl][nphi]: X_0 in [0, half), X_1 in
// [half, nphi)): for each (field fl, order m < M) calls epi(fl, m, re, im)
// with the six components' sums
template <class Epi>
__device__ __forceinline__ void lon_anal(const double* __restrict__ X, int nfl, int nphi, const LonTables& T,
                                         Epi epi) {
  const int n0 = nfl * T.nmg0, ntile = n0 + nfl * T.nmg1;
  for (int tile = threadIdx.x; tile < ntile; tile += blockDim.x) {
    const int p = tile < n0 ? 0 : 1, nmg = p ? T.nmg1 : T.nmg0, tl = p ? tile - n0 : tile;
    const int fl = tl / nmg, mg = tl % nmg;
    const double* x = X + (size_t)fl * 6 * nphi + p * T.half;
    const double2* tp = reinterpret_cast<const double2*>(T.twt) + (size_t)p * T.half * T.Mq + mg;
    double re[6][LON_TC], im[6][LON_TC];
#pragma unroll
    for (int c = 0; c < 6; ++c)
#pragma unroll
      for (int t = 0; t < LON_TC; ++t) re[c][t] = im[c][t] = 0.0;
    for (int i = 0; i < T.half; ++i) {
      double2 w[LON_TC];
#pragma unroll
      for (int t = 0; t < LON_TC; ++t) w[t] = __ldg(tp + (size_t)i * T.Mq + t * nmg);
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const double v = x[(size_t)c * nphi + i];
#pragma unroll
        for (int t = 0; t < LON_TC; ++t) {
          re[c][t] = fma(v, w[t].x, re[c][t]);
          im[c][t] = fma(v, w[t].y, im[c][t]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < LON_TC; ++t) {
      const int m = p + 2 * (mg + nmg * t);
      if (m >= T.M) continue;
      double r6[6], i6[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        r6[c] = re[c][t];
        i6[c] = im[c][t];
      }
      epi(fl, m, r6, i6);
    }
  }
}

// the coefficient region of the toroidal longitude pass: [6 LF][2 M2] for
// the synthesis, [m][10][2 LF] for the analysis inputs
__host__ __device__ __forceinline__ size_t lon_areg(int LF, const LonTables& T) {
  const size_t a6 = (size_t)6 * LF * 2 * T.M2, a10 = (size_t)10 * 2 * LF * T.M;
  return a6 > a10 ? a6 : a10;
}

constexpr int LON_THREADS = 384;
constexpr int LON_LF = 3;  // fields per CTA: one element's three shape coefficients (two CTAs per SM)
constexpr int LON_LF_TOR = 3;  // with the toroidal channels: staged in two halves, two CTAs per SM

// the CTA's slice of the products S[m][j][q][f][ri] (fields f0 .. f0 + nft - 1,
// a contiguous run of 2 nft doubles per (m, q)) to and from shared [m][q][2 nft]
// (16-byte cp.async pieces, all in flight together; ncf and 2 f0 are even)
// products q0 .. q0 + NS - 1 of the NQ per (m, j), staged as [m][q - q0][2 nft]
template <int NQ = 6, int NS = NQ>
__device__ __forceinline__ void stage_in(const double* __restrict__ S, double* __restrict__ X, int nlat, int ncf,
                                         int j, int f0, int nft, int M, int q0 = 0) {
  const int n = M * NS * nft;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int mq = t / nft, c = t % nft;
    lon_cp16(X + (size_t)mq * 2 * nft + 2 * c,
             S + ((size_t)(mq / NS) * nlat + j) * NQ * ncf + (size_t)(q0 + mq % NS) * ncf + 2 * f0 + 2 * c);
  }
  lon_commit();
  lon_wait<0>();
}

template <int NQ = 6>
__device__ __forceinline__ void stage_out(const double* __restrict__ X, double* __restrict__ S, int nlat, int ncf,
                                          int j, int f0, int nft, int M) {
  const int w = 2 * nft, n = M * NQ * w;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int mq = t / w, c = t % w;
    S[((size_t)(mq / NQ) * nlat + j) * NQ * ncf + (size_t)(mq % NQ) * ncf + 2 * f0 + c] = X[t];
  }
}

// One CTA per (latitude j, LF fields). Dyadic Fourier coefficients from the
// six synthesis products, synthesis to the grid, times -M(theta_j, phi_i) of
// the field's element, analysis, and the six analysis inputs, written in place
// over the synthesis products. With gstore set, the grid before -M dt is also
// stored, [j][field][component][i], for the adjoint.
template <int LF, int NQ = 6>
__global__ void __launch_bounds__(LON_THREADS, 1)
    k_v3_lon(double* __restrict__ S, int nlat, int nphi, int nf, double dt, const double* __restrict__ Mk3rate,
             LonTables T, const double* __restrict__ invsin, double* __restrict__ gstore, int trap) {
  extern __shared__ double sm[];
  const int j = blockIdx.x, f0 = blockIdx.y * LF;
  const int nft = min(LF, nf - f0);
  const int ncf = 2 * nf, half = T.half, wA = 2 * T.M2;
  double* A = sm;  // [6 LF][2 M2]; [m][q][2 nft] for the analysis inputs
  double* X = sm + (NQ == 6 ? (size_t)6 * LF * wA : lon_areg(LF, T));  // [6 LF][nphi]; staged products
  const double is = invsin[j];
  // 1. the CTA's synthesis products, staged in X as [m][q][2 nft] (contiguous
  //    runs of 2 nft doubles in S; the spheroidal six, then the toroidal four),
  //    then the dyadic coefficients rr, rt, rp, tt, pp, tp with the synthesis
  //    weights (1 at m = 0, 2 above), zero past M
  stage_in<NQ, 6>(S, X, nlat, ncf, j, f0, nft, T.M);
  __syncthreads();
  for (int t = threadIdx.x; t < nft * T.M2; t += blockDim.x) {
    const int fl = t / T.M2, m = t % T.M2;
    double pr[6][2];
    for (int q = 0; q < 6; ++q)
      for (int ri = 0; ri < 2; ++ri) pr[q][ri] = (m < T.M) ? X[((size_t)m * 6 + q) * 2 * nft + 2 * fl + ri] : 0.0;
    const double ms = m * is, w = (m == 0) ? 1.0 : 2.0;
    const double comp[6][2] = {{pr[0][0], pr[0][1]},
                               {pr[1][0], pr[1][1]},
                               {-ms * pr[2][1], ms * pr[2][0]},             // i (m / sin) P.X1
                               {pr[3][0] + pr[4][0], pr[3][1] + pr[4][1]},  // TT + PP
                               {pr[3][0] - pr[4][0], pr[3][1] - pr[4][1]},  // TT - PP
                               {-4.0 * pr[5][1], 4.0 * pr[5][0]}};          // 4 i H.X3
    for (int c = 0; c < 6; ++c) {
      A[(size_t)(fl * 6 + c) * wA + 2 * m] = w * comp[c][0];
      A[(size_t)(fl * 6 + c) * wA + 2 * m + 1] = w * comp[c][1];
    }
  }
  __syncthreads();
  if (NQ == 10) {  // Z3: (rt, rp) += e_r x grad_1 = (-i (m/sin) P.X4, D.X4); Z4: (tt, pp, tp) += (-Sh, Sh, Sg)
    stage_in<NQ, 4>(S, X, nlat, ncf, j, f0, nft, T.M, 6);
    __syncthreads();
    for (int t = threadIdx.x; t < nft * T.M; t += blockDim.x) {
      const int fl = t / T.M, m = t % T.M;
      double pr[4][2];
      for (int q = 0; q < 4; ++q)
        for (int ri = 0; ri < 2; ++ri) pr[q][ri] = X[((size_t)m * 4 + q) * 2 * nft + 2 * fl + ri];
      const double ms = m * is, w = (m == 0) ? 1.0 : 2.0;
      const double add[6][2] = {{0.0, 0.0},
                                {ms * pr[0][1], -ms * pr[0][0]},  // -i (m/sin) P.X4
                                {pr[1][0], pr[1][1]},             // D.X4
                                {pr[3][1], -pr[3][0]},            // -i H.X5
                                {-pr[3][1], pr[3][0]},            // +i H.X5
                                {pr[2][0], pr[2][1]}};            // G.X5
      for (int c = 1; c < 6; ++c) {
        A[(size_t)(fl * 6 + c) * wA + 2 * m] += w * add[c][0];
        A[(size_t)(fl * 6 + c) * wA + 2 * m + 1] += w * add[c][1];
      }
    }
    __syncthreads();
  }
  // 2. synthesis, times -M dt, and the parity combinations of the analysis
  lon_synth(A, nft, T, [&](int fl, int i, const double* g1, const double* g2) {
    const int f = f0 + fl;
    const double* Mr = Mk3rate + ((size_t)(f / 3) * nlat + j) * nphi;
    double m1 = Mr[i] * dt, m2 = Mr[i + half] * dt;
    if (trap) {  // trapezoidal: M / (1 + M/2) (src/vilma_response.f90:1468-1473)
      m1 = m1 / (1.0 + 0.5 * m1);
      m2 = m2 / (1.0 + 0.5 * m2);
    }
    for (int c = 0; c < 6; ++c) {
      if (gstore) {
        double* gs = gstore + (((size_t)j * nf + f) * 6 + c) * nphi;
        gs[i] = g1[c];
        gs[i + half] = g2[c];
      }
      const double a = -m1 * g1[c], b = -m2 * g2[c];
      X[(size_t)(fl * 6 + c) * nphi + i] = a + b;
      X[(size_t)(fl * 6 + c) * nphi + half + i] = a - b;
    }
  });
  __syncthreads();
  // 3. analysis (F_m = 2 pi / nphi sum_i f_i e^{-i m phi_i}) and the analysis
  //    inputs RR, RT, m/sin RP, TT + PP, TT - PP, TP
  const double scl = 2.0 * PI / (double)nphi;
  lon_anal(X, nft, nphi, T, [&](int fl, int m, const double* re, const double* im) {
    double F[6][2];
    for (int c = 0; c < 6; ++c) {
      F[c][0] = scl * re[c];
      F[c][1] = scl * im[c];
    }
    const double ms = m * is;
    const double out[10][2] = {{F[0][0], F[0][1]},
                               {F[1][0], F[1][1]},
                               {ms * F[2][0], ms * F[2][1]},
                               {F[3][0] + F[4][0], F[3][1] + F[4][1]},
                               {F[3][0] - F[4][0], F[3][1] - F[4][1]},
                               {F[5][0], F[5][1]},
                               {F[2][0], F[2][1]},                      // RP (wD)
                               {ms * F[1][0], ms * F[1][1]},            // m/sin RT (wP)
                               {F[5][0], F[5][1]},                      // TP (wG)
                               {F[3][0] - F[4][0], F[3][1] - F[4][1]}};  // TT - PP (wH)
    for (int q = 0; q < NQ; ++q)
      for (int ri = 0; ri < 2; ++ri) A[((size_t)m * NQ + q) * 2 * nft + 2 * fl + ri] = out[q][ri];
  });
  __syncthreads();
  stage_out<NQ>(A, S, nlat, ncf, j, f0, nft, T.M);
}

// shared memory of the longitude pass (forward: adj = 0) and its transpose;
// nq analysis inputs (10 with the toroidal channels, staged through the
// coefficient region, which then grows to hold them)
static size_t lon_smem(const vg_handle* h, int LF, bool adj, int nq = 6) {
  const LonTables T = lon_tables(h);
  const int nphi = h->grid.nphi;
  const size_t a = nq == 6 ? (size_t)6 * LF * 2 * T.M2 : lon_areg(LF, T);
  return (a + (size_t)6 * LF * nphi + (adj ? (size_t)LF * nphi : 0)) * sizeof(double);
}

static int lon_threads(const vg_handle* h, int LF) {
  const LonTables T = lon_tables(h);
  const int tiles = std::max(LF * T.ncg, LF * (T.nmg0 + T.nmg1));
  return std::min(LON_THREADS, (tiles + 31) / 32 * 32);
}

constexpr size_t LON_SMEM_MAX = 220 * 1024;
static void lon_attributes();  // the longitude kernels' shared-memory limit (defined after the transpose)

static void lon_check(const vg_handle* h) {
  if (lon_smem(h, LON_LF, true) > LON_SMEM_MAX || (h->tor_on && lon_smem(h, LON_LF_TOR, false, 10) > LON_SMEM_MAX))
    throw Error("visc3d: grid too large for the FP64 longitude pass");
}

// ------------------------------------------------------------------ scatter

// Channel normalisations and the increment form c += Delta
// (src/vilma_response.f90:1281-1318): one thread per (slot, 3-D element);
// the block's maxima of |new memory| per slot go into A.mnext.
template <class T, int NQ>
__device__ __forceinline__ double v3_scatter_one(const V3Args& A, const T* __restrict__ R,
                                                 const double* __restrict__ n6, int k, int ei) {
  double amax = 0.0;
  const int e = A.e3d[ei], l = A.kdeg[k];
  const double J = A.Jr[l], nn = n6[l];
  const T* row = R + (size_t)k * NQ * A.ncf;
  for (int s3 = 0; s3 < 3; ++s3) {
    const int f = 3 * ei + s3;
    double q[NQ][2];
#pragma unroll
    for (int p = 0; p < NQ; ++p)
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) q[p][ri] = (double)row[(size_t)p * A.ncf + 2 * f + ri];
    if (NQ == 10) {  // lambda 3: (wD.RP + i wP.(m/sin RT)) / J; lambda 4: (wG.TP / 2 + i wH.(TT - PP)) / n4
      const double n4 = 0.25 * nn;
      double t[2][2];
      t[0][0] = (q[NQ - 4][0] - q[NQ - 3][1]) / J;
      t[0][1] = (q[NQ - 4][1] + q[NQ - 3][0]) / J;
      t[1][0] = n4 != 0.0 ? (0.5 * q[NQ - 2][0] - q[NQ - 1][1]) / n4 : 0.0;
      t[1][1] = n4 != 0.0 ? (0.5 * q[NQ - 2][1] + q[NQ - 1][0]) / n4 : 0.0;
      for (int ri = 0; ri < 2; ++ri)
        for (int lam = 0; lam < 2; ++lam) {
          const size_t idx = tmem_idx(s3, ri, e, lam, k, A.ne, A.nk);
          A.tnxt[idx] = A.tmem[idx] + t[lam][ri];
        }
    }
    double d[4][2];
    d[0][0] = q[0][0];
    d[0][1] = q[0][1];
    d[1][0] = (q[1][0] + q[2][1]) / J;  // (wD.RT - i wP.(m/sin RP)) / J
    d[1][1] = (q[1][1] - q[2][0]) / J;
    d[2][0] = q[3][0] / (-2.0 * J);
    d[2][1] = q[3][1] / (-2.0 * J);
    d[3][0] = nn != 0.0 ? (q[4][0] + 2.0 * q[5][1]) / nn : 0.0;  // (wG.(TT-PP) - 2i wH.TP) / n6
    d[3][1] = nn != 0.0 ? (q[4][1] - 2.0 * q[5][0]) / nn : 0.0;
    for (int ri = 0; ri < 2; ++ri)
      for (int lam = 0; lam < 4; ++lam) {
        size_t idx = mem_idx(s3, ri, e, lam, k, A.ne, A.nk);
        const double v = A.mem[idx] + d[lam][ri];
        A.nxt[idx] = v;
        amax = nanmax(amax, fabs(v));
      }
  }
  return amax;
}

template <class T, int NQ = 6>
__global__ void __launch_bounds__(256) k_v3_scatter(V3Args A, const T* __restrict__ R,
                                                    const double* __restrict__ n6) {
  __shared__ double red[8][33];
  const int k = blockIdx.x * 32 + threadIdx.x, ei = blockIdx.y * 8 + threadIdx.y;
  double amax = 0.0;
  if (k < A.nk && ei < A.ne3d) amax = v3_scatter_one<T, NQ>(A, R, n6, k, ei);
  if (A.mnext) {  // the same in every thread of the block
    red[threadIdx.y][threadIdx.x] = amax;
    __syncthreads();
    if (threadIdx.y == 0 && k < A.nk) {
      double v = red[0][threadIdx.x];
#pragma unroll
      for (int t = 1; t < 8; ++t) v = nanmax(v, red[t][threadIdx.x]);
      atomic_max_bits(reinterpret_cast<unsigned long long*>(A.mnext) + k, v);
    }
  }
}

// the gather tile (the FP64 one is above the default 48 KB)
static void v3_tile_attributes() {
  static std::atomic<bool> done{false};  // set once; concurrent handles may race to it
  if (done) return;
  VG_CUDA(cudaFuncSetAttribute(k_v3_gather<double, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)v3_gather_smem<double>()));
  VG_CUDA(cudaFuncSetAttribute(k_v3_gather<double, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)v3_gather_smem<double, 6>()));
  VG_CUDA(cudaFuncSetAttribute(k_v3_gather<float, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)v3_gather_smem<float>()));
  done = true;
}

// ------------------------------------------------------------------ host

void visc3d_enable(vg_handle* h, const double* pert) {
  const Grid& G = h->grid;
  const int ne = h->ne, ng = G.ng;
  cudaStream_t s = h->stream;
  if (G.nphi % 2 != 0) throw Error("vg_enable_visc3d: the longitude pass needs an even nphi");
  if (h->lat_visc) throw Error("vg_enable_visc3d: lateral viscosity is already enabled for this handle");
  if (h->p.toroidal && h->p.visc3d_precision == VG_VISC3D_SPLIT_TC)
    throw Error("vg_enable_visc3d: the toroidal channels are carried on the FP64 and exact tensor-core 3-D paths "
                "(toroidal = 1 needs visc3d_precision = VG_VISC3D_FP64 or VG_VISC3D_EXACT_TC)");
  // Maxwell-CFL rate: the grid maximum of mu/eta_eff over every Maxwell element
  // (src/vilma_response.f90:1783-1793, MkPerDt3 covers all elements)
  double rate_max = 0.0;
  for (int e = 0; e < ne; ++e) {
    if (h->MkPerDt[e] == 0.0) continue;
    const double* pe = pert + (size_t)e * ng;
    for (int g = 0; g < ng; ++g) rate_max = std::max(rate_max, h->MkPerDt[e] * std::pow(10.0, -pe[g]));
  }
  // classification (src/vilma_response.f90:1024-1046), on the host: setup only
  std::vector<double> rate3;
  h->e3d_h.clear();
  h->pert_mean3d.clear();
  for (int e = 0; e < ne; ++e) {
    h->active1d_h[e] = 1;
    if (h->MkPerDt[e] == 0.0) continue;
    const double* pe = pert + (size_t)e * ng;
    double mx = -1e300, mn = 1e300;
    for (int g = 0; g < ng; ++g) {
      mx = std::max(mx, pe[g]);
      mn = std::min(mn, pe[g]);
    }
    if (mx - mn > h->p.visc3d_tol) {
      h->active1d_h[e] = 0;
      h->e3d_h.push_back(e);
      double sum = 0.0;
      for (int g = 0; g < ng; ++g) sum += pe[g];
      h->pert_mean3d.push_back(sum / (double)ng);  // for the 1-D pre-equilibration of the spin-up
      for (int g = 0; g < ng; ++g) rate3.push_back(h->MkPerDt[e] * std::pow(10.0, -pe[g]));
    } else {
      double sum = 0.0;
      for (int g = 0; g < ng; ++g) sum += pe[g];
      h->MkPerDt[e] = h->MkPerDt[e] * std::pow(10.0, -(sum / (double)ng));
    }
  }
  h->ne3d = (int)h->e3d_h.size();
  h->max_rate = rate_max;
  for (double v : h->MkPerDt) h->max_rate = std::max(h->max_rate, v);
  h->d_MkPerDt.upload(h->MkPerDt, s);
  h->d_active1d.upload(h->active1d_h, s);
  h->lat_visc = true;
  if (h->ne3d == 0) return;
  h->d_e3d.upload(h->e3d_h, s);
  h->d_MkPerDt3.upload(rate3, s);
  // tables
  const size_t tab = (size_t)G.nlm * G.nlat;
  for (DArr<double>* a : {&h->d_G6, &h->d_H6, &h->d_wP, &h->d_wD, &h->d_wG, &h->d_wH}) a->alloc(tab);
  dim3 tg((G.nlat + 63) / 64, G.nlm);
  k_visc3d_tables<<<tg, 64, 0, s>>>(G.nlm, G.nlat, G.d_lm_l.p, G.d_lm_m.p, G.d_plm.p, G.d_dplm.p, G.d_wts.p,
                                    G.d_cott.p, G.d_invsin.p, h->d_G6.p, h->d_H6.p, h->d_wP.p, h->d_wD.p, h->d_wG.p,
                                    h->d_wH.p);
  VG_CUDA(cudaGetLastError());
  h->d_n6.alloc(G.lmax + 1);
  k_visc3d_n6<<<(G.lmax + 64) / 64, 64, 0, s>>>(G.lmax, G.nlat, G.d_mbeg.p, h->d_G6.p, h->d_H6.p, G.d_wts.p,
                                               h->d_n6.p);
  VG_CUDA(cudaGetLastError());
  h->d_kbeg.upload(h->kbeg_h, s);
  VG_CUDA(cudaStreamSynchronize(s));
  // a genuinely 3-D element couples spheroidal and toroidal
  // (src/vilma_response.f90:1048-1052)
  if (h->p.toroidal) toroidal_enable(h);
  if (h->p.visc3d_precision == VG_VISC3D_SPLIT_TC) {
    visc3d_tc_enable(h);
    return;
  }
  if (h->p.visc3d_precision == VG_VISC3D_EXACT_TC) {
    visc3d_oz_enable(h);
    return;
  }
  // work buffers and longitude tables of the FP64 path
  const int nf = 3 * h->ne3d, ncf = 2 * nf, nch = h->tor_on ? 6 : 4, np = h->tor_on ? 10 : 6;
  h->d_X.alloc((size_t)(h->nk + 1) * nch * ncf);
  h->d_Y.alloc((size_t)G.M * G.nlat * np * ncf);
  h->d_dy.alloc((size_t)(h->nk + 1) * np * ncf);
  lon_tables_build(h);
  lon_check(h);  // the grid fits the longitude pass (throws otherwise)
  lon_attributes();
  VG_CUDA(cudaStreamSynchronize(s));
}

void visc3d_advance(vg_handle* h, const double* d_sigma, double dt, const double* dUn, const double* dVn,
                    bool trap, const double* dWn) {
  if (h->ne3d == 0) return;
  PhaseScope ps(h, VG_PH_VISC3D);
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  const int nf = 3 * h->ne3d, ncf = 2 * nf;
  V3Args A;
  A.mem = h->d_mem[h->cur].p;
  A.nxt = h->d_mem[1 - h->cur].p;
  A.tor = h->tor_on ? 1 : 0;
  A.tmem = h->tor_on ? h->d_tmem[h->cur].p : nullptr;
  A.tnxt = h->tor_on ? h->d_tmem[1 - h->cur].p : nullptr;
  A.dWn = h->tor_on ? (dWn ? dWn : h->d_dWn.p) : nullptr;
  A.sigma = d_sigma;
  A.kdeg = h->d_kdeg.p;
  A.k2lm = h->d_k2lm.p;
  A.e3d = h->d_e3d.p;
  A.Jr = h->d_Jr.p;
  A.xUn = h->d_xUn.p;
  A.xVn = h->d_xVn.p;
  A.dUn = dUn ? dUn : h->d_dUn.p;
  A.dVn = dVn ? dVn : h->d_dVn.p;
  A.mu = h->d_mu.p;
  A.ne = h->ne;
  A.nr = h->nr;
  A.nk = h->nk;
  A.ne3d = h->ne3d;
  A.nf = nf;
  A.ncf = ncf;
  A.mnext = h->d_mnorm.p + (size_t)(1 - h->cur) * h->nk;
  dim3 gg((h->nk + 31) / 32, (h->ne3d + 7) / 8);
  v3_tile_attributes();
  if (h->p.visc3d_precision == VG_VISC3D_SPLIT_TC) {
    float *X32 = nullptr, *dy32 = nullptr;
    visc3d_tc_buffers(h, &X32, &dy32);
    {
      PhaseScope pg(h, VG_PH_V3_GATHER);
      k_v3_gather<float, 4><<<gg, dim3(32, 8), v3_gather_smem<float>(), s>>>(A, X32);
      ++h->n_launch;
      VG_CUDA(cudaGetLastError());
    }
    visc3d_tc_run(h, dt, trap);
    PhaseScope pc(h, VG_PH_V3_SCATTER);
    k_v3_scatter<float><<<gg, dim3(32, 8), 0, s>>>(A, dy32, h->d_n6.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
    return;
  }
  if (h->p.visc3d_precision == VG_VISC3D_EXACT_TC) {
    {
      PhaseScope pg(h, VG_PH_V3_GATHER);
      A.gmax = visc3d_oz_gather_max(h);  // zeroes every scale group of the advance
      A.lm_rows = 1;
      if (h->tor_on)
        k_v3_gather<double, 6><<<gg, dim3(32, 8), v3_gather_smem<double, 6>(), s>>>(A, h->d_X.p);
      else
        k_v3_gather<double, 4><<<gg, dim3(32, 8), v3_gather_smem<double>(), s>>>(A, h->d_X.p);
      ++h->n_launch;
      VG_CUDA(cudaGetLastError());
      A.gmax = nullptr;
    }
    visc3d_oz_run(h, dt, trap);
    PhaseScope pc(h, VG_PH_V3_SCATTER);
    if (h->tor_on)
      k_v3_scatter<double, 10><<<gg, dim3(32, 8), 0, s>>>(A, h->d_dy.p, h->d_n6.p);
    else
      k_v3_scatter<double><<<gg, dim3(32, 8), 0, s>>>(A, h->d_dy.p, h->d_n6.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
    return;
  }
  {
    PhaseScope pg(h, VG_PH_V3_GATHER);
    if (h->tor_on)
      k_v3_gather<double, 6><<<gg, dim3(32, 8), v3_gather_smem<double, 6>(), s>>>(A, h->d_X.p);
    else
      k_v3_gather<double, 4><<<gg, dim3(32, 8), v3_gather_smem<double>(), s>>>(A, h->d_X.p);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  // synthesis
  const int np = h->tor_on ? 10 : 6;
  GemmArgs S;
  S.mode = 0;
  S.lmax = G.lmax;
  S.nlat = G.nlat;
  S.nk = h->nk;
  S.ncf = ncf;
  S.nin = h->tor_on ? 6 : 4;
  S.np = np;
  S.mbeg = G.d_mbeg.p;
  S.kbeg = h->d_kbeg.p;
  const double* st[10] = {G.d_plm.p, G.d_dplm.p, G.d_plm.p, G.d_plm.p, h->d_G6.p,
                          h->d_H6.p, G.d_plm.p,  G.d_dplm.p, h->d_G6.p, h->d_H6.p};
  const int sc[10] = {0, 1, 1, 2, 3, 3, 4, 4, 5, 5};
  for (int p = 0; p < np; ++p) {
    S.T[p] = st[p];
    S.chan[p] = sc[p];
  }
  S.in = h->d_X.p;
  S.out = h->d_Y.p;
  dim3 sg((ncf + GB_N - 1) / GB_N, (G.nlat + GB_M - 1) / GB_M, G.M * np);
  {
    PhaseScope pp(h, VG_PH_V3_SYNTH);
    k_v3_gemm<<<sg, 256, 0, s>>>(S);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  // longitude pass
  {
    PhaseScope pp(h, VG_PH_V3_LON_INV);
    const dim3 lg(G.nlat, (nf + LON_LF - 1) / LON_LF);
    if (h->tor_on)
      k_v3_lon<LON_LF_TOR, 10>
          <<<dim3(G.nlat, (nf + LON_LF_TOR - 1) / LON_LF_TOR), lon_threads(h, LON_LF_TOR),
             lon_smem(h, LON_LF_TOR, false, 10), s>>>(h->d_Y.p, G.nlat, G.nphi, nf, dt, h->d_MkPerDt3.p,
                                                      lon_tables(h), G.d_invsin.p, h->v3_gstore, trap ? 1 : 0);
    else
      k_v3_lon<LON_LF><<<lg, lon_threads(h, LON_LF), lon_smem(h, LON_LF, false), s>>>(
          h->d_Y.p, G.nlat, G.nphi, nf, dt, h->d_MkPerDt3.p, lon_tables(h), G.d_invsin.p, h->v3_gstore,
          trap ? 1 : 0);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  // analysis
  GemmArgs Aa = S;
  Aa.mode = 1;
  const double* at[10] = {h->d_wP.p, h->d_wD.p, h->d_wP.p, h->d_wP.p, h->d_wG.p,
                          h->d_wH.p, h->d_wD.p, h->d_wP.p, h->d_wG.p, h->d_wH.p};
  for (int p = 0; p < np; ++p) Aa.T[p] = at[p];
  Aa.in = h->d_Y.p;
  Aa.out = h->d_dy.p;
  dim3 ag((ncf + GB_N - 1) / GB_N, (G.M + GB_M - 1) / GB_M, G.M * np);
  {
    PhaseScope pp(h, VG_PH_V3_ANALYSIS);
    k_v3_gemm<<<ag, 256, 0, s>>>(Aa);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
  PhaseScope pc(h, VG_PH_V3_SCATTER);
  if (h->tor_on)
    k_v3_scatter<double, 10><<<gg, dim3(32, 8), 0, s>>>(A, h->d_dy.p, h->d_n6.p);
  else
    k_v3_scatter<double><<<gg, dim3(32, 8), 0, s>>>(A, h->d_dy.p, h->d_n6.p);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------ adjoint

// scatter^T: the memory adjoint of a 3-D element's increment back to the six
// products' analysis outputs (the normalisations of k_v3_scatter transposed)
// (with the toroidal channels, NQ = 10: also lambda 3, 4's normalisations,
// from the toroidal memory adjoint lam_t)
template <int NQ = 6>
__global__ void __launch_bounds__(256) k_v3_scatter_T(V3Args A, const double* __restrict__ lam,
                                                      const double* __restrict__ n6, double* __restrict__ dyb,
                                                      const double* __restrict__ lam_t) {
  const int k = blockIdx.x * 32 + threadIdx.x, ei = blockIdx.y * 8 + threadIdx.y;
  if (k >= A.nk || ei >= A.ne3d) return;
  const int e = A.e3d[ei], l = A.kdeg[k];
  const double J = A.Jr[l], nn = n6[l];
  double* row = dyb + (size_t)k * NQ * A.ncf;
  for (int s3 = 0; s3 < 3; ++s3) {
    const int f = 3 * ei + s3;
    double L[4][2];
    for (int ri = 0; ri < 2; ++ri)
      for (int lam_ = 0; lam_ < 4; ++lam_) L[lam_][ri] = lam[mem_idx(s3, ri, e, lam_, k, A.ne, A.nk)];
    double q[6][2];
    q[0][0] = L[0][0];
    q[0][1] = L[0][1];
    q[1][0] = L[1][0] / J;
    q[1][1] = L[1][1] / J;
    q[2][0] = -L[1][1] / J;
    q[2][1] = L[1][0] / J;
    q[3][0] = L[2][0] / (-2.0 * J);
    q[3][1] = L[2][1] / (-2.0 * J);
    q[4][0] = nn != 0.0 ? L[3][0] / nn : 0.0;
    q[4][1] = nn != 0.0 ? L[3][1] / nn : 0.0;
    q[5][0] = nn != 0.0 ? -2.0 * L[3][1] / nn : 0.0;
    q[5][1] = nn != 0.0 ? 2.0 * L[3][0] / nn : 0.0;
    for (int p = 0; p < 6; ++p)
      for (int ri = 0; ri < 2; ++ri) row[(size_t)p * A.ncf + 2 * f + ri] = q[p][ri];
    if (NQ == 10) {  // t0 = (q6 - i q7) / J, t1 = (q8 / 2 - i q9) / n4, transposed
      double T[2][2];
      for (int ri = 0; ri < 2; ++ri)
        for (int lam_ = 0; lam_ < 2; ++lam_) T[lam_][ri] = lam_t[tmem_idx(s3, ri, e, lam_, k, A.ne, A.nk)];
      const double n4 = 0.25 * nn;
      const double qt[4][2] = {{T[0][0] / J, T[0][1] / J},
                               {T[0][1] / J, -T[0][0] / J},
                               {n4 != 0.0 ? 0.5 * T[1][0] / n4 : 0.0, n4 != 0.0 ? 0.5 * T[1][1] / n4 : 0.0},
                               {n4 != 0.0 ? T[1][1] / n4 : 0.0, n4 != 0.0 ? -T[1][0] / n4 : 0.0}};
      for (int p = 0; p < 4; ++p)
        for (int ri = 0; ri < 2; ++ri) row[(size_t)(6 + p) * A.ncf + 2 * f + ri] = qt[p][ri];
    }
  }
}

// longitude pass transposed, one CTA per (latitude j, LF fields): the adjoint
// chain on Yb in place: analysis-input combinations^T, analysis^T (a
// synthesis with weights 2 pi / nphi), times -M dt, synthesis^T (an analysis
// with weights 1 at m = 0, 2 above), dyadic components^T; and
// d J / d (M dt)(j, i) += -sum over components and shapes of G_bar g, g the
// forward grid that the forward pass stored in gstore
// With the toroidal channels (NQ = 10) the four more analysis-input adjoints
// join the component adjoints (RP, m/sin RT, TP, TT - PP) and the four
// toroidal products' adjoints come out beside the six.
template <int LF, int NQ = 6>
__global__ void __launch_bounds__(LON_THREADS, 1)
    k_v3_lon_T(const double* __restrict__ gstore, double* __restrict__ Yb, int nlat, int nphi, int nf, double dt,
               const double* __restrict__ Mk3rate, LonTables T, const double* __restrict__ invsin,
               double* __restrict__ gradMdt, double gw) {
  extern __shared__ double sm[];
  const int j = blockIdx.x, f0 = blockIdx.y * LF;
  const int nft = min(LF, nf - f0);
  const int ncf = 2 * nf, half = T.half, wA = 2 * T.M2;
  double* A = sm;  // [6 LF][2 M2] adjoint Fourier coefficients; [m][NQ][2 nft] product adjoints
  double* X = A + (NQ == 6 ? (size_t)6 * LF * wA : lon_areg(LF, T));  // [6 LF][nphi] adjoint grid
  double* P = X + (size_t)6 * LF * nphi;   // [LF][nphi] per-field G_bar . g
  const double is = invsin[j];
  const double scl = 2.0 * PI / (double)nphi;
  // 1. adjoint dyadic Fourier coefficients from the analysis-input adjoints
  //    (staged in X as [m][q][2 nft])
  stage_in<NQ, 6>(Yb, X, nlat, ncf, j, f0, nft, T.M);
  __syncthreads();
  for (int t = threadIdx.x; t < nft * T.M2; t += blockDim.x) {
    const int fl = t / T.M2, m = t % T.M2;
    double o[6][2];
    for (int q = 0; q < 6; ++q)
      for (int ri = 0; ri < 2; ++ri) o[q][ri] = (m < T.M) ? X[((size_t)m * 6 + q) * 2 * nft + 2 * fl + ri] : 0.0;
    const double ms = m * is;
    const double Fb[6][2] = {{o[0][0], o[0][1]},
                             {o[1][0], o[1][1]},
                             {ms * o[2][0], ms * o[2][1]},
                             {o[3][0] + o[4][0], o[3][1] + o[4][1]},
                             {o[3][0] - o[4][0], o[3][1] - o[4][1]},
                             {o[5][0], o[5][1]}};
    for (int c = 0; c < 6; ++c) {
      A[(size_t)(fl * 6 + c) * wA + 2 * m] = scl * Fb[c][0];
      A[(size_t)(fl * 6 + c) * wA + 2 * m + 1] = scl * Fb[c][1];
    }
  }
  __syncthreads();
  if (NQ == 10) {  // out6 = F2 (RP), out7 = ms F1, out8 = F5, out9 = F3 - F4, transposed and added
    stage_in<NQ, 4>(Yb, X, nlat, ncf, j, f0, nft, T.M, 6);
    __syncthreads();
    for (int t = threadIdx.x; t < nft * T.M; t += blockDim.x) {
      const int fl = t / T.M, m = t % T.M;
      double o[4][2];
      for (int q = 0; q < 4; ++q)
        for (int ri = 0; ri < 2; ++ri) o[q][ri] = X[((size_t)m * 4 + q) * 2 * nft + 2 * fl + ri];
      const double ms = m * is;
      const double add[6][2] = {{0.0, 0.0},
                                {ms * o[1][0], ms * o[1][1]},
                                {o[0][0], o[0][1]},
                                {o[3][0], o[3][1]},
                                {-o[3][0], -o[3][1]},
                                {o[2][0], o[2][1]}};
      for (int c = 1; c < 6; ++c) {
        A[(size_t)(fl * 6 + c) * wA + 2 * m] += scl * add[c][0];
        A[(size_t)(fl * 6 + c) * wA + 2 * m + 1] += scl * add[c][1];
      }
    }
    __syncthreads();
  }
  // 2. analysis^T: G_bar(i) = scl sum_m (Fre cos(m phi_i) - Fim sin(m phi_i));
  //    the per-field G_bar . g and g_bar = -M dt G_bar in parity form
  lon_synth(A, nft, T, [&](int fl, int i, const double* b1, const double* b2) {
    const int f = f0 + fl;
    const double* Mr = Mk3rate + ((size_t)(f / 3) * nlat + j) * nphi;
    const double m1 = Mr[i] * dt, m2 = Mr[i + half] * dt;
    double p1 = 0.0, p2 = 0.0;
    for (int c = 0; c < 6; ++c) {
      const double* gs = gstore + (((size_t)j * nf + f) * 6 + c) * nphi;
      p1 += b1[c] * gs[i];
      p2 += b2[c] * gs[i + half];
      const double a = -m1 * b1[c], b = -m2 * b2[c];
      X[(size_t)(fl * 6 + c) * nphi + i] = a + b;
      X[(size_t)(fl * 6 + c) * nphi + half + i] = a - b;
    }
    P[(size_t)fl * nphi + i] = p1;
    P[(size_t)fl * nphi + i + half] = p2;
  });
  __syncthreads();
  // 3. d J / d (M dt) of each element (three shape fields), one CTA per (j, element)
  for (int t = threadIdx.x; t < (nft / 3) * nphi; t += blockDim.x) {
    const int el = t / nphi, i = t % nphi;
    const double acc = P[(size_t)(3 * el) * nphi + i] + P[(size_t)(3 * el + 1) * nphi + i] +
                       P[(size_t)(3 * el + 2) * nphi + i];
    gradMdt[((size_t)(f0 / 3 + el) * nlat + j) * nphi + i] -= gw * acc;
  }
  // 4. synthesis^T: c_bar(m) = w_m sum_i g_bar(i) (cos, -sin)(m phi_i), then
  //    the dyadic components^T into the product adjoints (written over Yb)
  lon_anal(X, nft, nphi, T, [&](int fl, int m, const double* re, const double* im) {
    const double w = (m == 0) ? 1.0 : 2.0;
    double cb[6][2];
    for (int c = 0; c < 6; ++c) {
      cb[c][0] = w * re[c];
      cb[c][1] = (m == 0) ? 0.0 : w * im[c];
    }
    const double ms = m * is;
    const double Sb[6][2] = {{cb[0][0], cb[0][1]},
                             {cb[1][0], cb[1][1]},
                             {ms * cb[2][1], -ms * cb[2][0]},
                             {cb[3][0] + cb[4][0], cb[3][1] + cb[4][1]},
                             {cb[3][0] - cb[4][0], cb[3][1] - cb[4][1]},
                             {4.0 * cb[5][1], -4.0 * cb[5][0]}};
    for (int q = 0; q < 6; ++q)
      for (int ri = 0; ri < 2; ++ri) A[((size_t)m * NQ + q) * 2 * nft + 2 * fl + ri] = Sb[q][ri];
    if (NQ == 10) {  // P.X4 (rt -= i ms), D.X4 (rp), G.X5 (tp), H.X5 (tt -= i, pp += i), transposed
      const double St[4][2] = {{-ms * cb[1][1], ms * cb[1][0]},
                               {cb[2][0], cb[2][1]},
                               {cb[5][0], cb[5][1]},
                               {-cb[3][1] + cb[4][1], cb[3][0] - cb[4][0]}};
      for (int q = 0; q < 4; ++q)
        for (int ri = 0; ri < 2; ++ri) A[((size_t)m * NQ + 6 + q) * 2 * nft + 2 * fl + ri] = St[q][ri];
    }
  });
  __syncthreads();
  stage_out<NQ>(A, Yb, nlat, ncf, j, f0, nft, T.M);
}

// gather^T: the synthesis-input adjoint (per product, combined into the four
// channels) back to the memory (identity of tau + Delta plus G) and to the
// strain, whose transposed coefficients go to the nodal drift adjoints per
// element (E planes: U0, U1, V0, V1, sigma_bar share)
// (with the toroidal channels, NP = 10: channels 4, 5 = P.X4 + D.X4 and
// G.X5 + H.X5 back to the toroidal memory adjoint and, through the toroidal
// strain transposed, to the nodal W adjoint per element, Et planes W0, W1)
template <int NP = 6>
__global__ void __launch_bounds__(256) k_v3_gather_T(V3Args A, const double* __restrict__ Rb,
                                                     const double* __restrict__ lam, double* __restrict__ lam_new,
                                                     double* __restrict__ E, const double* __restrict__ lam_t,
                                                     double* __restrict__ lam_t_new, double* __restrict__ Et) {
  const int k = blockIdx.x * 32 + threadIdx.x, ei = blockIdx.y * 8 + threadIdx.y;
  if (k >= A.nk || ei >= A.ne3d) return;
  const int e = A.e3d[ei], l = A.kdeg[k];
  const double Jr = A.Jr[l], twoMu = 2.0 * A.mu[e];
  const double* xu = A.xUn + (size_t)l * A.nr;
  const double* xv = A.xVn + (size_t)l * A.nr;
  const double* row = Rb + (size_t)k * NP * A.ncf;
  const size_t plane = (size_t)2 * A.ne * A.nk;
  for (int ri = 0; ri < 2; ++ri) {
    if (NP == 10) {  // strain_coeffs_tor transposed: a = -w1 + w2, b = (-w1, w1), c = (-w2, w2)
      double w1 = 0.0, w2 = 0.0;
      for (int s3 = 0; s3 < 3; ++s3) {
        const int n = (3 * ei + s3) * 2 + ri;
        const double xt[2] = {row[(size_t)6 * A.ncf + n] + row[(size_t)7 * A.ncf + n],
                              row[(size_t)8 * A.ncf + n] + row[(size_t)9 * A.ncf + n]};
        double g[2];
        for (int lt = 0; lt < 2; ++lt) {
          const size_t idx = tmem_idx(s3, ri, e, lt, k, A.ne, A.nk);
          lam_t_new[idx] = lam_t[idx] + xt[lt];
          g[lt] = twoMu * xt[lt];
        }
        if (s3 == 0) {  // a[0] = -w1 + w2 (a[1] = 0)
          w1 -= g[0];
          w2 += g[0];
        } else if (s3 == 1) {  // b = (-w1, w1 or 0)
          w1 += -g[0] + (Jr <= 2.0 ? 0.0 : g[1]);
        } else {  // c = (-w2, w2 or 0)
          w2 += -g[0] + (Jr <= 2.0 ? 0.0 : g[1]);
        }
      }
      const size_t at = ((size_t)ri * A.ne + e) * A.nk + k;
      Et[0 * plane + at] = w1;
      Et[1 * plane + at] = w2;
    }
    double eb[3][4];
    for (int s3 = 0; s3 < 3; ++s3) {
      const int n = (3 * ei + s3) * 2 + ri;
      const double x[4] = {row[(size_t)0 * A.ncf + n], row[(size_t)1 * A.ncf + n] + row[(size_t)2 * A.ncf + n],
                           row[(size_t)3 * A.ncf + n], row[(size_t)4 * A.ncf + n] + row[(size_t)5 * A.ncf + n]};
      for (int lam_ = 0; lam_ < 4; ++lam_) {
        const double y = (lam_ == 2) ? -Jr * x[lam_] : x[lam_];
        const size_t idx = mem_idx(s3, ri, e, lam_, k, A.ne, A.nk);
        lam_new[idx] = lam[idx] + y;
        eb[s3][lam_] = twoMu * y;
      }
    }
    const double b3 = (Jr <= 2.0) ? 0.0 : eb[1][3], c3 = (Jr <= 2.0) ? 0.0 : eb[2][3];
    const double u0 = -eb[0][0] + eb[1][1] - eb[1][2] / Jr;
    const double u1 = eb[0][0] + eb[2][1] - eb[2][2] / Jr;
    const double v0 = -eb[0][1] - eb[1][1] + 0.5 * eb[1][2] + 0.5 * b3;
    const double v1 = eb[0][1] - eb[2][1] + 0.5 * eb[2][2] + 0.5 * c3;
    const size_t at = ((size_t)ri * A.ne + e) * A.nk + k;
    E[0 * plane + at] = u0;
    E[1 * plane + at] = u1;
    E[2 * plane + at] = v0;
    E[3 * plane + at] = v1;
    E[4 * plane + at] = u0 * xu[e] + u1 * xu[e + 1] + v0 * xv[e] + v1 * xv[e + 1];
  }
}

static void lon_attributes() {
  for (const void* k :
       {(const void*)k_v3_lon<LON_LF>, (const void*)k_v3_lon<LON_LF_TOR, 10>, (const void*)k_v3_lon_T<LON_LF>,
        (const void*)k_v3_lon_T<LON_LF_TOR, 10>})
    VG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LON_SMEM_MAX));
}

void visc3d_adjoint(vg_handle* h, const double* gstore, double dt, const double* lam, double* lam_new, double* E,
                    double* gradMdt, double gw, const double* lam_t, double* lam_t_new, double* Et) {
  if (h->ne3d == 0) return;
  if (h->p.visc3d_precision != VG_VISC3D_FP64)
    throw Error("vg_misfit_grad: the 3-D adjoint follows the FP64 path (visc3d_precision = FP64)");
  const bool tor = h->tor_on;
  if (tor && !(lam_t && lam_t_new && Et)) throw Error("visc3d_adjoint: the toroidal adjoint buffers are required");
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  const int nf = 3 * h->ne3d, ncf = 2 * nf, np = tor ? 10 : 6;
  const size_t ny = (size_t)G.M * G.nlat * np * ncf, nr6 = (size_t)(h->nk + 1) * np * ncf;
  if (h->d_v3a_Yb.n != ny) {
    h->d_v3a_Yb.alloc(ny);
    h->d_v3a_dyb.alloc(nr6);  // slot row nk (degree 0) stays zero
    h->d_v3a_Rb.alloc(nr6);
  }
  V3Args A;
  A.mem = h->d_mem[h->cur].p;
  A.nxt = nullptr;
  A.sigma = nullptr;
  A.tor = tor ? 1 : 0;
  A.tmem = nullptr;
  A.tnxt = nullptr;
  A.dWn = nullptr;
  A.kdeg = h->d_kdeg.p;
  A.k2lm = h->d_k2lm.p;
  A.e3d = h->d_e3d.p;
  A.Jr = h->d_Jr.p;
  A.xUn = h->d_xUn.p;
  A.xVn = h->d_xVn.p;
  A.dUn = h->d_dUn.p;
  A.dVn = h->d_dVn.p;
  A.mu = h->d_mu.p;
  A.ne = h->ne;
  A.nr = h->nr;
  A.nk = h->nk;
  A.ne3d = h->ne3d;
  A.nf = nf;
  A.ncf = ncf;
  dim3 gg((h->nk + 31) / 32, (h->ne3d + 7) / 8);
  GemmArgs S;
  S.mode = 0;
  S.lmax = G.lmax;
  S.nlat = G.nlat;
  S.nk = h->nk;
  S.ncf = ncf;
  S.nin = tor ? 6 : 4;
  S.np = np;
  S.mbeg = G.d_mbeg.p;
  S.kbeg = h->d_kbeg.p;
  const double* st[10] = {G.d_plm.p, G.d_dplm.p, G.d_plm.p, G.d_plm.p, h->d_G6.p,
                          h->d_H6.p, G.d_plm.p,  G.d_dplm.p, h->d_G6.p, h->d_H6.p};
  const double* at[10] = {h->d_wP.p, h->d_wD.p, h->d_wP.p, h->d_wP.p, h->d_wG.p,
                          h->d_wH.p, h->d_wD.p, h->d_wP.p, h->d_wG.p, h->d_wH.p};
  const int sc[10] = {0, 1, 1, 2, 3, 3, 4, 4, 5, 5};
  for (int p = 0; p < np; ++p) {
    S.T[p] = st[p];
    S.chan[p] = sc[p];
  }
  dim3 sgrid((ncf + GB_N - 1) / GB_N, (G.nlat + GB_M - 1) / GB_M, G.M * np);
  // adjoint chain
  if (tor)
    k_v3_scatter_T<10><<<gg, dim3(32, 8), 0, s>>>(A, lam, h->d_n6.p, h->d_v3a_dyb.p, lam_t);
  else
    k_v3_scatter_T<6><<<gg, dim3(32, 8), 0, s>>>(A, lam, h->d_n6.p, h->d_v3a_dyb.p, nullptr);
  GemmArgs Ab = S;  // analysis^T: the weighted tables, per-product input rows
  Ab.nin = np;
  for (int p = 0; p < np; ++p) {
    Ab.T[p] = at[p];
    Ab.chan[p] = p;
  }
  Ab.in = h->d_v3a_dyb.p;
  Ab.out = h->d_v3a_Yb.p;
  k_v3_gemm<<<sgrid, 256, 0, s>>>(Ab);
  if (tor) {
    const dim3 lg(G.nlat, (nf + LON_LF_TOR - 1) / LON_LF_TOR);
    k_v3_lon_T<LON_LF_TOR, 10><<<lg, lon_threads(h, LON_LF_TOR), lon_smem(h, LON_LF_TOR, true, 10), s>>>(
        gstore, h->d_v3a_Yb.p, G.nlat, G.nphi, nf, dt, h->d_MkPerDt3.p, lon_tables(h), G.d_invsin.p, gradMdt, gw);
  } else {
    const dim3 lg(G.nlat, (nf + LON_LF - 1) / LON_LF);
    k_v3_lon_T<LON_LF><<<lg, lon_threads(h, LON_LF), lon_smem(h, LON_LF, true), s>>>(
        gstore, h->d_v3a_Yb.p, G.nlat, G.nphi, nf, dt, h->d_MkPerDt3.p, lon_tables(h), G.d_invsin.p, gradMdt, gw);
  }
  GemmArgs Sb = S;  // synthesis^T: the unweighted tables, per product out
  Sb.mode = 1;
  Sb.in = h->d_v3a_Yb.p;
  Sb.out = h->d_v3a_Rb.p;
  dim3 agrid((ncf + GB_N - 1) / GB_N, (G.M + GB_M - 1) / GB_M, G.M * np);
  k_v3_gemm<<<agrid, 256, 0, s>>>(Sb);
  if (tor)
    k_v3_gather_T<10><<<gg, dim3(32, 8), 0, s>>>(A, h->d_v3a_Rb.p, lam, lam_new, E, lam_t, lam_t_new, Et);
  else
    k_v3_gather_T<6><<<gg, dim3(32, 8), 0, s>>>(A, h->d_v3a_Rb.p, lam, lam_new, E, nullptr, nullptr, nullptr);
  h->n_launch += 5;
  VG_CUDA(cudaGetLastError());
}

}  // namespace vg
