// Rotational feedback (true polar wander) on the device: vilma_rotation
// (src/vilma_rotation.f90), coupled at the interval level as
// solid_earth_update does (src/vilma_coupling.f90:399-424).
//
// Two degree-2 viscoelastic channels carry the Liouville convolutions as
// Maxwell memory: the LOAD channel (forced by the rigid (2,1) inertia of the
// surface load) and the TIDAL channel (forced by the centrifugal potential of
// the polar motion m). Both use the response's own degree-2 band factor (same
// earth, same mesh: the operator radial_operator_assemble builds for j = 2);
// only their right-hand sides differ (load_rhs / tidal_rhs,
// src/vilma_radial_fe.f90:616-645). Per interval:
//   begin   freeze both channels' drift from the entering memory (dF, dU,
//           nodal strain drift): the dissipative right-hand side of each
//           (channel, re/im) and a band solve (k_rot_elem, k_rot_begin)
//   s_rot   the rotational sea-level term N_rot - u_rot on the Gauss grid from
//           the entering m, held across the interval and added in the
//           sea-level equation
//   advance after the stepper: the converged load is synthesised, its rigid
//           inertia integrated, and the polar motion advanced in sub-steps of at
//           most dt_fe_max (begin, algebraic Liouville solve, forward-Euler
//           commit of both channels' memory).
// Everything is O(ne) or one grid pass; the scalars stay on the device.
#include <algorithm>
#include <cmath>

#include "vg_device.cuh"
#include "vg_internal.cuh"

namespace vg {

// scalar slots of d_rot_sc
enum { RS_DF_LOAD = 0, RS_DU_LOAD = 2, RS_DF_TID = 4, RS_DU_TID = 6, RS_M = 8, RS_CLOAD = 10, RS_N = 12 };

struct RotArgs {
  int ne, nr, nd, nlat, nphi;
  const double *r, *mu, *mkdt, *x;    // x: unit responses [ch][U, V][nr]
  const double *sa, *sb, *sc, *nrm;  // degree-2 strain constants (16, 16, 16, 4)
  const double *ab, *dr, *dc;        // degree-2 band factor (equilibrated)
  const int* ipiv;
  double *mem, *dn, *scal, *f, *fl;  // fl: element contributions [4][ne][4]
};

// channel_begin of both channels (src/vilma_rotation.f90:442-463): the
// dissipative right-hand side of each (channel, re/im) in the reference's
// element order (src/vilma_viscoelastic.f90:441-480), then the equilibrated
// band solve (src/vilma_radial_fe.f90:578-605), in two kernels:
//   k_rot_elem   one thread per (channel, re/im, element): the element's
//                contributions to its four test dofs (two Gauss points, the
//                FP64 divisions of the strain constants), into A.fl
//   k_rot_begin  one block: the nodal forcing of the four right-hand sides
//                (node n: element n-1's second test dof, then element n's
//                first, as the serial loop adds them) times the row scales,
//                the degree-2 band factor and its pivots staged in shared
//                memory when they fit (rot_smem below), one thread per
//                right-hand side for the sequential sweeps with their active
//                window in registers (band_solve_window), then the column
//                scales and the outputs.
// The arithmetic and its order are the reference's throughout.
constexpr int ROT_THREADS = 256;
constexpr int ROT_ELEM_THREADS = 64;

__global__ void __launch_bounds__(ROT_ELEM_THREADS) k_rot_elem(RotArgs A) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const int ne = A.ne;
  if (w >= 4 * ne) return;
  const double xg = 0.5773502691896257;
  const int q = w / ne, e = w % ne, ch = q >> 1, ri = q & 1;
  const double* mem = A.mem + (size_t)ch * 6 * ne * 4;
  const double* Am = mem + (size_t)(0 * 2 + ri) * ne * 4;
  const double* Bm = mem + (size_t)(1 * 2 + ri) * ne * 4;
  const double* Cm = mem + (size_t)(2 * 2 + ri) * ne * 4;
  const double rk = A.r[e], rk1 = A.r[e + 1], h = rk1 - rk;
  double floc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int ig = 0; ig < 2; ++ig) {
    const double gp = ig == 0 ? -xg : xg;
    const double ra = 0.5 * (h * gp + rk + rk1);
    const double psik = (rk1 - ra) / h, psik1 = (ra - rk) / h;
    double tauV[4];
    for (int m = 0; m < 4; ++m) tauV[m] = Am[e * 4 + m] / h + Bm[e * 4 + m] * psik / ra + Cm[e * 4 + m] * psik1 / ra;
    for (int tt = 0; tt < 4; ++tt) {
      double D = 0.0;
      for (int m = 0; m < 4; ++m) {
        const double deps = A.sa[tt * 4 + m] / h + A.sb[tt * 4 + m] * psik / ra + A.sc[tt * 4 + m] * psik1 / ra;
        D = D + A.nrm[m] * tauV[m] * deps;
      }
      floc[tt] = floc[tt] - D * ra * ra * h * 0.5;
    }
  }
  for (int tt = 0; tt < 4; ++tt) A.fl[((size_t)q * ne + e) * 4 + tt] = floc[tt];
}

__global__ void __launch_bounds__(ROT_THREADS) k_rot_begin(RotArgs A, int staged) {
  extern __shared__ double rsm[];
  const int t = threadIdx.x;
  const int ne = A.ne, nr = A.nr, nd = A.nd;
  const double* sfl = A.fl;  // [4][ne][4] element contributions
  const double* ab = A.ab;
  const int* ipiv = A.ipiv;
  double* fbase = A.f;
  if (staged) {
    double* sab = rsm;                                       // [nd][VG_LDAB]
    double* sf = sab + (size_t)nd * VG_LDAB;                 // [4][nd]
    int* sip = reinterpret_cast<int*>(sf + (size_t)4 * nd);  // [nd]
    for (int i = t; i < nd * VG_LDAB; i += blockDim.x) sab[i] = A.ab[i];
    for (int i = t; i < nd; i += blockDim.x) sip[i] = A.ipiv[i];
    ab = sab;
    ipiv = sip;
    fbase = sf;
  }
  __syncthreads();
  // the nodal forcing of the four right-hand sides times the row scales
  for (int w = t; w < 4 * nd; w += blockDim.x) {
    const int q = w / nd, i = w % nd, n = i >> 2, c = i & 3;
    const double* fl = sfl + (size_t)q * ne * 4;
    double u = 0.0;
    if (c < 2 && n < nr) {
      if (n >= 1) u += fl[(n - 1) * 4 + (c == 0 ? 1 : 3)];
      if (n < ne) u += fl[n * 4 + (c == 0 ? 0 : 2)];
    }
    fbase[(size_t)q * nd + i] = A.dr[i] * u;
  }
  __syncthreads();
  if (t < 4) band_solve_window<6, 12>(ab, VG_LDAB, nd, ipiv, fbase + (size_t)t * nd);
  __syncthreads();
  for (int w = t; w < 4 * nd; w += blockDim.x) {
    const int i = w % nd;
    fbase[w] = A.dc[i] * fbase[w];
  }
  __syncthreads();
  if (t < 4) {
    const int ch = t >> 1, ri = t & 1;
    const double* f = fbase + (size_t)t * nd;
    const int base = ch == 0 ? RS_DF_LOAD : RS_DF_TID;
    A.scal[base + ri] = f[4 * (nr - 1) + 2];  // dF
    A.scal[base + 2 + ri] = f[4 * (nr - 1)];  // dU
  }
  for (int w = t; w < 4 * nr; w += blockDim.x) {
    const int q = w / nr, node = w % nr, ch = q >> 1, ri = q & 1;
    const double* f = fbase + (size_t)q * nd;
    double* dn = A.dn + (size_t)ch * 4 * nr;
    dn[(size_t)(0 + ri) * nr + node] = f[4 * node];      // dUn
    dn[(size_t)(2 + ri) * nr + node] = f[4 * node + 1];  // dVn
  }
}

// s_rot = N_rot - u_rot (src/vilma_rotation.f90:192-222) from the current m and
// the tidal channel's frozen drift
__global__ void k_rot_srot(int nlat, int nphi, const double* __restrict__ scal, const double* __restrict__ geo,
                           double kTe, double Ue_t, double kN, double ku, double* __restrict__ srot) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nlat * nphi) return;
  const int j = idx / nphi, i = idx % nphi;
  const double mr = scal[RS_M], mi = scal[RS_M + 1];
  const double cNr = mr + (kTe * mr - scal[RS_DF_TID]), cNi = mi + (kTe * mi - scal[RS_DF_TID + 1]);
  const double cUr = Ue_t * mr + scal[RS_DU_TID], cUi = Ue_t * mi + scal[RS_DU_TID + 1];
  const double gam = geo[j], cphi = geo[nlat + i], sphi = geo[nlat + nphi + i];
  srot[idx] = gam * (kN * (cNr * cphi + cNi * sphi) - ku * (cUr * cphi + cUi * sphi));
}

// per-row sums of the rigid-inertia integrands load sin(theta)cos(theta) (cos phi, sin phi)
__global__ void k_rot_rows(int nlat, int nphi, const double* __restrict__ load, const double* __restrict__ geo,
                           double* __restrict__ rows) {
  __shared__ double red[128];
  const int j = blockIdx.x;
  const double sc2 = geo[j];
  double s13 = 0.0, s23 = 0.0;
  for (int i = threadIdx.x; i < nphi; i += blockDim.x) {
    const double v = load[(size_t)j * nphi + i] * sc2;
    s13 += v * geo[nlat + i];
    s23 += v * geo[nlat + nphi + i];
  }
  s13 = block_sum(s13, red);
  s23 = block_sum(s23, red);
  if (threadIdx.x == 0) {
    rows[j] = s13;
    rows[nlat + j] = s23;
  }
}

struct SolveArgs {
  int nlat;
  double dlon, a4, scl, Fe_load, CminusA, k_s, kTe, dt;
  const double* w;  // Gauss weights
  const double* rows;
};

// rotation_solve_m + rotation_commit (src/vilma_rotation.f90:170-190, 224-233):
// the rigid inertia from the row sums (in row order), the algebraic Liouville
// solve for m, then the forward-Euler memory commit of both channels with
// (cload, m): one thread per (channel, re/im, element).
__global__ void k_rot_solve_commit(RotArgs A, SolveArgs S) {
  __shared__ double s_c[4];  // cload re, im, m re, im
  if (threadIdx.x == 0) {
    double i13 = 0.0, i23 = 0.0;
    for (int j = 0; j < S.nlat; ++j) {
      i13 += S.w[j] * S.rows[j] * S.dlon;
      i23 += S.w[j] * S.rows[S.nlat + j] * S.dlon;
    }
    const double Ir = -S.a4 * i13, Ii = -S.a4 * i23;
    const double clr = Ir * S.scl, cli = Ii * S.scl;
    const double Itr = -(S.Fe_load * clr + A.scal[RS_DF_LOAD]), Iti = -(S.Fe_load * cli + A.scal[RS_DF_LOAD + 1]);
    const double pr = Itr / S.CminusA, pi = Iti / S.CminusA;
    const double den = 1.0 - S.kTe / S.k_s;
    const double mr = (pr - A.scal[RS_DF_TID] / S.k_s) / den, mi = (pi - A.scal[RS_DF_TID + 1] / S.k_s) / den;
    A.scal[RS_CLOAD] = clr;
    A.scal[RS_CLOAD + 1] = cli;
    A.scal[RS_M] = mr;
    A.scal[RS_M + 1] = mi;
    s_c[0] = clr;
    s_c[1] = cli;
    s_c[2] = mr;
    s_c[3] = mi;
  }
  __syncthreads();
  const int ne = A.ne, nr = A.nr;
  for (int t = threadIdx.x; t < 4 * ne; t += blockDim.x) {
    const int ch = t / (2 * ne), ri = (t / ne) & 1, e = t % ne;
    const double c = s_c[ch * 2 + ri];
    const double* xU = A.x + (size_t)(ch * 2 + 0) * nr;
    const double* xV = A.x + (size_t)(ch * 2 + 1) * nr;
    const double* dn = A.dn + (size_t)ch * 4 * nr;
    const double U0 = c * xU[e] + dn[(size_t)(0 + ri) * nr + e], U1 = c * xU[e + 1] + dn[(size_t)(0 + ri) * nr + e + 1];
    const double V0 = c * xV[e] + dn[(size_t)(2 + ri) * nr + e], V1 = c * xV[e + 1] + dn[(size_t)(2 + ri) * nr + e + 1];
    double a[4], b[4], cc[4];
    strain_coeffs(U0, U1, V0, V1, 6.0, a, b, cc);
    const double Me = A.mkdt[e] * S.dt;
    const double om = 1.0 - Me, two_muM = 2.0 * A.mu[e] * Me;
    double* mem = A.mem + (size_t)ch * 6 * ne * 4;
    double* Am = mem + (size_t)(0 * 2 + ri) * ne * 4 + e * 4;
    double* Bm = mem + (size_t)(1 * 2 + ri) * ne * 4 + e * 4;
    double* Cm = mem + (size_t)(2 * 2 + ri) * ne * 4 + e * 4;
    for (int m = 0; m < 4; ++m) {
      Am[m] = om * Am[m] - two_muM * a[m];
      Bm[m] = om * Bm[m] - two_muM * b[m];
      Cm[m] = om * Cm[m] - two_muM * cc[m];
    }
  }
}

// unit responses of both channels on the response's degree-2 factor (load,
// tidal), and the tidal response of the fluidised earth (k^T_f)
__global__ void k_rot_unit(int nr, int nd, double r_earth, double g_surf, const double* __restrict__ ab,
                           const double* __restrict__ dr, const double* __restrict__ dc, const int* __restrict__ ipiv,
                           const double* __restrict__ abf, const double* __restrict__ drf,
                           const double* __restrict__ dcf, const int* __restrict__ ipivf, double* __restrict__ work,
                           double* __restrict__ xout, double* __restrict__ surf) {
  const int t = threadIdx.x;
  if (t >= 3) return;
  const bool fluid = t == 2;
  const double* A_ = fluid ? abf : ab;
  const double* R_ = fluid ? drf : dr;
  const double* C_ = fluid ? dcf : dc;
  const int* P_ = fluid ? ipivf : ipiv;
  double* x = work + (size_t)t * nd;
  for (int i = 0; i < nd; ++i) x[i] = 0.0;
  const int fs = 4 * (nr - 1) + 2, us = 4 * (nr - 1);
  if (t == 0) {  // load_rhs, sigma = 1
    x[us] = -r_earth * r_earth * 1.0 * g_surf;
    x[fs] = -r_earth * r_earth * 1.0;
  } else {  // tidal_rhs, phi_t = 1, degree 2
    x[fs] = -r_earth / (4.0 * PI * GRAV_G) * 5.0 * 1.0;
  }
  for (int i = 0; i < nd; ++i) x[i] = R_[i] * x[i];
  band_solve_strided(A_, VG_LDAB, nd, 6, 12, P_, x, 1);
  for (int i = 0; i < nd; ++i) x[i] = C_[i] * x[i];
  surf[t * 2 + 0] = x[fs];  // F(a)
  surf[t * 2 + 1] = x[us];  // U(a)
  if (!fluid)
    for (int node = 0; node < nr; ++node) {
      xout[(size_t)(t * 2 + 0) * nr + node] = x[4 * node];
      xout[(size_t)(t * 2 + 1) * nr + node] = x[4 * node + 1];
    }
}

static RotArgs rot_args(vg_handle* h) {
  RotArgs A;
  A.ne = h->ne;
  A.nr = h->nr;
  A.nd = h->ndof;
  A.nlat = h->grid.nlat;
  A.nphi = h->grid.nphi;
  A.r = h->d_r.p;
  A.mu = h->d_mu.p;
  A.mkdt = h->d_rot_mkdt.p;
  A.x = h->d_rot_x.p;
  A.sa = h->d_sa.p + 2 * 16;
  A.sb = h->d_sb.p + 2 * 16;
  A.sc = h->d_sc.p + 2 * 16;
  A.nrm = h->d_nrmc.p + 2 * 4;
  A.ab = h->d_ab.p;  // degree 2 is the first band record
  A.dr = h->d_dr.p;
  A.dc = h->d_dc.p;
  A.ipiv = h->d_ipiv.p;
  A.mem = h->d_rot_mem.p;
  A.dn = h->d_rot_dn.p;
  A.scal = h->d_rot_sc.p;
  A.f = h->d_rot_f.p;
  A.fl = h->d_rot_fl.p;
  return A;
}

// rotation_init (src/vilma_rotation.f90:114-152): channels, elastic tidal Love
// numbers, the secular k_s = k^T_f, the stability ceiling; memory and m zero.
void rotation_setup(vg_handle* h) {
  const vg_params& p = h->p;
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  const int ne = h->ne, nr = h->nr, nd = h->ndof;
  std::vector<double> mkdt(ne, 0.0);
  double mx = 0.0;
  for (int e = 0; e < ne; ++e) {
    const int L = h->elem_layer[e];
    mkdt[e] = p.eta[L] > 0.0 ? p.mu[L] / p.eta[L] : 0.0;  // channel_init: mu / eta whenever eta > 0
    mx = std::max(mx, mkdt[e]);
  }
  h->rot_dt_fe_max = mx > 0.0 ? 1.0 / mx : HUGE_VAL;
  h->d_rot_mkdt.upload(mkdt, s);
  h->d_rot_x.alloc((size_t)4 * nr);
  h->d_rot_mem.alloc((size_t)2 * 6 * ne * 4);
  h->d_rot_dn.alloc((size_t)2 * 4 * nr);
  h->d_rot_sc.alloc(RS_N);
  h->d_rot_f.alloc((size_t)4 * nd);
  h->d_rot_fl.alloc((size_t)16 * ne);
  h->d_rot_rows.alloc((size_t)2 * G.nlat);
  h->d_srot.alloc(G.ng);
  h->d_rot_load.alloc(G.ng);
  std::vector<double> geo((size_t)G.nlat + 2 * G.nphi);
  for (int j = 0; j < G.nlat; ++j) geo[j] = std::sin(G.colat[j]) * std::cos(G.colat[j]);
  for (int i = 0; i < G.nphi; ++i) {
    const double lon = 2.0 * PI * (double)i / (double)G.nphi;
    geo[G.nlat + i] = std::cos(lon);
    geo[G.nlat + G.nphi + i] = std::sin(lon);
  }
  h->d_rot_geo.upload(geo, s);
  DArr<double> abf, drf, dcf, surf;
  DArr<int> ipivf;
  build_fluid_deg2_band(h, abf, drf, dcf, ipivf);
  surf.alloc(6);
  k_rot_unit<<<1, 32, 0, s>>>(nr, nd, p.r_earth, h->g, h->d_ab.p, h->d_dr.p, h->d_dc.p, h->d_ipiv.p, abf.p, drf.p,
                              dcf.p, ipivf.p, h->d_rot_f.p, h->d_rot_x.p, surf.p);
  VG_CUDA(cudaGetLastError());
  double sv[6];
  surf.download(sv, 6, s);
  VG_CUDA(cudaStreamSynchronize(s));
  h->rot_Fe[0] = sv[0];
  h->rot_Ue[0] = sv[1];
  h->rot_Fe[1] = sv[2];
  h->rot_Ue[1] = sv[3];
  h->rot_a = p.r_earth;
  h->rot_g = h->g;
  h->rot_kTe = -h->rot_Fe[1] - 1.0;
  h->rot_hTe = h->g * h->rot_Ue[1];
  h->rot_ks_fluid = -sv[4] / 1.0 - 1.0;
  h->rot_ks_flat = 3.0 * GRAV_G * h->rot_CminusA / (std::pow(h->rot_a, 5) * h->rot_Omega * h->rot_Omega);
  h->rot_ks = h->rot_ks_fluid;
  h->rot_on = true;
}

// rotation_begin_step (src/vilma_rotation.f90:154-168): drift of both channels
// shared memory of k_rot_begin
// (the element contributions always; the band, pivots and right-hand sides
// when they fit; `staged` says which)
static size_t rot_smem(const vg_handle* h, int& staged) {
  const size_t b = (size_t)h->ndof * VG_LDAB * sizeof(double) + (size_t)4 * h->ndof * sizeof(double) +
                   (size_t)h->ndof * sizeof(int);
  staged = b <= 200 * 1024 ? 1 : 0;
  const size_t need = staged ? b : 0;
  if (need > 48 * 1024) raise_smem_limit((const void*)k_rot_begin, need);
  return need;
}

// the drift of both channels from the entering memory
static void rot_begin_launch(vg_handle* h, const RotArgs& A, size_t sm, int staged, cudaStream_t s) {
  k_rot_elem<<<(4 * A.ne + ROT_ELEM_THREADS - 1) / ROT_ELEM_THREADS, ROT_ELEM_THREADS, 0, s>>>(A);
  k_rot_begin<<<1, ROT_THREADS, sm, s>>>(A, staged);
  h->n_launch += 2;
  VG_CUDA(cudaGetLastError());
}

void rotation_begin(vg_handle* h) {
  int staged = 0;
  const size_t sm = rot_smem(h, staged);
  rot_begin_launch(h, rot_args(h), sm, staged, h->stream);
}

// the rotational sea-level term held across the interval
void rotation_s_rot(vg_handle* h) {
  const Grid& G = h->grid;
  const double kN = h->rot_Omega * h->rot_Omega * h->rot_a * h->rot_a / h->rot_g;
  const double ku = h->rot_Omega * h->rot_Omega * h->rot_a * h->rot_a;
  k_rot_srot<<<(G.ng + 255) / 256, 256, 0, h->stream>>>(G.nlat, G.nphi, h->d_rot_sc.p, h->d_rot_geo.p, h->rot_kTe,
                                                        h->rot_Ue[1], kN, ku, h->d_srot.p);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
}

// After the interval: polar motion advanced under the interval-end load, in
// n_sub = ceil(dt / dt_fe_max) sub-steps (src/vilma_coupling.f90:411-421).
void rotation_advance(vg_handle* h, const double* d_sigma, double dt) {
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  sht_synthesis_dev(h, d_sigma, h->d_rot_load.p, 1);
  k_rot_rows<<<G.nlat, 128, 0, s>>>(G.nlat, G.nphi, h->d_rot_load.p, h->d_rot_geo.p, h->d_rot_rows.p);
  ++h->n_launch;
  VG_CUDA(cudaGetLastError());
  const int n_sub = std::max(1, (int)std::ceil(dt / h->rot_dt_fe_max));
  const double dt_sub = dt / (double)n_sub;
  SolveArgs S;
  S.nlat = G.nlat;
  S.dlon = 2.0 * PI / (double)G.nphi;
  S.a4 = std::pow(h->rot_a, 4);
  S.scl = 5.0 / (4.0 * PI * GRAV_G * h->rot_a);
  S.Fe_load = h->rot_Fe[0];
  S.CminusA = h->rot_CminusA;
  S.k_s = h->rot_ks;
  S.kTe = h->rot_kTe;
  S.dt = dt_sub;
  S.w = G.d_wts.p;
  S.rows = h->d_rot_rows.p;
  const RotArgs A = rot_args(h);
  int staged = 0;
  const size_t sm = rot_smem(h, staged);
  for (int k = 0; k < n_sub; ++k) {
    rot_begin_launch(h, A, sm, staged, s);
    k_rot_solve_commit<<<1, 256, 0, s>>>(A, S);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  }
}

}  // namespace vg
