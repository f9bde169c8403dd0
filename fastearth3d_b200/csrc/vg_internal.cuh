// Internal declarations of the B200 backend (not part of the C-ABI).
//
// Data layout in HBM (one model instance, FP64 throughout unless stated):
//   memory state   mem[buf][((s*2 + ri)*ne + e)*4 + lam][k]  — shape s in {A,B,C},
//                  ri in {re,im}, element e, channel lam, slot k FASTEST, so a
//                  thread per (l,m) slot reads and writes coalesced rows. Two
//                  buffers: the advance writes the other one, and a rejected
//                  sub-step is a pointer swap, not a copy.
//   nodal drift    dUn/dVn[ri][node][k]
//   band factors   ab[(l*ldab + row)*ndof + col] for l >= 2 (band storage of
//                  LAPACK dgbtf2, row index kv+1+i-j), degree 1 apart (dense)
//   grid fields    (nphi, nlat), phi fastest, colatitude north first
//   Legendre       plm/dplm[lm][j] (j fastest), lm m-major
#pragma once
#include <cuda_runtime.h>
#include <atomic>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vilma_gpu.h"

// leading dimension of the per-column band records of degrees >= 2:
// rows 0..18 = dgbtf2 band (kl = ku = 6), 19 = 1/pivot, 20 = pivot offset
#define VG_LDAB 21

#define VG_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t _e = (call);                                                             \
    if (_e != cudaSuccess)                                                               \
      throw vg::Error(std::string(#call) + ": " + cudaGetErrorString(_e));              \
  } while (0)

namespace vg {

struct Error : std::exception {
  std::string msg;
  explicit Error(std::string m) : msg(std::move(m)) {}
  const char* what() const noexcept override { return msg.c_str(); }
};

constexpr double PI = 3.14159265358979323846;
constexpr double GRAV_G = 6.67430e-11;       // src/vilma_constants.f90
constexpr double RHO_ICE = 931.0;
constexpr double RHO_WATER = 1000.0;
constexpr double SEC_PER_YEAR = 31556926.0;
constexpr double KYR = 1000.0 * SEC_PER_YEAR;
constexpr double TINY = 2.2250738585072014e-308;
constexpr double HUGE_ = 1.7976931348623157e308;

template <class T>
struct DArr {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    release();
    n = count;
    if (count) {
      VG_CUDA(cudaMalloc(&p, count * sizeof(T)));
      // The handle's stream is non-blocking, so nothing orders this legacy-stream
      // memset before later work on it: finish the zeroing here (setup only).
      VG_CUDA(cudaMemset(p, 0, count * sizeof(T)));
      VG_CUDA(cudaDeviceSynchronize());
    }
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    VG_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& v, cudaStream_t s) {
    if (v.size() != n) alloc(v.size());
    upload(v.data(), v.size(), s);
  }
  void download(T* h, size_t count, cudaStream_t s) const {
    VG_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  ~DArr() { release(); }
  DArr() = default;
  DArr(const DArr&) = delete;
  DArr& operator=(const DArr&) = delete;
};

// Scalars the SLE fixed point and the stepper decide on, kept on the device and
// read back as one small struct when the host needs a decision.
struct SleScalars {
  double C_int, ice_int, zeta_int, Cs_int, dphi, dmax, smax, mass_Cs;
  int flips, n_inner;  // coastline flips; inner iterations done by the fused loop
  int bar_error;       // a grid barrier of the fused loop gave up
  unsigned long long mem_norm_bits;  // max |memory| of the state the last advance wrote
};

// Phase timers, the device counterpart of the reference's [PROFILE] buckets
// (t_drift, t_mem, t_sht/t_apply of src/vilma_response.f90:179-186,
// src/vilma_sle.f90:100-119): CUDA events recorded on the handle's stream
// around each phase, read and reset by vg_profile_read.
struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> ev[VG_NPHASE];  // start/stop pairs
  double ms[VG_NPHASE] = {};
  long long calls[VG_NPHASE] = {};
};

struct Grid {
  int lmax, mmax, M, nlat, nphi, ng, nlm;
  std::vector<double> x, colat, sint, wts;  // host
  DArr<double> d_wts, d_sint, d_cott, d_invsin;
  DArr<double> d_plm, d_dplm;   // (nlm, nlat)
  DArr<double> d_cos, d_sin;    // (nphi) twiddles cos/sin(2 pi t / nphi)
  DArr<int> d_lm_m;             // lm -> m
  DArr<int> d_lm_l;             // lm -> l
  DArr<int> d_mbeg;             // m -> first lm (size M+1)
};

}  // namespace vg

struct vg_handle {
  vg_params p;
  std::string err;
  int device = 0;
  // bound on the device-side waits that hand work between CTAs or warps (grid
  // barriers of the fused sea-level loop, producer / consumer waits of the
  // tensor-core stages); a wait that runs out raises a status the host turns
  // into an error (vg_set_wait_limit)
  unsigned long long wait_ns = 2000000000ull;
  cudaStream_t stream = nullptr;
  // second stream: the degree-1 drift (one CTA) runs there beside the band
  // sweeps of degrees >= 2, forked after the forcing and joined before the
  // drift is read
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // the whole drift on the second stream (its degree 1 on a third) beside the
  // sea-level pass setup, joined before the fused loop reads it
  cudaStream_t aux2 = nullptr;
  cudaEvent_t ev_dfork = nullptr, ev_djoin = nullptr;
  // sizes
  int nr = 0, ne = 0, ndof = 0, nk = 0, ne3d = 0;
  int kl = 0, ku = 0, kv = 0, ldab = 0;  // band of degrees >= 2
  int ns1 = 0, ldab1 = 0, kv1 = 0, kl1 = 0;  // degree-1 bordered system
  double a = 0, g = 0, dt = 0, time_s = 0, time_yr = 0, max_rate = 0;
  vg::Grid grid;
  // host copies of setup data
  std::vector<double> r, mu, MkPerDt;
  std::vector<int> elem_layer, kdeg_h, k2lm_h, kbeg_h;
  std::vector<char> active1d_h;
  std::vector<int> e3d_h;
  std::vector<double> pert_mean3d;  // lateral mean of the log10 perturbation per 3-D element
  // operators
  vg::DArr<double> d_ab, d_dr, d_dc, d_rdiag;  // degrees 2..lmax (band, column-major, ldab 19)
  vg::DArr<int> d_ipiv;
  vg::DArr<double> d_ab1, d_dr1, d_dc1, d_null1, d_G1;  // degree 1 (bordered, dense band)
  vg::DArr<double> d_bh;                        // equilibrated drift RHS (2, 2*nr, nk)
  vg::DArr<double> d_Krhs;                      // dissipative-forcing coefficients (lmax+1, ne, 48)
  vg::DArr<int4> d_tasks;                       // drift sweep tasks: (degree, first slot, slots)
  int ntask = 0;
  vg::DArr<int> d_ipiv1;
  // per-element / per-degree constants
  vg::DArr<double> d_r, d_mu, d_MkPerDt;
  vg::DArr<char> d_active1d;
  vg::DArr<double> d_Jr, d_nrmc, d_sa, d_sb, d_sc, d_gu, d_gn, d_gv, d_xUn, d_xVn;
  vg::DArr<int> d_kdeg, d_k2lm, d_lm2k;
  // state
  vg::DArr<double> d_mem[2];
  int cur = 0;
  vg::DArr<double> d_dUn, d_dVn, d_drift;  // drift: dUa re,im, dFa re,im, dVa re,im (6*nk)
  vg::DArr<double> d_mnorm, d_xs;          // per-slot memory norm (2 buffers x nk); band-solve scratch
  vg::DArr<unsigned long long> d_maxbits;  // max |memory| of each buffer (double bits); [2] kernel status bits
  vg::DArr<vg::SleScalars> d_sc_;
  vg::SleScalars* h_sc = nullptr;  // pinned
  double mem_norm = 0.0;           // ||state cur||_inf (host copy)
  // 3-D
  bool lat_visc = false;
  vg::DArr<double> d_MkPerDt3;  // (ne3d, nlat, nphi)
  vg::DArr<int> d_e3d;
  vg::DArr<double> d_G6, d_H6, d_n6;  // spin-2 kernels (nlm, nlat), norms (lmax+1)
  vg::DArr<double> d_wP, d_wD, d_wG, d_wH;  // quadrature-weighted analysis kernels (nlm, nlat)
  vg::DArr<int> d_kbeg;               // first slot of each degree (lmax + 2)
  vg::DArr<double> d_X, d_Y, d_dy;    // 3-D work buffers: synthesis input, Fourier products, increments
  vg::DArr<double> d_v3a_Yb, d_v3a_dyb, d_v3a_Rb;  // 3-D adjoint: product adjoints
  double* v3_gstore = nullptr;  // when set, the FP64 longitude pass also stores its grid there (adjoint sweeps)
  vg::DArr<double> d_lon_tw, d_lon_twt;  // FP64 longitude pass: dense twiddle tables (by order, by longitude)
  // toroidal degree of freedom (p.toroidal and a genuinely 3-D element;
  // vg_toroidal.cu): memory tmem[buf][((s*2 + ri)*ne + e)*2 + lam][k] with
  // lam 0 = lambda 3, 1 = lambda 4, double-buffered with d_mem (same `cur`)
  bool tor_on = false;
  vg::DArr<double> d_tmem[2];
  vg::DArr<double> d_dWn, d_dWa;           // nodal W drift [ri][node][k], surface W(a) [ri][k]
  vg::DArr<double> d_tGinv;                // inverse W operators, degree l at (l - 1) nr^2 (row-major)
  vg::DArr<double> d_tGinvT, d_tWa_scratch;  // their transposes (the adjoint, built at first use), a W(a) sink
  vg::DArr<double> d_tg;                   // W drift forcing [ri][node][k]
  vg::DArr<double> d_tK;                   // forcing maps of the toroidal memory (lmax + 1, ne, 12)
  vg::DArr<double> d_edWn, d_dW_avg, d_dWa_prev, d_tmem_s, d_tmem_c;  // trapezoidal scheme
  // trapezoidal scheme (scheme = VG_SCHEME_TRAP; vg_trap.cu)
  vg::DArr<double> d_edUn, d_edVn;      // endpoint nodal drift (2 nr nk each)
  vg::DArr<double> d_dU_avg, d_dV_avg;  // mean of the entering and endpoint nodal drift
  vg::DArr<double> d_sigma_n, d_sigma_next, d_sigma_avg, d_sigma_n_s;  // loads (2 nlm each)
  vg::DArr<double> d_dUa_prev;          // surface U drift of the previous endpoint pass (2 nk)
  vg::DArr<double> d_mem_s, d_mem_c;    // step doubling: tau_n and tau_coarse
  vg::DArr<unsigned long long> d_trap_red;  // max reductions (err, tau, drift change, drift)
  bool sigma_primed = false, sigma_primed_s = false;
  double time_s_saved = 0.0, dt_try = 0.0;  // dt_try carried across intervals [s]
  int couple_pass = 0, couple_iters_last = 0;
  long long n_floor = 0;
  // sea-level equation fields (ng each unless stated)
  vg::DArr<double> d_z_bed_eq, d_h_ice_eq, d_h_ice, d_ice1, d_ice_now, d_dice_now, d_rsl, d_rsl_n,
      d_C, d_C0, d_C_next, d_dig, d_wcorr, d_Sraw, d_zbed, d_tmp;
  vg::DArr<double> d_F;        // Fourier coefficients (2 * M * nlat * batch)
  vg::DArr<double> d_Gs;       // Legendre sums (2 * M * nlat * batch)
  vg::DArr<int2> d_sle_chunk;  // fused sea-level loop: Legendre synthesis chunks (m, first l - m)
  vg::DArr<int> d_sle_cbeg;    // first chunk of each order
  vg::DArr<double> d_sle_Gp;   // partial Legendre sums (chunk, nlat, 4)
  int sle_nchunk = 0;
  vg::DArr<double> d_sigma, d_ulm, d_nlm;  // spectra (2*nlm)
  vg::DArr<double> d_rowpart;  // per-row partial sums (8 * nlat)
  vg::DArr<unsigned int> d_gbar;  // grid barrier of the fused inner loop: count, generation, error
  int sle_grid = 0;               // CTAs of the cooperative inner-loop launch (one per SM)
  // counters
  long long n_accept = 0, n_reject = 0, n_solve = 0, n_drift_solved = 0;
  int n_sub_last = 0, n_outer_last = 0, n_inner_last = 0, n_flip_last = 0;
  double worst_mass_resid = 0, bsl = 0;
  bool have_reference = false;
  long long n_launch = 0;  // kernels launched by the time step (all phases)
  vg::Prof prof;
  // rotational feedback (two degree-2 channels and the polar motion)
  bool rot_on = false;
  bool srot_ext = false;  // vg_advance: a host-given rotational potential in d_srot for this interval
  double rot_kTe = 0, rot_hTe = 0, rot_ks = 0, rot_ks_fluid = 0, rot_ks_flat = 0;
  double rot_Fe[2] = {0, 0}, rot_Ue[2] = {0, 0};  // unit responses: load, tidal channel
  double rot_a = 0, rot_g = 0, rot_CminusA = 2.63e35, rot_Omega = 7.292115e-5, rot_dt_fe_max = HUGE_VAL;
  vg::DArr<double> d_rot_mkdt;  // channel mu/eta per element (ne)
  vg::DArr<double> d_rot_x;     // unit nodal responses [ch][U, V][nr]
  vg::DArr<double> d_rot_mem;   // memory [ch][A re, A im, B re, B im, C re, C im][ne][4]
  vg::DArr<double> d_rot_dn;    // nodal drift [ch][dUn re, dUn im, dVn re, dVn im][nr]
  vg::DArr<double> d_rot_sc;    // scalars (see vg_rotation.cu)
  vg::DArr<double> d_rot_f;     // channel solve work (4 x ndof)
  vg::DArr<double> d_rot_fl;    // channel element contributions (4 x ne x 4)
  vg::DArr<double> d_rot_rows;  // per-row partial inertia sums (2 x nlat)
  vg::DArr<double> d_rot_geo;   // sin(theta)cos(theta) [nlat], cos(lon), sin(lon) [nphi each]
  vg::DArr<double> d_srot, d_rot_load;  // grid fields
  // split-precision tensor-core plan of the 3-D advance (owned, opaque here)
  void* tc_plan = nullptr;
  void (*tc_plan_release)(void*) = nullptr;
  // work buffers of the misfit / adjoint entry points (owned, opaque here)
  void* sle_tape = nullptr;  // while set, the coupled forward records its decisions there (vg_adjoint.cu)
  void* adj_work = nullptr;
  void (*adj_release)(void*) = nullptr;
  ~vg_handle() {
    if (tc_plan_release) tc_plan_release(tc_plan);
    if (adj_release) adj_release(adj_work);
  }
};

namespace vg {
// setup (vg_setup.cu)
void setup_handle(vg_handle* h);
void build_grid(Grid& G, int lmax, int nlat, int nphi, cudaStream_t s);
// response kernels (vg_radial.cu)
// drift of memory buffer buf (-1: the current one) into the nodal targets
// (nullptr: the handle's dUn, dVn) and the surface drift
void launch_drift(vg_handle* h, int buf = -1, double* dUn = nullptr, double* dVn = nullptr, double* dWn = nullptr);
// the same without the toroidal drift, the band sweeps on s0 and degree 1 on s1
void launch_drift_on(vg_handle* h, int buf, double* dUn, double* dVn, cudaStream_t s0, cudaStream_t s1);
// memory advance of one step (3-D elements pseudo-spectrally, the others per
// slot), current buffer -> the other one, with the strain of (sigma, dUn,
// dVn) (nullptr: the handle's drift), and the next buffer's per-slot norms and
// their maximum; trap: the trapezoidal rule with sigma, dUn, dVn the means of
// the step's two ends
void advance_memory(vg_handle* h, const double* d_sigma, double dt, const double* dUn = nullptr,
                    const double* dVn = nullptr, bool trap = false, const double* dWn = nullptr);
void launch_apply(vg_handle* h, const double* d_sigma, double* d_u, double* d_n);
void compute_mem_norm(vg_handle* h, int buf);
double read_mem_norm(vg_handle* h, int buf);
// SHT (vg_sht.cu)
void fourier_analysis_dev(vg_handle* h, const double* d_f, int batch, double* d_F);
void legendre_analysis_dev(vg_handle* h, const double* d_F, int batch, double* d_q);
void legendre_synth_dev(vg_handle* h, const double* d_q, int batch, double* d_G);
void fourier_synth_dev(vg_handle* h, const double* d_G, int batch, double* d_f);
void sht_analysis_dev(vg_handle* h, const double* d_f, double* d_q, int batch);
void sht_synthesis_dev(vg_handle* h, const double* d_q, double* d_f, int batch);
// SLE + stepper (vg_sle.cu)
void sle_solve_dev(vg_handle* h, double dt, bool report_only);
void update_dev(vg_handle* h, const double* d_ice1, double dt_yr);
void update_bsl(vg_handle* h);
// 3-D (vg_visc3d.cu)
void visc3d_enable(vg_handle* h, const double* pert_host);
// 3-D memory advance (current buffer -> the other one), folding the new
// maxima into the next buffer's per-slot norms (zeroed by the caller); dUn,
// dVn and trap as for advance_memory (the pointwise factor M / (1 + M/2) when
// trap)
void visc3d_advance(vg_handle* h, const double* d_sigma, double dt, const double* dUn = nullptr,
                    const double* dVn = nullptr, bool trap = false, const double* dWn = nullptr);
// transposed 3-D advance (FP64 path) of one step whose longitude-pass grid the
// forward stored in gstore: lam_new (3-D entries) = lam + gather^T, E (3-D
// elements) = strain adjoints, gw * d J / d (M dt) accumulated into gradMdt
// (ne3d, nlat, nphi)
// (with the toroidal channels also lam_t -> lam_t_new and the toroidal
// strain adjoints Et (W0, W1 planes) of the 3-D elements)
void visc3d_adjoint(vg_handle* h, const double* gstore, double dt, const double* lam, double* lam_new, double* E,
                    double* gradMdt, double gw = 1.0, const double* lam_t = nullptr, double* lam_t_new = nullptr,
                    double* Et = nullptr);
// exact tensor-core stages (vg_oz.cu): converter warps per stage (8 or 4);
// oz_get_ncw returns false when the handle has no exact-stage plan
void oz_set_ncw(vg_handle* h, const int ncw[4]);
bool oz_get_ncw(const vg_handle* h, int ncw[4]);
// The interval driver's state (memory of the current buffer, spheroidal and
// toroidal, its per-slot norms and both buffers' maxima, rsl, entering ice,
// ocean function, z_bed, the last load spectrum, the trapezoidal scheme's
// carried step and sigma_n, the rotational feedback's state, clocks and
// counters), saved and put back by the entry points that run trial intervals
// (the coupled adjoint, the autotuner); vg_api.cu
struct DriverSnap {
  DArr<double> mem, mnorm, rsl, hice, C, zbed, sig;
  DArr<double> tmem;                 // the toroidal memory of the current buffer (toroidal channels)
  DArr<double> sig_n;                // the trapezoidal scheme's sigma_n
  DArr<double> rot_sc, rot_mem;      // rotational feedback: polar motion and scalars, channel memories
  DArr<unsigned long long> maxbits;  // both buffers' max |memory| (the drift skip gate's scale)
  int cur = 0;
  bool sigma_primed = false;
  double dt_try = 0;
  double time_s = 0, time_yr = 0, mem_norm = 0, bsl = 0, worst = 0;
  long long n_accept = 0, n_reject = 0, n_solve = 0;
  int n_sub = 0, n_outer = 0, n_inner = 0, n_flip = 0;
  void save(vg_handle* h);
  void restore(vg_handle* h);  // synchronises the handle's stream
};
// Tape of the coupled forward for the sea-level adjoint (vg_adjoint.cu): with
// h->sle_tape set, the forward-Euler driver reports every sub-step attempt
// (interpolation fraction, length; accepted or not) and the sea-level solve
// every pass (its ocean function, ocean area and inner iterations done)
void tape_attempt_begin(vg_handle* h, double frac, double dt);
void tape_pass(vg_handle* h, double C_int, int n_inner);
void tape_attempt_end(vg_handle* h, bool accepted);
// rotational feedback (vg_rotation.cu)
void build_fluid_deg2_band(vg_handle* h, DArr<double>& ab, DArr<double>& dr, DArr<double>& dc, DArr<int>& ipiv);
void rotation_setup(vg_handle* h);
void rotation_begin(vg_handle* h);
void rotation_s_rot(vg_handle* h);
void rotation_advance(vg_handle* h, const double* d_sigma, double dt);
// 3-D split-precision tensor-core stages (vg_tc.cu)
void visc3d_tc_enable(vg_handle* h);
void visc3d_tc_buffers(vg_handle* h, float** X, float** dy);
void visc3d_tc_run(vg_handle* h, double dt, bool trap = false);
// 3-D exact int8 tensor-core stages (vg_oz.cu)
void visc3d_oz_enable(vg_handle* h);
unsigned long long* visc3d_oz_gather_max(vg_handle* h);
void visc3d_oz_run(vg_handle* h, double dt, bool trap = false);
// toroidal degree of freedom (vg_toroidal.cu; operator assembly in vg_setup.cu)
void toroidal_tridiag(const std::vector<double>& r, const std::vector<double>& mu, int j, std::vector<double>& diag,
                      std::vector<double>& off, std::vector<char>& dead);
std::vector<double> toroidal_rotation_weights(const std::vector<double>& r, const std::vector<double>& mu,
                                              int& nshell);
void toroidal_enable(vg_handle* h);
// W drift of memory buffer buf into dWn (nullptr: the handle's) and d_dWa
void launch_drift_tor(vg_handle* h, int buf, double* dWn);
// lambda 3, 4 advance of the spectrally advanced elements (cur -> nxt) from the
// nodal W drift dWn (the step's mean for trap), folding |toroidal memory| of
// every element of nxt into the per-slot norms mn
void launch_advance_1d_tor(vg_handle* h, double dt, const double* dWn, bool trap, double* mn);
// fold |toroidal memory of buffer buf| into the per-slot norms mn
void mem_norm_tor(vg_handle* h, int buf, double* mn);
// toroidal adjoint pieces (vg_toroidal.cu): the 1-D lambda 3, 4 advance
// transposed (lam_t -> lam_t_new, the element W adjoints Et), and the W drift
// transposed from Et into lam_t_new (adds; Wb, gb (2, nr, nk) work arrays)
void advance_1d_tor_T(vg_handle* h, double dt, const double* lam_t, double* lam_t_new, double* Et);
void drift_tor_T(vg_handle* h, const double* Et, double* Wb, double* gb, double* lam_t_new);
// trapezoidal scheme (vg_trap.cu)
void trap_setup(vg_handle* h);
void trap_prepare(vg_handle* h);
bool trap_endpoint_pass(vg_handle* h, double dt);
void trap_finalize(vg_handle* h, double dt);
void trap_save(vg_handle* h);
void trap_restore(vg_handle* h);
void trap_stash_coarse(vg_handle* h);
void trap_coarse_fine_error(vg_handle* h, double& err_inf, double& tau_inf);
void trap_prime(vg_handle* h);
// misc
void sync_scalars(vg_handle* h);
// Raise a kernel's dynamic shared-memory limit to at least `bytes`, never
// lowering it: handles of different sizes share the kernel, and may launch it
// concurrently from different host threads (vg_update_batch).
void raise_smem_limit(const void* kernel, size_t bytes);
// phase timer scope: records a start event now and a stop event at scope exit
struct PhaseScope {
  vg_handle* h;
  int ph;
  PhaseScope(vg_handle* hh, int p);
  ~PhaseScope();
};
void prof_collect(vg_handle* h);
}  // namespace vg
