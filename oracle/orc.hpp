// CPU ORACLE — test infrastructure only.
//
// A C++17/OpenMP restatement of the reference algorithm of VILMA v2's
// viscoelastic time step (fesmc/FastEarth3D, Fortran 2008 + OpenMP). It exists
// to check the CUDA library and to serve as the timed CPU baseline; nothing in
// the product library links, loads or calls it. Each routine cites the
// reference file:line it restates.
//
// Parity anchors (the reference itself cannot be built here: no Fortran
// compiler, no SHTns/FFTW/netCDF): the vendored normal-mode Love-number table
// data/benchmarks/love_M3-L70-V01/mod_M3-L70-V01 (fluid and elastic limits),
// the Spada-2011 disc benchmark data/benchmarks/disc_spada2011/{u,n}_disc.txt,
// and the reference tests' known-answer identities (band vs dense LU, SHT round
// trip and integrals, 3-D == 1-D for a laterally uniform viscosity, ocean-mass
// conservation). SHTns 3.7.5 is replaced by the restatement of its published
// conventions in orc_sht.cpp (orthonormal, no Condon-Shortley phase, Gauss
// grid, m >= 0 stored, m > 0 counted twice for real fields).
#pragma once
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

namespace orc {

using cplx = std::complex<double>;

constexpr double PI = 3.14159265358979323846;
constexpr double GRAV_G = 6.67430e-11;        // vilma_constants.f90:19
constexpr double RHO_ICE = 931.0;             // vilma_constants.f90:29
constexpr double RHO_WATER = 1000.0;          // vilma_constants.f90:30
constexpr double SEC_PER_YEAR = 31556926.0;   // vilma_constants.f90:35
constexpr double KYR = 1000.0 * SEC_PER_YEAR; // vilma_constants.f90:36
constexpr double OMEGA_EARTH = 7.292115e-5;   // vilma_constants.f90:33

enum Rheology { RHEOL_ELASTIC = 0, RHEOL_MAXWELL = 1, RHEOL_FLUID = 2 };

// vilma_earth_structure.f90:23-45 — layers surface-first.
struct Layer {
  double r_bot = 0, r_top = 0, rho = 0, mu = 0, eta = 0;
  int rheology = RHEOL_MAXWELL;
};
struct Earth {
  double r_earth = 6.371e6;
  std::vector<Layer> layers;
};
double earth_mass_below(const Earth& e, double r);
double earth_gravity_at(const Earth& e, double r);
double earth_moi(const Earth& e);
Earth build_M3L70V01();

// vilma_radial_fe.f90:56-62.
struct Mesh {
  int nr = 0, ne = 0;
  std::vector<double> r;
  std::vector<int> elem_layer;  // 0-based layer index per element
};
// ne_layer: per-layer element counts (surface-first, like layers); nullptr or
// all-zero -> the reference depth-target rule (vilma_radial_fe.f90:140-224).
Mesh radial_mesh_build(const Earth& e, const int* ne_layer);

inline int idx_u(int k) { return 4 * k; }      // 0-based node k
inline int idx_v(int k) { return 4 * k + 1; }
inline int idx_f(int k) { return 4 * k + 2; }
inline int idx_p(int e) { return 4 * e + 3; }  // 0-based element e
inline int ndof_of(int nr) { return 4 * nr - 1; }

// vilma_band.f90:19-25; ab column-major (ldab, n).
struct Band {
  int n = 0, kl = 0, ku = 0, kv = 0, ldab = 0;
  std::vector<double> ab;
  std::vector<int> ipiv;  // 0-based
  double& at(int row1, int col1) { return ab[(size_t)(col1 - 1) * ldab + (row1 - 1)]; }
  double at(int row1, int col1) const { return ab[(size_t)(col1 - 1) * ldab + (row1 - 1)]; }
};
bool band_build(Band& b, int n, const std::vector<int>& rows, const std::vector<int>& cols,
                const std::vector<double>& vals);
void band_solve(const Band& b, double* x);  // in place

struct BorderedBand {
  int nd = 0, nb = 0, ns = 0;
  Band band;
  std::vector<double> dr, dc, w;  // w: (nd, nb) column-major
};

struct RadialOp {
  int j = -1, nr = 0, ne = 0, ndof = 0;
  double r_earth = 0, g_surf = 0;
  BorderedBand sys;
  std::vector<double> nullmode;  // j = 1 only
};
std::vector<double> build_dense_operator(const Earth& e, const Mesh& m, int j, bool with_uniq);
std::vector<double> uniq_weight(const Mesh& m);
void radial_operator_assemble(RadialOp& op, const Earth& e, const Mesh& m, int j);
void radial_operator_solve_vec(const RadialOp& op, const double* b, double* x, const double* border);
void radial_operator_load_rhs(const RadialOp& op, double sigma, double* b);
void loading_love(const Earth& e, int j, double sigma, double Ua, double Va, double Fa,
                  double& h, double& l, double& k);
// w: (nd, nb) column-major border columns, nb = 0 for none
void bordered_band_factor(BorderedBand& sys, const std::vector<double>& A, int nd, const std::vector<double>& w,
                          int nb);
void bordered_band_solve(const BorderedBand& sys, const double* b, double* x, const double* border);

// vilma_radial_fe.f90:699-817: the per-degree toroidal W operator (nr x nr,
// tridiagonal; dead nodes pinned; degree 1 bordered by per-shell net-rotation
// constraints)
struct TorOp {
  int j = -1, nr = 0, ne = 0;
  BorderedBand sys;
  std::vector<char> pinned;  // per node
};
std::vector<double> build_toroidal_operator(const std::vector<double>& r, const std::vector<double>& mu, int j);
std::vector<double> rotation_weights(const std::vector<double>& r, const std::vector<double>& mu, int& nshell);
void toroidal_operator_assemble(TorOp& op, const std::vector<double>& r, const std::vector<double>& mu, int j);
void toroidal_operator_solve_vec(const TorOp& op, const double* b, double* x);

// ---------------------------------------------------------------- SHT grid
struct Sht {
  int lmax = 0, mmax = 0, nlat = 0, nphi = 0, nlm = 0;
  std::vector<double> x, colat, sint, wts;  // nlat, north first
  std::vector<double> plm, dplm;            // (nlm, nlat): plm[lm*nlat + j]
  std::vector<double> cott, invsin;         // nlat
  std::vector<int> ldeg, mord;              // nlm
  std::vector<double> llp1;                 // nlm
  std::vector<double> n6;                   // 0..lmax, spin-2 norm
  std::vector<double> n4;                   // 0..lmax, toroidal spin-2 norm
  // FFT plan (mixed radix over nphi)
  std::vector<int> fft_factors;
  std::vector<cplx> tw;  // exp(-2 pi i k / nphi)
  int lmidx(int l, int m) const { return m * (lmax + 1) - m * (m - 1) / 2 + (l - m); }
};
void sht_init(Sht& s, int lmax, int nlat, int nphi);
double sht_surface_integral(const Sht& s, const double* f);
void sht_synth(const Sht& s, const cplx* q, double* f);
void sht_analysis(const Sht& s, const double* f, cplx* q);
void sht_sph_synth(const Sht& s, const cplx* sl, double* vt, double* vp);
void sht_sph_analysis(const Sht& s, const double* vt, const double* vp, cplx* sl);
// c: (nch, nlm) channel-major, nch = 4 (lambda 1,2,5,6) or 6 (+ lambda 3,4)
void tensor_synth(const Sht& s, const cplx* c, double* dyad /*6*np*nl*/, int nch = 4);
void tensor_analysis(const Sht& s, const double* dyad, cplx* c, int nch = 4);
// e_r x grad_1 T = (-F, E) (vilma_sht.f90:258-277) and its analysis
void sht_tor_synth(const Sht& s, const cplx* tl, double* vt, double* vp);
void sht_tor_analysis(const Sht& s, const double* vt, const double* vp, cplx* tl);
void sht_calibrate_n6(Sht& s);

// ---------------------------------------------------------------- response
constexpr int NLAM = 4;
constexpr int NLAM_TOR = 2;  // vilma_viscoelastic.f90: lambda 3, 4
// vilma_viscoelastic.f90:60-64 memory-scheme codes (forward Euler, trapezoidal)
enum Scheme { SCHEME_FE = 0, SCHEME_TRAP = 2 };

struct Response {
  int lmax = 0, nr = 0, ne = 0, ndof = 0, nlm = 0, nk = 0;
  double g = 0, a = 0, dt = 0, time = 0;
  double skip_tol = 1e-4, visc3d_tol = 1e-3;
  bool deg1_cm = true;
  std::vector<RadialOp> ops;  // index l (0 unused)
  std::vector<double> r, mu, Mk, MkPerDt;
  std::vector<char> active1d;
  std::vector<double> Jr;                 // index l
  std::vector<double> nrmc;               // (l)*4 + lam
  std::vector<double> sa, sb, sc;         // (l)*16 + t*4 + lam
  std::vector<double> gu, gn, gv;         // 0..lmax
  std::vector<double> xUn, xVn;           // l*nr + node
  std::vector<int> k2lm, kdeg, kbeg;      // kbeg: index l, size lmax+2
  // memory (NLAM, ne, nk): [k][e][lam]
  std::vector<double> Are, Aim, Bre, Bim, Cre, Cim;
  std::vector<cplx> dUa, dFa, dVa;
  std::vector<double> dUn_re, dUn_im, dVn_re, dVn_im;  // [k][node]
  std::vector<double> mnorm;
  // 3-D
  bool lat_visc = false;
  int ne3d = 0;
  std::vector<int> e3d;
  std::vector<double> Mk3, MkPerDt3;  // [e][j][i] (nphi fastest)
  std::vector<double> pert_mean3d;    // lateral mean of the log10 perturbation per 3-D element
  // memory scheme and the sea-level <-> memory co-convergence
  // (vilma_response.f90:176-223, 1480-1663)
  int scheme = SCHEME_FE;
  double couple_tol = 1e-6;
  int couple_pass = 0, couple_iters_last = 0;
  bool couple_done = false;
  std::vector<cplx> sigma_n, sigma_next;  // start-of-step load, staged endpoint load
  bool sigma_primed = false;
  std::vector<double> edUn_re, edUn_im, edVn_re, edVn_im;  // endpoint drift [k][node]
  std::vector<cplx> dUa_prev;
  std::vector<double> Are0, Aim0, Bre0, Bim0, Cre0, Cim0;  // tau_n snapshot
  // step-doubling buffers: A = tau_n (+ time, sigma_n), B = tau_coarse
  std::vector<double> Are_s, Aim_s, Bre_s, Bim_s, Cre_s, Cim_s;
  std::vector<double> Are_c, Aim_c, Bre_c, Bim_c, Cre_c, Cim_c;
  double time_s = 0;
  std::vector<cplx> sigma_n_s;
  bool sigma_primed_s = false;
  // toroidal channels (vilma_response.f90:126-146, 1055-1118): carried once a
  // 3-D element exists and `toroidal` is set. Memory (NLAM_TOR, ne, nk):
  // [k][e][lam], lam 0 = lambda 3, 1 = lambda 4.
  bool toroidal = false;
  int nlam = NLAM;
  std::vector<TorOp> tops;                       // index l (0 unused)
  std::vector<double> nrmt, sat, sbt, sct;       // l*2 + lam; l*4 + t*2 + lam
  std::vector<double> Atre, Atim, Btre, Btim, Ctre, Ctim;
  std::vector<cplx> dWa, dWa_prev;               // surface W drift (nk)
  std::vector<double> dWn_re, dWn_im, edWn_re, edWn_im;  // [k][node]
  std::vector<double> Atre0, Atim0, Btre0, Btim0, Ctre0, Ctim0;
  std::vector<double> Atre_s, Atim_s, Btre_s, Btim_s, Ctre_s, Ctim_s;
  std::vector<double> Atre_c, Atim_c, Btre_c, Btim_c, Ctre_c, Ctim_c;
  // profile counters
  double t_drift = 0, t_mem = 0;
  long n_drift = 0, n_mem = 0, n_solved = 0;
};
void response_init_ve(Response& R, const Earth& e, const Mesh& m, const Sht& s, double dt);
void response_begin_step(Response& R, const Sht& s);
void response_apply(const Response& R, const Sht& s, const cplx* sigma, cplx* u, cplx* n);
void response_advance(Response& R, const Sht& s, const cplx* sigma);  // vilma_advance
void response_set_dt(Response& R, double dt);
double response_max_rate(const Response& R);
double response_memory_norm(const Response& R);
void response_enable_lateral_visc(Response& R, const Sht& s, const double* pert /*[e][j][i]*/);
void response_enable_toroidal(Response& R);
void response_prepare_endpoint(Response& R);
void response_advance_endpoint(Response& R, const Sht& s, const cplx* sigma);
bool response_endpoint_converged(const Response& R);
void response_finalize_step(Response& R);
void response_prime_sigma(Response& R, const cplx* sig0);
void response_save_state(Response& R);
void response_restore_state(Response& R);
void response_stash_coarse(Response& R);
void response_coarse_fine_error(const Response& R, double& err_inf, double& tau_inf);

// ---------------------------------------------------------------- SLE / stepper / coupling
struct SleSolver {
  int n_outer = 3, n_inner = 20, max_mem_iter = 20;
  double tol = 1e-7;
  bool fixed_ocean = false, subgrid = true, warm_start = false;
  long n_solve = 0, n_outer_tot = 0, n_inner_tot = 0;
  int last_outer = 0, last_inner = 0, last_flips = 0;  // of the last solve (the device's vg_info counters)
};
struct SleResult {
  int n_outer_done = 0, n_inner_last = 0, n_coast_flip = 0, n_couple_done = 0;
  double resid = 0, mass_resid = 0, ocean_frac = 0, esl = 0;
};
void ocean_function(int n, const double* topo, const double* ice, double* C);
void sle_solve(SleSolver& sle, const Sht& s, Response& R, const double* d_ice, const double* ice,
               const double* topo0, double* rsl, double* C, SleResult& res, bool report_only,
               cplx* sigma_out, const double* s_rot);

struct Stepper {
  double cfl = 1.0, guard_growth = 1e3, dt_min = 0, dt_max = 1e300;
  // trapezoidal step-doubling controller (vilma_timestep.f90:40-53)
  double rtol = 1e-4, atol = 1e-3, safety = 0.9, grow_max = 5.0, shrink_min = 0.2, dt_try = 0.0;
  long n_accept = 0, n_reject = 0, n_solve = 0, n_floor = 0;
  int n_sub_last = 0;
  double worst_mass_resid = 0;
};
// returns 0 on success, nonzero on a collapsed guard (reference error stop)
int stepper_advance(Stepper& st, const Sht& s, Response& R, SleSolver& sle, const double* topo0,
                    const double* ice0, const double* ice1, const double* ice_ref, double t0,
                    double t1, double* rsl, double* C, const double* s_rot, cplx* sigma_out);

// ---------------------------------------------------------------- rotation
// vilma_rotation.f90: two degree-2 viscoelastic channels (load, tidal) carrying
// Maxwell memory, and the algebraic (Chandler-neglected) Liouville equation.
struct Deg2Channel {
  bool tidal = false;
  int nr = 0, ne = 0, ndof = 0;
  double Jr = 6.0, dt = 0.0;
  RadialOp op;
  std::vector<double> r, mu, Mk, MkPerDt;
  double norm[4] = {0, 0, 0, 0}, sa[16] = {}, sb[16] = {}, sc[16] = {};
  double Fe = 0.0, Ue = 0.0;
  std::vector<double> xUn, xVn;
  std::vector<double> Are, Aim, Bre, Bim, Cre, Cim;  // (NLAM, ne): [e][lam]
  cplx dF = 0.0, dU = 0.0;
  std::vector<double> dUn_re, dUn_im, dVn_re, dVn_im;
};
struct Rotation {
  bool enabled = false;
  cplx m = 0.0;
  double time = 0.0;
  double a = 6.371e6, g = 9.81, CminusA = 2.63e35, Omega = 7.292115e-5;
  double k_s = 0.0, k_s_fluid = 0.0, k_s_flat = 0.0, kTe = 0.0, hTe = 0.0;
  double dt_fe_max = 1.7976931348623157e308;
  cplx cload = 0.0;
  Deg2Channel load_ch, tidal_ch;
};
void radial_operator_tidal_rhs(const RadialOp& op, double phi_t, double* b);
void rotation_init(Rotation& rt, const Earth& e, const Mesh& m, double dt);
void rotation_begin_step(Rotation& rt, double dt);
void rotation_solve_m(Rotation& rt, const Sht& s, const double* load);
void rotation_s_rot(const Rotation& rt, const Sht& s, double* srot);
void rotation_commit(Rotation& rt);
void rotation_update(Rotation& rt, const Sht& s, const double* load, double dt);
cplx inertia21(const Sht& s, const double* load, double a);

}  // namespace orc
