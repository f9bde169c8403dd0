// Exact-product tensor-core stages of the 3-D viscosity advance (sm_100a).
//
// The pseudo-spectral stress product of advance_memory_3d
// (src/vilma_response.f90:1171-1319, transforms of src/vilma_tensor_sh.f90:168-387)
// is four dense contractions per FE sub-step (Legendre synthesis, longitude
// inverse DFT with the pointwise -M dt, longitude forward DFT, Legendre
// analysis). Here each runs on the 5th-generation tensor cores with 8-bit
// integer operands and exact 32-bit integer accumulation (tcgen05.mma
// kind::i8), by digit slicing (the Ozaki scheme):
//
//   every FP64 operand value x of a scale group g is written as a fixed-point
//   integer xi = rint(x 2^(38 - E_g)), |x| < 2^E_g (so |xi| < 2^38, inside the
//   range of five balanced digits), and xi as five signed 8-bit digits,
//   xi = sum_s d_s 256^(4 - s). A product of two such
//   values is sum_{s,t} d_s g_t 256^(8 - s - t); the digit pairs of one level
//   s + t = lambda share a weight, so each level is one int32 accumulator in
//   tensor memory, summed exactly over K. Levels 0..4 are kept (15 digit-pair
//   MMAs per K step); the dropped levels weigh < 2^-36 of |x|max |y|max per
//   term. The epilogue combines the five levels in FP64 and applies the
//   row and column scales.
//
// So the products carry ~36 significant bits relative to their operand
// groups' maxima instead of the ~22 of a two-term TF32 split, and every stage
// keeps its data in FP64 in HBM (S, Gs, dy) and applies the viscosity rates in
// FP64. Scale groups: the operand rows of one stage that come from one field
// (gather: channel x column; synthesis output: product x field, with the
// inverse stage's m / sin(theta) factor folded in; inverse output: product x
// field; forward output: product x column). Their maxima are reduced by the
// producing kernel (atomicMax on the bit pattern of non-negative doubles) and
// read by the consumer, which derives the fixed-point exponent from them.
// B operands (Legendre tables, DFT twiddles) are constant: sliced once at
// enable time with one exponent per column, laid out exactly as the shared-
// memory image of a K chunk and copied by one TMA bulk copy per chunk.
//
// Kernel shape: persistent, one CTA per SM (tensor memory: 5 levels x 2
// sub-GEMMs x 48 columns) looping over the stage's tiles, warp-specialised
// (producer of TMA bulk copies, MMA issuer, converters that slice the staged
// FP64 rows into the five digit planes in the canonical K-major no-swizzle
// layout, epilogue warps that overlap the next tile's staging); see the
// persistent kernel below.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include <cuda.h>  // CUtensorMap (encoded through the runtime's driver entry point)

#include "vg_device.cuh"
#include "vg_internal.cuh"
#include "vg_tcgen05.cuh"

namespace vg {
namespace oz {

using namespace vg::ptx;

constexpr int TM = 128;        // tile rows (MMA M)
constexpr int TN = 48;         // max columns of one sub-GEMM (MMA N)
constexpr int KC = 32;         // K per pipeline chunk = one i8 k-step
constexpr int NLEV = 5;        // digit levels kept (15 digit-pair products)
constexpr int NDIG = 5;        // 8-bit digits per operand value
constexpr int A_PLANE = TM * KC;              // bytes of one digit plane of the A chunk
constexpr int A_BYTES = NDIG * A_PLANE;
constexpr int B_BYTES_MAX = NDIG * TN * KC;
constexpr int TMEM_COLS = 512;                // 2 * NLEV * TN = 480 used
constexpr int MAX_L = 511;
constexpr int FIX_BITS = 38;                  // |xi| < 2^38: within the five digits' range [-0x8080808080, 0x7F7F7F7F7F]
constexpr unsigned long long HW_WAIT_NS = 2000000000ull;  // bound on waits for copies and MMAs
static_assert(A_BYTES % 128 == 0 && B_BYTES_MAX % 128 == 0, "ring stages stay 128-byte aligned");

enum { ST_SYNTH = 0, ST_INV = 1, ST_FWD = 2, ST_ANA = 3 };

// digit image of one (batch key, sub-GEMM, N tile) of a constant B operand
struct ImgInfo {
  long long off;  // byte offset of chunk 0: chunks of NDIG x 2 x npad x 16 bytes follow
  int kpad, npad, nvalid, kvalid;
  int sc;         // first of the image's npad column factors 2^(E_col - 6)
};

struct Args {
  // the stage's A rows as a tensor map: one TMA tile load fetches a K chunk of
  // a row tile (synthesis: X by lm pairs; inverse: S by order pairs; forward:
  // Gs; analysis: S by latitude)
  CUtensorMap tmap;
  int L, nlat, nh, nphi, half, F, NC, NCOL, nk, ne3d;
  // toroidal channels carried (1): 6 gathered channels, 12 product slots in
  // S, 10 synthesis and analysis tile types, 10 analysis outputs per slot
  int tor, nslot, ntype, nq;
  int nts, nti, ntf, nta;
  const int* kbeg;
  const int* mbeg;     // first lm of each order
  const double* X;     // [lm][4][NC]            gathered memory + 2 mu strain, lm order
  double* S;           // [M][nlat][6][NC]       synthesis products, later the analysis inputs
  double* Gs;          // [nlat][2][half][NCOL]  even / odd longitude combinations of -M dt g
  double* dy;          // [(nk + 1)][6][NC]      analysis outputs
  const double* nmdt;  // [nlat][nphi][ne3d]     -M dt (trapezoidal: -M dt / (1 + M dt / 2)) of the sub-step
  const double* invsin;
  const unsigned char* img;
  const double* bscale;
  const ImgInfo* info;
  // scale-group maxima (bits of non-negative doubles): gX [4][NC], gS [6][F],
  // gG [6][F], gA [6][NC]
  unsigned long long *gX, *gS, *gG, *gA;
  unsigned long long* status;
  unsigned long long wait_ns;
};

// ------------------------------------------------------------------ helpers

// instruction descriptor: S32 accumulate, A and B signed 8-bit, both K-major
__host__ __device__ constexpr uint32_t idesc_i8(int m, int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}

// TMA tile load of a 4-D box (no multicast, this GPU's memory), completing on
// the mbarrier's transaction count; coordinates innermost first
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(saddr(dst)),
      "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(saddr(bar))
      : "memory");
}

// 32 lanes x 8 consecutive 32-bit columns (no wait: the caller waits once)
__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, int* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}
// 32 lanes x 4 consecutive 32-bit columns (no wait)
__device__ __forceinline__ void tmem_ld4_nowait(uint32_t taddr, int* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// exponent E with |x| < 2^E for every x of a group whose maximum is `bits`
// (0 for an all-zero group), clamped so that the scale factors stay finite
__device__ __forceinline__ int group_exp(unsigned long long bits) {
  const double mx = __longlong_as_double((long long)bits);
  int e = 0;
  if (mx > 0.0 && mx <= 1.7976931348623157e308) frexp(mx, &e);
  return min(max(e, -900), 900);
}

__device__ __forceinline__ double pow2(int e) { return ldexp(1.0, e); }

// five 8-bit digit planes of sixteen values (K consecutive) of one row.
// t = fma(v, rs, 2^52 + B) with B = sum_k 128 * 256^k rounds v * rs to an
// integer xi and puts u = xi + B (0 <= u < 2^40 since |xi| < 2^38) in the low
// mantissa bits of t; digit k = byte k of u minus 128, i.e. byte k of u with
// its top bit flipped read as int8. pl[s] holds digit s (most significant
// first) of the sixteen values, four values per 32-bit word.
__device__ __forceinline__ void to_digits16(const double* v, double rs, uint4* pl) {
  constexpr double MAGIC = 4503599627370496.0 + 551911719040.0;  // 2^52 + 0x8080808080
  uint32_t w[5][4];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    uint32_t lo[4], hi[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double t = fma(v[4 * g + q], rs, MAGIC);
      lo[q] = (uint32_t)__double2loint(t);
      hi[q] = (uint32_t)__double2hiint(t);
    }
    // byte transpose of the four low words: out_b = byte b of lo[0..3]
    const uint32_t t0 = __byte_perm(lo[0], lo[1], 0x5140), t1 = __byte_perm(lo[2], lo[3], 0x5140);
    const uint32_t t2 = __byte_perm(lo[0], lo[1], 0x7362), t3 = __byte_perm(lo[2], lo[3], 0x7362);
    w[4][g] = __byte_perm(t0, t1, 0x5410) ^ 0x80808080u;  // byte 0: the least significant digit
    w[3][g] = __byte_perm(t0, t1, 0x7632) ^ 0x80808080u;
    w[2][g] = __byte_perm(t2, t3, 0x5410) ^ 0x80808080u;
    w[1][g] = __byte_perm(t2, t3, 0x7632) ^ 0x80808080u;
    const uint32_t h01 = __byte_perm(hi[0], hi[1], 0x0040), h23 = __byte_perm(hi[2], hi[3], 0x0040);
    w[0][g] = __byte_perm(h01, h23, 0x5410) ^ 0x80808080u;  // byte 4: the most significant digit
  }
#pragma unroll
  for (int s = 0; s < NDIG; ++s) pl[s] = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
}

// a signed 32-bit integer as a double, exactly: 2^52 + 2^51 + (a + 2^31)
// assembled from its bits, less the offset (one integer and one FP64 add)
__device__ __forceinline__ double i2d_exact(int a) {
  return __hiloint2double(0x43380000, a ^ (int)0x80000000) - 6755401588539392.0;
}

// exact uint32 -> FP64 (the same bit assembly, unsigned)
__device__ __forceinline__ double u2d_exact(unsigned a) {
  return __hiloint2double(0x43300000, (int)a) - 4503599627370496.0;
}

// five int32 levels (weights 256^-lambda) -> sum_s a_s 2^(32 - 8 s) times the
// power-of-two scale `sc`: the sum is formed exactly in 64-bit integers and
// rounded once (hi 2^32 + lo, both halves exact in FP64, one FMA)
__device__ __forceinline__ double combine_levels(const int* a0, const int* a1, const int* a2, const int* a3,
                                                 const int* a4, int i, double sc) {
  const long long t = ((long long)a0[i] << 32) + ((long long)a1[i] << 24) + ((long long)a2[i] << 16) +
                      ((long long)a3[i] << 8) + (long long)a4[i];
  const double hi = i2d_exact((int)(t >> 32)), lo = u2d_exact((unsigned)t);
  return fma(hi, sc * 4294967296.0, lo * sc);
}

__device__ __forceinline__ int slot_row(const int* kbeg, int l, int m, int nk) {
  return l >= 1 ? __ldg(&kbeg[l]) + m : nk;
}

// table sign under theta -> pi - theta (times (-1)^(l+m)): P, G even; dP, H odd
__device__ __forceinline__ double table_sigma(int p) { return (p == 1 || p == 5) ? -1.0 : 1.0; }
__device__ __forceinline__ int table_of(int p) {  // p -> table: 0 1 0 0 2 3
  return p == 1 ? 1 : (p == 4 ? 2 : (p == 5 ? 3 : 0));
}
__device__ __forceinline__ int chan_of(int p) { return (p == 0) ? 0 : (p <= 2 ? 1 : (p == 3 ? 2 : 3)); }

// With the toroidal channels (TOR) the synthesis has ten tile types and the
// analysis ten. Synthesis types 6-9 are the toroidal products P.X4, D.X4,
// H.X5, G.X5, written to the product slots 7, 8, 10, 11 of S: each is the
// partner (slot + 6) of the dyadic component it adds to in the inverse stage
// (rt += -i (m/sin) P.X4, rp += D.X4, tt - pp += -2 i H.X5 (slot 4's factor 2
// is applied later), tp += G.X5 (slot 5's factor 4 likewise)); slots 6 and 9
// stay zero. Analysis types 6-9 are the toroidal quadratures of the
// components rp (wD), (m/sin) rt (wP), tp (wG), tt - pp (wH).
__device__ __forceinline__ int tab_sign_idx(int table) { return (table == 1 || table == 3) ? -1 : 1; }
__device__ __forceinline__ int syn_table(int t) {  // 0 1 0 0 2 3 | 0 1 3 2
  return t < 6 ? table_of(t) : (t == 6 ? 0 : (t == 7 ? 1 : (t == 8 ? 3 : 2)));
}
__device__ __forceinline__ int syn_chan(int t) { return t < 6 ? chan_of(t) : (t < 8 ? 4 : 5); }
__device__ __forceinline__ int syn_slot(int t) { return t < 6 ? t : (t == 6 ? 7 : (t == 7 ? 8 : (t == 8 ? 10 : 11))); }
__device__ __forceinline__ int ana_table(int t) {  // 0 1 0 0 2 3 | 1 0 2 3
  return t < 6 ? table_of(t) : (t == 6 ? 1 : (t == 7 ? 0 : (t == 8 ? 2 : 3)));
}
__device__ __forceinline__ int ana_src(int t) { return t < 6 ? t : (t == 6 ? 2 : (t == 7 ? 1 : (t == 8 ? 5 : 4))); }
__device__ __forceinline__ int ana_group(int t) { return t < 6 ? t : (t == 6 ? 6 : (t == 7 ? 7 : (t == 8 ? 5 : 4))); }

struct Cta {
  int rows, row0, batch_m, p, j, nt;
  ImgInfo sub[2];
};

// ------------------------------------------------------------------ persistent kernel
//
// One CTA per SM loops over the stage's tiles (static stride). Warp roles:
//   warp 0       producer (lane 0): one TMA tile load per K chunk of the raw
//                FP64 A rows (the tile's rows x 32 K, through the stage's
//                tensor map; the analysis: two, the mirrored latitudes in the
//                second) into the raw ring, and the chunk's B digit image
//                into the B ring
//   warp 1       MMA issuer (lane 0): 15 digit-pair MMAs per chunk into the
//                five level accumulators, commits that free the chunk's A
//                and B stages, and one that hands the tile's accumulators to
//                the epilogue
//   warps 2-9    converters: raw FP64 -> five 8-bit digit planes (16 K of
//                one row per thread), zero outside the valid rows and K, the
//                CUDA-core side sums of the longitude stages
//   warps 10-17  epilogue: two per tensor-memory lane quarter, one row per
//                thread, levels combined in FP64, scaled, the stage's outputs
//                and the next stage's scale groups
// The epilogue of tile t runs while the producer and converters already
// stage tile t + 1; its accumulators are released to the MMA warp by an
// mbarrier. Handoff waits are bounded by the handle's wait limit, waits for
// copies and MMAs by a fixed bound; after an abort every copy and MMA in
// flight is waited for before the tensor memory is freed.
namespace p {
constexpr int W_PROD = 0, W_MMA = 1, W_CONV = 2, NWARP = 18;
constexpr int NTHR = NWARP * 32;
// the 16 converter + epilogue warps split NCW : 16 - NCW (a launch-time
// choice per stage, the autotuner's; every split gives the same results)
template <int NCW>
struct Roles {
  static constexpr int NCONV = NCW * 32, NEPI = (16 - NCW) * 32;
  static constexpr int W_EPI = W_CONV + NCW;
  static constexpr int NPART = (16 - NCW) / 4;  // epilogue warps per tensor-memory lane quarter
  static constexpr int GSTEP = NCONV / TM;      // a converter thread's K groups of 16: g0, g0 + GSTEP, .. < 2
  static_assert(NCW == 4 || NCW == 8, "converter warps");
};
// TWO: a raw chunk is two row boxes (the analysis: the mirrored latitudes;
// the inverse with the toroidal channels: the partner slots' rows)
template <int STAGE, bool TWO = (STAGE == ST_ANA)>
struct Ring {
  static constexpr int NRAW = TWO ? 2 : 3;  // raw FP64 chunks in flight
  static constexpr int RAW_BYTES = (TWO ? 2 : 1) * KC * TM * 8;
  static constexpr int NDST = TWO ? 2 : 4;  // A digit stages
  static constexpr int NB = 4;                          // B digit stages
  static constexpr size_t RAW_OFF = 0;
  static constexpr size_t A_OFF = RAW_OFF + (size_t)NRAW * RAW_BYTES;
  static constexpr size_t B_OFF = A_OFF + (size_t)NDST * A_BYTES;
  static constexpr size_t SUM_OFF = B_OFF + (size_t)NB * B_BYTES_MAX;  // [2 tiles][2 subs][2 halves][TM]
  static constexpr size_t BAR_OFF = SUM_OFF + 2 * 2 * 2 * TM * 8;
  static constexpr int NBAR = 2 * NRAW + 2 * NDST + 2 * NB + 2 + 4;
  static constexpr size_t BYTES = BAR_OFF + (size_t)NBAR * 8 + 16;
  static constexpr size_t SMEM = 1024 + BYTES;
};
static_assert(Ring<ST_SYNTH>::SMEM <= 227 * 1024, "synthesis ring");
static_assert(Ring<ST_ANA>::SMEM <= 227 * 1024, "analysis ring");
static_assert(Ring<ST_INV, true>::SMEM <= 227 * 1024, "inverse ring with the toroidal partner rows");
static_assert(Ring<ST_SYNTH>::SMEM > 114 * 1024 && Ring<ST_ANA>::SMEM > 114 * 1024,
              "one CTA per SM: the tensor-memory plan takes 480 of its 512 columns");
}  // namespace p

template <int STAGE, bool TOR>
__device__ __forceinline__ int tile_count(const Args& A) {
  constexpr int NTY = TOR ? 10 : 6;
  if (STAGE == ST_SYNTH) return ((A.NC + TM - 1) / TM) * A.nts * (A.L + 1) * NTY;
  if (STAGE == ST_ANA) return ((A.NC + TM - 1) / TM) * A.nta * (A.L + 1) * NTY;
  if (STAGE == ST_INV) return ((A.NCOL + TM - 1) / TM) * A.nti * A.nlat;
  return ((A.NCOL + TM - 1) / TM) * A.ntf * A.nlat;
}

// tile t -> (row tile, N tile, batch): the row tile fastest, so the CTAs that
// share a batch's B images and A rows run close together
template <int STAGE, bool TOR>
__device__ __forceinline__ Cta tile_info(const Args& A, int t) {
  constexpr int NTY = TOR ? 10 : 6;
  Cta c;
  const int rt_n = (STAGE == ST_SYNTH || STAGE == ST_ANA) ? (A.NC + TM - 1) / TM : (A.NCOL + TM - 1) / TM;
  const int nt_count = STAGE == ST_SYNTH ? A.nts : (STAGE == ST_ANA ? A.nta : (STAGE == ST_INV ? A.nti : A.ntf));
  const int rt = t % rt_n, rest = t / rt_n;
  c.nt = rest % nt_count;
  const int bz = rest / nt_count;
  c.row0 = rt * TM;
  if (STAGE == ST_SYNTH || STAGE == ST_ANA) {
    c.batch_m = bz / NTY;
    c.p = bz % NTY;
    c.j = 0;
    c.rows = min(TM, A.NC - c.row0);
    const int tab = !TOR ? table_of(c.p) : (STAGE == ST_SYNTH ? syn_table(c.p) : ana_table(c.p));
    const int base = ((c.batch_m * 4 + tab) * 2) * nt_count;
    c.sub[0] = A.info[base + c.nt];
    c.sub[1] = A.info[base + nt_count + c.nt];
  } else {
    c.batch_m = 0;
    c.p = 0;
    c.j = bz;
    c.rows = min(TM, A.NCOL - c.row0);
    c.sub[0] = A.info[c.nt];
    c.sub[1] = A.info[nt_count + c.nt];
  }
  return c;
}

// the group exponent of a tile row (analysis rows: + 1, the E / O bound)
template <int STAGE, bool TOR>
__device__ __forceinline__ int row_exp(const Args& A, const Cta& c, int row) {
  if (STAGE == ST_SYNTH) return group_exp(A.gX[(TOR ? syn_chan(c.p) : chan_of(c.p)) * A.NC + row]);
  if (STAGE == ST_INV) {  // rows (p, f) = p F + f; with the toroidal channels plus the partner slot's bound
    if (!TOR) return group_exp(A.gS[row]);
    const double s = __longlong_as_double((long long)A.gS[row]) +
                     __longlong_as_double((long long)A.gS[row + 6 * A.F]);
    return group_exp((unsigned long long)__double_as_longlong(s));
  }
  if (STAGE == ST_FWD) return group_exp(A.gG[row]);
  return group_exp(A.gA[(TOR ? ana_group(c.p) : c.p) * A.NC + row]) + 1;
}

// K values of chunk (sub, kc) with data: K index k of the chunk is valid if
// k < valid_k(...) (synthesis: l = m + sub + 2 kk <= L; inverse: m <= L, two K
// per order; forward: i < half; analysis: j < nh)
template <int STAGE>
__device__ __forceinline__ int valid_k(const Args& A, const Cta& c, int sub, int kc) {
  int kmax;
  if (STAGE == ST_SYNTH) {
    kmax = (A.L - c.batch_m - sub) >= 0 ? (A.L - c.batch_m - sub) / 2 + 1 : 0;
  } else if (STAGE == ST_INV) {
    const int m0 = sub ? 1 : 2;
    kmax = 2 * ((A.L - m0) >= 0 ? (A.L - m0) / 2 + 1 : 0);
  } else if (STAGE == ST_FWD) {
    kmax = A.half;
  } else {
    kmax = A.nh;
  }
  return max(0, min(KC, kmax - kc * KC));
}

template <int STAGE, int NCW, bool TOR = false>
__global__ void __launch_bounds__(p::NTHR, 1) k_ozp_stage(const __grid_constant__ Args A) {
  using R = p::Ring<STAGE, STAGE == ST_ANA || (STAGE == ST_INV && TOR)>;
  using Q = p::Roles<NCW>;
  constexpr int NSL = TOR ? 12 : 6, NQO = TOR ? 10 : 6;  // product slots of S, analysis outputs per slot
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  unsigned char* raw = sm + R::RAW_OFF;
  unsigned char* adig = sm + R::A_OFF;
  unsigned char* bdig = sm + R::B_OFF;
  double* rsum = (double*)(sm + R::SUM_OFF);
  uint64_t* bar = (uint64_t*)(sm + R::BAR_OFF);
  uint64_t* raw_full = bar;
  uint64_t* raw_empty = raw_full + R::NRAW;
  uint64_t* a_full = raw_empty + R::NRAW;
  uint64_t* a_empty = a_full + R::NDST;
  uint64_t* b_full = a_empty + R::NDST;
  uint64_t* b_empty = b_full + R::NB;
  uint64_t* acc_full = b_empty + R::NB;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* sum_full = acc_empty + 1;  // [2]
  uint64_t* sum_empty = sum_full + 2;  // [2]
  uint32_t* tslot = (uint32_t*)(bar + R::NBAR);
  volatile int* abort_flag = (volatile int*)(tslot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntile = tile_count<STAGE, TOR>(A);
  constexpr bool SIDE = (STAGE == ST_INV || STAGE == ST_FWD);

  if (tid == 0) {
    for (int i = 0; i < R::NRAW; ++i) {
      mbar_init(&raw_full[i], 1);
      mbar_init(&raw_empty[i], Q::NCONV);
    }
    for (int i = 0; i < R::NDST; ++i) {
      mbar_init(&a_full[i], Q::NCONV);
      mbar_init(&a_empty[i], 1);
    }
    for (int i = 0; i < R::NB; ++i) {
      mbar_init(&b_full[i], 1);
      mbar_init(&b_empty[i], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, Q::NEPI);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&sum_full[i], Q::NCONV);
      mbar_init(&sum_empty[i], Q::NEPI);
    }
    fence_mbar_init();
    *abort_flag = 0;
  }
  if (warp == p::W_PROD) tmem_alloc(tslot, TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  if (warp == p::W_PROD) {
    // ------------------------------------------------------------ producer
    // every lane takes the same path: lane 0 waits, the result is broadcast
    int gc = 0;       // chunks issued
    int last_b = -1;  // B copies issued: chunk ids 0 .. last_b (for the exit wait)
    bool stop = false;
    for (int t = blockIdx.x; t < ntile && !stop; t += gridDim.x) {
      const Cta c = tile_info<STAGE, TOR>(A, t);
      const int nch0 = c.sub[0].kpad / KC, nch = nch0 + c.sub[1].kpad / KC;
      if (nch == 0 || c.rows <= 0) continue;
      for (int ch = 0; ch < nch; ++ch, ++gc) {
        const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
        const int rs = gc % R::NRAW, bs = gc % R::NB;
        int ok = 1;
        if (lane == 0) {
          if (gc >= R::NRAW &&
              !mbar_wait_or_abort_ns(&raw_empty[rs], (uint32_t)((gc / R::NRAW - 1) & 1), abort_flag, A.wait_ns))
            ok = 0;
          if (ok && gc >= R::NB &&
              !mbar_wait_or_abort_ns(&b_empty[bs], (uint32_t)((gc / R::NB - 1) & 1), abort_flag, A.wait_ns))
            ok = 0;
          if (!ok) {
            atomicOr(A.status, 1ull << (24 + STAGE));
            *abort_flag = 1;
          }
        }
        if (!__shfl_sync(0xffffffffu, ok, 0)) {
          stop = true;
          break;
        }
        // raw rows of this chunk: one TMA tile load of the row tile's 32 K
        // (the analysis: a second one for the mirrored latitudes, stored in
        // reverse order); rows past the tile's end and K past the tensor read
        // as zeros, K past the valid range is zeroed by the converters
        if (lane == 0) {
          unsigned char* rdst = raw + (size_t)rs * R::RAW_BYTES;
          if (STAGE == ST_SYNTH) {
            // lm = mbeg[m] + sub + 2 kk = 2 q + par
            const int lm0 = __ldg(&A.mbeg[c.batch_m]) + sub + 2 * kc * KC;
            mbar_expect_tx(&raw_full[rs], (uint32_t)R::RAW_BYTES);
            tma_load_4d(rdst, &A.tmap, c.row0, TOR ? syn_chan(c.p) : chan_of(c.p), lm0 & 1, lm0 >> 1, &raw_full[rs]);
          } else if (STAGE == ST_INV) {
            // m = 2 mq + mpar: even orders from 2 (sub 0), odd orders from 1 (sub 1)
            const int mq0 = (sub ? 0 : 1) + kc * (KC / 2);
            mbar_expect_tx(&raw_full[rs], (uint32_t)R::RAW_BYTES);
            tma_load_4d(rdst, &A.tmap, 2 * c.row0, c.j, sub, mq0, &raw_full[rs]);
            if (TOR && STAGE == ST_INV)  // the partner slots' rows (6 F further), after the tile's own
              tma_load_4d(rdst + (size_t)KC * TM * 8, &A.tmap, 2 * (c.row0 + 6 * A.F), c.j, sub, mq0, &raw_full[rs]);
          } else if (STAGE == ST_FWD) {
            mbar_expect_tx(&raw_full[rs], (uint32_t)R::RAW_BYTES);
            tma_load_4d(rdst, &A.tmap, c.row0, kc * KC, 2 * c.j + sub, 0, &raw_full[rs]);
          } else {
            const int j0 = kc * KC, jm0 = A.nlat - KC - j0;  // mirrors of j0 .. j0 + 31, ascending
            mbar_expect_tx(&raw_full[rs], (uint32_t)R::RAW_BYTES);
            tma_load_4d(rdst, &A.tmap, c.row0, TOR ? ana_src(c.p) : c.p, j0, c.batch_m, &raw_full[rs]);
            tma_load_4d(rdst + (size_t)KC * TM * 8, &A.tmap, c.row0, TOR ? ana_src(c.p) : c.p, jm0, c.batch_m, &raw_full[rs]);
          }
        }
        __syncwarp();
        // the chunk's B digit image
        if (lane == 0) {
          const ImgInfo I = sub ? c.sub[1] : c.sub[0];
          const uint32_t bytes = (uint32_t)(NDIG * 2 * I.npad * 16);
          mbar_expect_tx(&b_full[bs], bytes);
          bulk_g2s(bdig + (size_t)bs * B_BYTES_MAX, A.img + I.off + (size_t)kc * bytes, bytes, &b_full[bs]);
        }
        last_b = gc;
        __syncwarp();
      }
    }
    // copies still in flight (after an abort): wait for the last ones of each ring
    if (lane == 0) {
      for (int q = max(0, gc - R::NRAW); q < gc; ++q)
        if (!mbar_wait_ns(&raw_full[q % R::NRAW], (uint32_t)((q / R::NRAW) & 1), HW_WAIT_NS))
          atomicOr(A.status, 1ull << (20 + STAGE));
      for (int q = max(0, last_b + 1 - R::NB); q <= last_b; ++q)
        if (!mbar_wait_ns(&b_full[q % R::NB], (uint32_t)((q / R::NB) & 1), HW_WAIT_NS))
          atomicOr(A.status, 1ull << (20 + STAGE));
    }
    __syncwarp();
  } else if (warp == p::W_MMA) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      int gc = 0, gt = 0;
      bool stop = false;
      for (int t = blockIdx.x; t < ntile && !stop; t += gridDim.x) {
        const Cta c = tile_info<STAGE, TOR>(A, t);
        const int nch0 = c.sub[0].kpad / KC, nch = nch0 + c.sub[1].kpad / KC;
        if (nch == 0 || c.rows <= 0) continue;
        // the epilogue has read the previous tile's accumulators
        if (gt >= 1 && !mbar_wait_or_abort_ns(acc_empty, (uint32_t)((gt - 1) & 1), abort_flag, A.wait_ns)) {
          atomicOr(A.status, 1ull << (28 + STAGE));
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        for (int ch = 0; ch < nch; ++ch, ++gc) {
          const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
          const int ds = gc % R::NDST, bs = gc % R::NB;
          if (!mbar_wait_or_abort_ns(&a_full[ds], (uint32_t)((gc / R::NDST) & 1), abort_flag, A.wait_ns) ||
              !mbar_wait_or_abort_ns(&b_full[bs], (uint32_t)((gc / R::NB) & 1), abort_flag, HW_WAIT_NS)) {
            atomicOr(A.status, 1ull << (28 + STAGE));
            *abort_flag = 1;
            stop = true;
            break;
          }
          tc_fence_after();
          const ImgInfo I = sub ? c.sub[1] : c.sub[0];
          const unsigned char* Ab = adig + (size_t)ds * A_BYTES;
          const unsigned char* Bb = bdig + (size_t)bs * B_BYTES_MAX;
          const uint32_t idesc = idesc_i8(TM, I.npad);
#pragma unroll
          for (int s = 0; s < NDIG; ++s) {
            const uint64_t da = sdesc(saddr(Ab + s * A_PLANE), TM * 16, 128);
#pragma unroll
            for (int u = 0; u < NLEV - s; ++u) {
              const uint64_t db = sdesc(saddr(Bb + u * 2 * I.npad * 16), I.npad * 16, 128);
              const uint32_t d = tmem + (uint32_t)(((s + u) * 2 + sub) * TN);
              mma_i8(d, da, db, idesc, (kc > 0 || s > 0) ? 1u : 0u);
            }
          }
          mma_commit(&a_empty[ds]);
          mma_commit(&b_empty[bs]);
        }
        if (stop) break;
        mma_commit(acc_full);  // every MMA of the tile
        ++gt;
      }
      // drain: the last commit completes once every MMA issued has
      if (gc > 0 && !mbar_wait_ns(&a_empty[(gc - 1) % R::NDST], (uint32_t)(((gc - 1) / R::NDST) & 1), HW_WAIT_NS))
        atomicOr(A.status, 1ull << (16 + STAGE));
    }
    __syncwarp();
  } else if (warp < Q::W_EPI) {
    // ------------------------------------------------------------ converters
    const int ct = tid - p::W_CONV * 32;  // 0 .. NCONV - 1
    const int lr = ct % TM, g0 = ct / TM;  // row, first K group of 16
    int gc = 0, gt = 0;
    for (int t = blockIdx.x; t < ntile && !*abort_flag; t += gridDim.x) {
      const Cta c = tile_info<STAGE, TOR>(A, t);
      const int nch0 = c.sub[0].kpad / KC, nch = nch0 + c.sub[1].kpad / KC;
      if (nch == 0 || c.rows <= 0) continue;
      const bool live = lr < c.rows;
      const int row = c.row0 + lr;
      const int e = live ? row_exp<STAGE, TOR>(A, c, row) : 0;
      const double rs = pow2(FIX_BITS - e);
      const double is_j = (STAGE == ST_INV) ? A.invsin[c.j] : 0.0;
      const int prow = (STAGE == ST_INV) ? row / A.F : 0;
      // the tile's side sums (sub 0, sub 1) of this thread's first and second K group
      double side0a = 0.0, side0b = 0.0, side1a = 0.0, side1b = 0.0;
      bool ok = true;
      for (int ch = 0; ch < nch; ++ch, ++gc) {
        const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
        const int rsi = gc % R::NRAW, ds = gc % R::NDST;
        if (!mbar_wait_sleep_ns(&raw_full[rsi], (uint32_t)((gc / R::NRAW) & 1), abort_flag, HW_WAIT_NS) ||
            (gc >= R::NDST &&
             !mbar_wait_sleep_ns(&a_empty[ds], (uint32_t)((gc / R::NDST - 1) & 1), abort_flag, A.wait_ns))) {
          atomicOr(A.status, 1ull << (24 + STAGE));
          *abort_flag = 1;
          ok = false;
          break;
        }
        const int kv = valid_k<STAGE>(A, c, sub, kc);
        const double* rv = (const double*)(raw + (size_t)rsi * R::RAW_BYTES);
#pragma unroll 1
        for (int it = 0; it < 2 / Q::GSTEP; ++it) {
          const int g = g0 + it * Q::GSTEP;
          double v[16];
          double sacc = 0.0;  // this chunk's part of the side sum
          if (STAGE == ST_INV) {
            // K pairs (re, im) of one order: one 16-byte load per pair
#pragma unroll
            for (int q = 0; q < 16; q += 2) {
              const int k = 16 * g + q, mo = k >> 1;
              double tre = 0.0, tim = 0.0;
              if (live && k < kv) {
                const double2 z = *reinterpret_cast<const double2*>(rv + (size_t)mo * TM * 2 + 2 * lr);
                tre = z.x;
                tim = z.y;
                if (prow == 2) {  // i (m / sin theta) z
                  const int m = (sub ? 1 : 2) + 2 * (kc * (KC / 2) + mo);
                  const double a = (double)m * is_j;
                  tre = -a * z.y;
                  tim = a * z.x;
                } else if (prow == 5) {  // i z
                  tre = -z.y;
                  tim = z.x;
                }
                if (TOR) {  // the partner slot: rt -= i (m/sin) P.X4, rp += D.X4, (tt - pp) -= i H.X5, tp += G.X5 / 4
                  const double2 w = *reinterpret_cast<const double2*>(rv + (size_t)KC * TM + (size_t)mo * TM * 2 + 2 * lr);
                  if (prow == 1) {
                    const int m = (sub ? 1 : 2) + 2 * (kc * (KC / 2) + mo);
                    const double a = (double)m * is_j;
                    tre += a * w.y;
                    tim -= a * w.x;
                  } else if (prow == 2) {
                    tre += w.x;
                    tim += w.y;
                  } else if (prow == 4) {
                    tre += w.y;
                    tim -= w.x;
                  } else if (prow == 5) {
                    tre += 0.25 * w.x;
                    tim += 0.25 * w.y;
                  }
                }
                sacc += 2.0 * tre;
              }
              v[q] = tre;
              v[q + 1] = (k + 1 < kv && live) ? tim : 0.0;
            }
          } else {
            const double sg = (STAGE == ST_ANA) ? (TOR ? (double)tab_sign_idx(ana_table(c.p)) : table_sigma(c.p)) * (sub ? -1.0 : 1.0) : 0.0;
            // with the toroidal channels the forward stage leaves rp without its m / sin theta: types 2
            // ((m/sin) rp) and 7 ((m/sin) rt) apply it here, per latitude (the mirror has the same sin)
            const bool msf = (STAGE == ST_ANA) && TOR && (c.p == 2 || c.p == 7);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
              const int k = 16 * g + q;
              double x = 0.0;
              if (live && k < kv) {
                if (STAGE == ST_ANA) {
                  const int j = kc * KC + k, jm = A.nlat - 1 - j;
                  const double r0 = rv[(size_t)k * TM + lr];
                  const double r1 = (jm != j) ? rv[(size_t)(KC + KC - 1 - k) * TM + lr] : 0.0;
                  x = r0 + sg * r1;
                  if (msf) x *= (double)c.batch_m * __ldg(&A.invsin[j]);
                } else {
                  x = rv[(size_t)k * TM + lr];
                  if (STAGE == ST_FWD) sacc += x;
                }
              }
              v[q] = x;
            }
          }
          if (sub) {
            if (it)
              side1b += sacc;
            else
              side1a += sacc;
          } else {
            if (it)
              side0b += sacc;
            else
              side0a += sacc;
          }
          uint4 pl[NDIG];
          to_digits16(v, rs, pl);
          unsigned char* Ab = adig + (size_t)ds * A_BYTES + ((size_t)g * TM + lr) * 16;
#pragma unroll
          for (int s = 0; s < NDIG; ++s) *reinterpret_cast<uint4*>(Ab + s * A_PLANE) = pl[s];
        }
        fence_async_smem();
        mbar_arrive(&a_full[ds]);
        mbar_arrive(&raw_empty[rsi]);
      }
      if (!ok) break;
      if (SIDE) {  // the tile's side sums, for its epilogue
        const int tb = gt & 1;
        if (gt >= 2 &&
            !mbar_wait_sleep_ns(&sum_empty[tb], (uint32_t)(((gt >> 1) - 1) & 1), abort_flag, A.wait_ns)) {
          atomicOr(A.status, 1ull << (24 + STAGE));
          *abort_flag = 1;
          break;
        }
        rsum[((tb * 2 + 0) * 2 + g0) * TM + lr] = side0a;
        rsum[((tb * 2 + 1) * 2 + g0) * TM + lr] = side1a;
        if (Q::GSTEP == 1) {
          rsum[((tb * 2 + 0) * 2 + 1) * TM + lr] = side0b;
          rsum[((tb * 2 + 1) * 2 + 1) * TM + lr] = side1b;
        }
        mbar_arrive(&sum_full[tb]);
      }
      ++gt;
    }
  } else {
    // ------------------------------------------------------------ epilogue
    // tcgen05.ld is warp-collective: lane 0 waits, the result is broadcast
    const int ew = warp - Q::W_EPI;  // 0 .. NEPI / 32 - 1
    const int quad = warp & 3, part = ew >> 2;  // lane quarter, column part
    const int r = quad * 32 + lane;
    const uint32_t tbase = tmem + ((uint32_t)(quad * 32) << 16);
    int gt = 0;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
      const Cta c = tile_info<STAGE, TOR>(A, t);
      const int nch0 = c.sub[0].kpad / KC, nch1 = c.sub[1].kpad / KC;
      if (nch0 + nch1 == 0 || c.rows <= 0) continue;
      int ok = 1;
      if (lane == 0) {
        if (!mbar_wait_sleep_ns(acc_full, (uint32_t)(gt & 1), abort_flag, A.wait_ns)) ok = 0;
        if (ok && SIDE &&
            !mbar_wait_sleep_ns(&sum_full[gt & 1], (uint32_t)((gt >> 1) & 1), abort_flag, A.wait_ns))
          ok = 0;
        if (!ok) {
          atomicOr(A.status, 1ull << (28 + STAGE));
          *abort_flag = 1;
        }
      }
      if (!__shfl_sync(0xffffffffu, ok, 0)) break;
      tc_fence_after();
      double sev = 0.0, sod = 0.0;
      if (SIDE) {
        const int tb = gt & 1;
        sev = rsum[((tb * 2 + 0) * 2 + 0) * TM + r] + rsum[((tb * 2 + 0) * 2 + 1) * TM + r];
        sod = rsum[((tb * 2 + 1) * 2 + 0) * TM + r] + rsum[((tb * 2 + 1) * 2 + 1) * TM + r];
        mbar_arrive(&sum_empty[tb]);
      }
      const int row = c.row0 + r;
      const bool live = r < c.rows;
      const bool has0 = nch0 > 0, has1 = nch1 > 0;
      const int npad_max = max(has0 ? c.sub[0].npad : 0, has1 ? c.sub[1].npad : 0);
      const double rf = pow2((live ? row_exp<STAGE, TOR>(A, c, row) : 0) - FIX_BITS);
      auto load_block = [&](int sub, int cb, double* out) {
        const bool hs = sub ? has1 : has0;
        const int np = sub ? c.sub[1].npad : c.sub[0].npad;
        if (!hs || cb >= np) {
#pragma unroll
          for (int i = 0; i < 8; ++i) out[i] = 0.0;
          return;
        }
        int a[NLEV][8];
#pragma unroll
        for (int lv = 0; lv < NLEV; ++lv) tmem_ld8_nowait(tbase + (uint32_t)((lv * 2 + sub) * TN + cb), a[lv]);
        tmem_wait_ld();
        const double* cs = A.bscale + (sub ? c.sub[1].sc : c.sub[0].sc) + cb;
#pragma unroll
        for (int i = 0; i < 8; ++i) out[i] = combine_levels(a[0], a[1], a[2], a[3], a[4], i, rf) * __ldg(&cs[i]);
      };
      // both parities of 4 columns: the tensor-memory loads are issued first,
      // the stage's scattered global loads (rates, 1 / sin) run in their
      // shadow, then one wait
      auto issue_pair4 = [&](int cb, int (*a)[NLEV][4]) {
#pragma unroll
        for (int sb = 0; sb < 2; ++sb)
#pragma unroll
          for (int lv = 0; lv < NLEV; ++lv) tmem_ld4_nowait(tbase + (uint32_t)((lv * 2 + sb) * TN + cb), a[sb][lv]);
      };
      // the combined levels times the column scales (a few values every thread
      // reads: cache hits); columns past a parity's image read as zero
      auto combine_pair4 = [&](int cb, int (*a)[NLEV][4], double* ev, double* od) {
        const bool ok0 = has0 && cb < c.sub[0].npad, ok1 = has1 && cb < c.sub[1].npad;
        const double* cs0 = A.bscale + c.sub[0].sc + cb;
        const double* cs1 = A.bscale + c.sub[1].sc + cb;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          ev[i] = ok0 ? combine_levels(a[0][0], a[0][1], a[0][2], a[0][3], a[0][4], i, rf) * __ldg(&cs0[i]) : 0.0;
          od[i] = ok1 ? combine_levels(a[1][0], a[1][1], a[1][2], a[1][3], a[1][4], i, rf) * __ldg(&cs1[i]) : 0.0;
        }
      };
      if (STAGE == ST_SYNTH) {
        const int m = c.batch_m, pp = TOR ? syn_slot(c.p) : c.p;  // the product slot
        const double sg = TOR ? (double)tab_sign_idx(syn_table(c.p)) : table_sigma(c.p);
        // the group weights: the inverse stage's factor on this slot (m / sin theta on slots 2 and 7,
        // 1 / 4 on slot 11)
        const bool wms = (pp == 2 || (TOR && pp == 7));
        const double wq = (TOR && pp == 11) ? 0.25 : 1.0;
        double gmax = 0.0;
        for (int cb = part * 4; cb < npad_max; cb += 4 * Q::NPART) {
          int a[2][NLEV][4];
          double wn[4], ws[4];
          issue_pair4(cb, a);
          tmem_wait_ld();
          if (!live) continue;
#pragma unroll
          for (int i = 0; i < 4; ++i) {  // the weights of the group maximum (m / sin theta for p = 2)
            const int j = min(c.nt * TN + cb + i, A.nh - 1), jm = A.nlat - 1 - j;
            wn[i] = wms ? (double)m * __ldg(&A.invsin[j]) : 1.0;
            ws[i] = wms ? (double)m * __ldg(&A.invsin[jm]) : 1.0;
          }
          double ev[4], od[4];
          combine_pair4(cb, a, ev, od);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int j = c.nt * TN + cb + i;
            if (j < A.nh) {
              const int jm = A.nlat - 1 - j;
              const double vn = ev[i] + od[i];
              A.S[(((size_t)m * A.nlat + j) * NSL + pp) * A.NC + row] = vn;
              gmax = fmax(gmax, fabs(vn) * wn[i]);
              if (jm != j) {
                const double vs = sg * (ev[i] - od[i]);
                A.S[(((size_t)m * A.nlat + jm) * NSL + pp) * A.NC + row] = vs;
                gmax = fmax(gmax, fabs(vs) * ws[i]);
              }
            }
          }
        }
        if (live) atomic_max_bits(&A.gS[pp * A.F + row / 2], gmax * wq);
      } else if (STAGE == ST_INV) {
        const int pp = row / A.F, f = row % A.F, e3 = f / 3;
        double c0 = 0.0;  // m = 0 term (weight 1), the real part of z_0 (and of the partner slot's share)
        if (live && pp != 2) {
          const double2 z =
              *reinterpret_cast<const double2*>(A.S + (((size_t)0 * A.nlat + c.j) * NSL + pp) * A.NC + 2 * f);
          c0 = (pp == 5) ? -z.y : z.x;
        }
        if (live && TOR) {
          const double2 w =
              *reinterpret_cast<const double2*>(A.S + (((size_t)0 * A.nlat + c.j) * NSL + pp + 6) * A.NC + 2 * f);
          c0 += (pp == 2) ? w.x : (pp == 4 ? w.y : (pp == 5 ? 0.25 * w.x : 0.0));
        }
        const double* nm_j = A.nmdt + (size_t)c.j * A.nphi * A.ne3d + e3;
        double* gs = A.Gs + (size_t)c.j * 2 * A.half * A.NCOL + row;
        double* gd = gs + (size_t)A.half * A.NCOL;
        double gmax = 0.0;
        // longitudes i and i + half from the even / odd parts, times -M dt there
        auto emit = [&](int i, double ev, double od, double n1, double n2) {
          const double g1 = n1 * (ev + od);
          const double g2 = n2 * (ev - od);
          const double sv = g1 + g2, dv = g1 - g2;
          gs[(size_t)i * A.NCOL] = sv;
          gd[(size_t)i * A.NCOL] = dv;
          gmax = fmax(gmax, fmax(fabs(sv), fabs(dv)));
        };
        if (live && c.nt == 0 && part == 0)
          emit(0, c0 + sev, sod, __ldg(&nm_j[0]), __ldg(&nm_j[(size_t)A.half * A.ne3d]));
        for (int cb = part * 4; cb < npad_max; cb += 4 * Q::NPART) {
          int a[2][NLEV][4];
          double n1[4], n2[4];
          issue_pair4(cb, a);
          tmem_wait_ld();
          if (!live) continue;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int ii = min(1 + c.nt * TN + cb + i, A.half - 1);
            n1[i] = __ldg(&nm_j[(size_t)ii * A.ne3d]);
            n2[i] = __ldg(&nm_j[(size_t)(ii + A.half) * A.ne3d]);
          }
          double ev[4], od[4];
          combine_pair4(cb, a, ev, od);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int ii = 1 + c.nt * TN + cb + i;
            if (ii < A.half) emit(ii, ev[i] + c0, od[i], n1[i], n2[i]);
          }
        }
        if (live) atomic_max_bits(&A.gG[row], gmax);
      } else if (STAGE == ST_FWD) {
        const int pp = row / A.F, f = row % A.F;
        const double isj = A.invsin[c.j];
        const double beta_c = (pp == 3 || pp == 4) ? 2.0 : (pp == 5 ? 4.0 : 1.0);
        auto out = [&](int m) -> double2* {
          return reinterpret_cast<double2*>(A.S + (((size_t)m * A.nlat + c.j) * NSL + pp) * A.NC + 2 * f);
        };
        // with the toroidal channels rp is stored without m / sin theta (the analysis applies it) and
        // rp, rt carry a second scale group: plain rp (type 6) and (m/sin) rt (type 7)
        const bool tor2 = TOR && pp == 2, tor1 = TOR && pp == 1;
        double gre = 0.0, gim = 0.0, hre = 0.0, him = 0.0;  // hre, him: the second group
        if (live && c.nt == 0 && part == 0) {
          // m = 0: F_0 = (2 pi / nphi) sum_i s_i, real
          const double v = (pp == 2 && !tor2) ? 0.0 : beta_c * sev * (2.0 * PI / (double)A.nphi);
          *out(0) = make_double2(v, 0.0);
          if (tor2)
            hre = fabs(v);  // (m/sin) rp is zero at m = 0
          else
            gre = fabs(v);
        }
        for (int sub = 0; sub < 2; ++sub) {
          if (!(sub ? has1 : has0)) continue;
          const int npad = sub ? c.sub[1].npad : c.sub[0].npad, nval = sub ? c.sub[1].nvalid : c.sub[0].nvalid;
          for (int cb = part * 8; cb < npad; cb += 8 * Q::NPART) {
            double v[8];
            load_block(sub, cb, v);
            if (!live) continue;
#pragma unroll
            for (int i = 0; i < 8; i += 2) {
              const int kk = c.nt * TN + cb + i;  // (m, re) column; (m, im) follows
              if (kk >= c.nt * TN + nval) break;
              const int m = (sub ? 1 : 2) + 2 * (kk >> 1);
              const double ms = (double)m * isj;
              const double beta = (pp == 2 && !tor2) ? ms : beta_c;
              const double re = beta * v[i], im = beta * v[i + 1];
              *out(m) = make_double2(re, im);
              if (tor2) {  // type 2 groups (m/sin) rp, type 6 plain rp
                gre = fmax(gre, fabs(ms * re));
                gim = fmax(gim, fabs(ms * im));
                hre = fmax(hre, fabs(re));
                him = fmax(him, fabs(im));
              } else {
                gre = fmax(gre, fabs(re));
                gim = fmax(gim, fabs(im));
                if (tor1) {  // type 7 groups (m/sin) rt
                  hre = fmax(hre, fabs(ms * re));
                  him = fmax(him, fabs(ms * im));
                }
              }
            }
          }
        }
        if (live) {
          atomic_max_bits(&A.gA[pp * A.NC + 2 * f], gre);
          atomic_max_bits(&A.gA[pp * A.NC + 2 * f + 1], gim);
          if (tor1 || tor2) {
            const int g2 = tor2 ? 6 : 7;
            atomic_max_bits(&A.gA[g2 * A.NC + 2 * f], hre);
            atomic_max_bits(&A.gA[g2 * A.NC + 2 * f + 1], him);
          }
        }
      } else {
        const int m = c.batch_m, pp = c.p;
        for (int sub = 0; sub < 2; ++sub) {
          if (!(sub ? has1 : has0)) continue;
          const int npad = sub ? c.sub[1].npad : c.sub[0].npad;
          for (int cb = part * 8; cb < npad; cb += 8 * Q::NPART) {
            double v[8];
            load_block(sub, cb, v);
            if (!live) continue;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const int kk = c.nt * TN + cb + i;
              const int l = m + sub + 2 * kk;
              if (l > A.L) break;
              A.dy[((size_t)slot_row(A.kbeg, l, m, A.nk) * NQO + pp) * A.NC + row] = v[i];
            }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(acc_empty);
      ++gt;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == p::W_PROD) tmem_dealloc(tmem, TMEM_COLS);
}

// -M dt of every (latitude, longitude, element) for one sub-step (trapezoidal:
// the implicit half-step factor M dt / (1 + M dt / 2)), negated
__global__ void k_oz_rate_factors(const double* __restrict__ rate, double* __restrict__ nm, size_t n, double dt,
                                  int trap) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double m = rate[i] * dt;
    if (trap) m = m / (1.0 + 0.5 * m);
    nm[i] = -m;
  }
}

// ------------------------------------------------------------------ operand images

struct ImgJob {
  int kind;  // 0 synth table, 1 analysis table, 2 inverse twiddle, 3 forward twiddle
  int table, m, par, n0;
  ImgInfo info;
};

__device__ double img_value(const ImgJob& J, int k, int n, const double* const* tabs, int L, int nlat, int nphi) {
  if (n >= J.info.nvalid || k >= J.info.kvalid) return 0.0;
  const double two_pi = 2.0 * PI;
  if (J.kind == 0) {  // B[kk][j] = T(l = m + par + 2 kk, m; j)
    const int j = J.n0 + n, l = J.m + J.par + 2 * k;
    const int lm = J.m * (L + 1) - J.m * (J.m - 1) / 2 + (l - J.m);
    return tabs[J.table][(size_t)lm * nlat + j];
  }
  if (J.kind == 1) {  // B[j][kk] = Tw(l = m + par + 2 kk, m; j)
    const int l = J.m + J.par + 2 * (J.n0 + n), j = k;
    const int lm = J.m * (L + 1) - J.m * (J.m - 1) / 2 + (l - J.m);
    return tabs[4 + J.table][(size_t)lm * nlat + j];
  }
  if (J.kind == 2) {  // B[(m, ri)][i] = 2 cos(m phi_i), -2 sin(m phi_i)
    const int i = 1 + J.n0 + n, m = (J.par ? 1 : 2) + 2 * (k >> 1);
    const int t_ = (int)(((long long)m * i) % nphi);
    const double ang = two_pi * (double)t_ / (double)nphi;
    return (k & 1) ? -2.0 * sin(ang) : 2.0 * cos(ang);
  }
  // B[i][(m, ri)] = (2 pi / nphi) (cos(m phi_i), -sin(m phi_i))
  const int kk = J.n0 + n, i = k, m = (J.par ? 1 : 2) + 2 * (kk >> 1);
  const int t_ = (int)(((long long)m * i) % nphi);
  const double ang = two_pi * (double)t_ / (double)nphi, scl = two_pi / (double)nphi;
  return (kk & 1) ? -scl * sin(ang) : scl * cos(ang);
}

// One CTA per image: per column the exponent of its largest entry, then every
// entry's five digits at [chunk][digit][K group][n][16 bytes], and the
// column factors 2^(E - 6) the epilogue applies.
__global__ void k_oz_images(const ImgJob* __restrict__ jobs, unsigned char* __restrict__ img,
                            double* __restrict__ bscale, const double* const* tabs, int L, int nlat, int nphi) {
  __shared__ int s_exp[TN];
  const ImgJob J = jobs[blockIdx.x];
  const int kpad = J.info.kpad, npad = J.info.npad;
  for (int n = threadIdx.x; n < npad; n += blockDim.x) {
    double mx = 0.0;
    for (int k = 0; k < J.info.kvalid; ++k) mx = fmax(mx, fabs(img_value(J, k, n, tabs, L, nlat, nphi)));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    s_exp[n] = e;
    bscale[J.info.sc + n] = ldexp(1.0, e - (FIX_BITS - 32));
  }
  __syncthreads();
  unsigned char* base = img + J.info.off;
  constexpr long long LIM = 1ll << FIX_BITS;
  for (int t = threadIdx.x; t < kpad * npad; t += blockDim.x) {
    const int n = t % npad, k = t / npad;
    const double v = img_value(J, k, n, tabs, L, nlat, nphi);
    long long xi = __double2ll_rn(ldexp(v, FIX_BITS - s_exp[n]));  // |xi| < 2^38 by the exponent
    xi = xi < -LIM ? -LIM : (xi > LIM - 1 ? LIM - 1 : xi);
    const unsigned long long u = ((unsigned long long)(xi + 0x8080808080ll)) ^ 0x8080808080ull;
    const int ch = k / KC, kg = (k % KC) / 16, kb = k % 16;
    unsigned char* cbase = base + (size_t)ch * NDIG * 2 * npad * 16;
#pragma unroll
    for (int s = 0; s < NDIG; ++s)
      cbase[((size_t)(s * 2 + kg) * npad + n) * 16 + kb] = (unsigned char)(u >> (8 * (NDIG - 1 - s)));
  }
}

}  // namespace oz

// ------------------------------------------------------------------ host

namespace {
int round_up_oz(int x, int m) { return (x + m - 1) / m * m; }
}

struct OzPlan {
  oz::Args a;
  CUtensorMap tm[4];  // per stage: synthesis, inverse, forward, analysis
  int ntile_rows_nc, ntile_rows_col;
  int nsm = 148, tiles[4] = {0, 0, 0, 0};  // persistent grids: min(tiles, SMs) CTAs
  int ncw[4] = {8, 8, 8, 8};  // converter warps per stage (8 or 4; the autotuner's choice)
  DArr<double> S, Gs, rate, bscale;
  // -M dt factors of the inverse stage for the last two (dt, trapezoidal) keys
  DArr<double> nmdt[2];
  double nm_dt[2] = {0.0, 0.0};
  int nm_trap[2] = {-1, -1}, nm_next = 0;
  DArr<unsigned char> img;
  DArr<unsigned long long> gmax;  // gX, gS, gG, gA back to back
  size_t gmax_n = 0;
  DArr<oz::ImgInfo> info_synth, info_ana, info_inv, info_fwd;
};

static void oz_release(void* p) { delete static_cast<OzPlan*>(p); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    VG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
    if (!f || q != cudaDriverEntryPointSuccess) throw Error("vg_enable_visc3d: cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  return fn;
}

// a 4-D FP64 tensor map (dims innermost first, strides in bytes of dims 1-3)
// with a 4-D box, no swizzle, zeros outside the tensor
static void encode_map(CUtensorMap* tm, const double* base, const cuuint64_t dims[4], const cuuint64_t strides[3],
                       const cuuint32_t box[4]) {
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const CUresult r = tensor_map_encoder()(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims,
                                          strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error("vg_enable_visc3d: tensor map encoding failed");
}

void visc3d_oz_enable(vg_handle* h) {
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  const int L = G.lmax, nlat = G.nlat, nphi = G.nphi, half = nphi / 2;
  if (G.mmax != L) throw Error("vg_enable_visc3d: the exact tensor-core path needs mmax = lmax");
  if (L > oz::MAX_L) throw Error("vg_enable_visc3d: the exact tensor-core path supports lmax <= 511");
  const int nh = (nlat + 1) / 2;
  const int F = 3 * h->ne3d, NC = 2 * F, NCOL = 6 * F;
  auto* P = new OzPlan();
  h->tc_plan = P;
  h->tc_plan_release = oz_release;
  oz::Args& a = P->a;
  a.L = L;
  a.nlat = nlat;
  a.nh = nh;
  a.nphi = nphi;
  a.half = half;
  a.F = F;
  a.NC = NC;
  a.NCOL = NCOL;
  a.nk = h->nk;
  a.ne3d = h->ne3d;
  // the toroidal channels: two more gathered channels, the partner product
  // slots 6-11 of S, four more synthesis and analysis tile types
  const bool tor = h->tor_on;
  const int nch = tor ? 6 : 4;
  a.tor = tor ? 1 : 0;
  a.nslot = tor ? 12 : 6;
  a.ntype = tor ? 10 : 6;
  a.nq = tor ? 10 : 6;
  const int NSLOT = a.nslot;
  const int TN = oz::TN, KC = oz::KC;
  a.nts = (nh + TN - 1) / TN;
  const int kev = 2 * (L / 2), kod = 2 * ((L + 1) / 2);  // (m, re/im) counts: even m >= 2, odd m
  a.nti = std::max(1, (half - 1 + TN - 1) / TN);
  a.ntf = std::max(1, (std::max(kev, kod) + TN - 1) / TN);
  a.nta = ((L / 2 + 1) + TN - 1) / TN;
  std::vector<oz::ImgJob> jobs;
  long long off = 0;
  int sc = 0;
  auto add = [&](int kind, int table, int m, int par, int n0, int nvalid, int kvalid) {
    oz::ImgJob J;
    J.kind = kind;
    J.table = table;
    J.m = m;
    J.par = par;
    J.n0 = n0;
    J.info.nvalid = std::max(0, nvalid);
    J.info.kvalid = std::max(0, kvalid);
    J.info.sc = 0;
    if (J.info.nvalid == 0 || J.info.kvalid == 0) {
      J.info.kpad = 0;
      J.info.npad = 16;
      J.info.off = 0;
      return J;
    }
    J.info.npad = round_up_oz(J.info.nvalid, 16);  // M = 128 MMAs take N in steps of 16
    J.info.kpad = round_up_oz(J.info.kvalid, KC);
    J.info.off = off;
    J.info.sc = sc;
    sc += J.info.npad;
    off += (long long)oz::NDIG * J.info.kpad * J.info.npad;
    off = (off + 127) / 128 * 128;
    jobs.push_back(J);
    return J;
  };
  std::vector<oz::ImgInfo> isyn, iana, iinv(2 * a.nti), ifwd(2 * a.ntf);
  for (int m = 0; m <= L; ++m)
    for (int t = 0; t < 4; ++t)
      for (int par = 0; par < 2; ++par) {
        const int K = (L - m - par) >= 0 ? (L - m - par) / 2 + 1 : 0;  // l = m + par + 2 kk <= L
        for (int nt = 0; nt < a.nts; ++nt) isyn.push_back(add(0, t, m, par, nt * TN, std::min(TN, nh - nt * TN), K).info);
        for (int nt = 0; nt < a.nta; ++nt) iana.push_back(add(1, t, m, par, nt * TN, std::min(TN, K - nt * TN), nh).info);
      }
  for (int par = 0; par < 2; ++par) {
    const int K = par ? kod : kev;
    for (int nt = 0; nt < a.nti; ++nt) iinv[par * a.nti + nt] = add(2, 0, 0, par, nt * TN, std::min(TN, half - 1 - nt * TN), K).info;
    for (int nt = 0; nt < a.ntf; ++nt) ifwd[par * a.ntf + nt] = add(3, 0, 0, par, nt * TN, std::min(TN, K - nt * TN), half).info;
  }
  P->img.alloc((size_t)off);
  P->bscale.alloc((size_t)std::max(sc, 1));
  P->info_synth.upload(isyn, s);
  P->info_ana.upload(iana, s);
  P->info_inv.upload(iinv, s);
  P->info_fwd.upload(ifwd, s);
  {
    DArr<oz::ImgJob> d_jobs;
    d_jobs.upload(jobs, s);
    const double* tabs_h[8] = {G.d_plm.p, G.d_dplm.p, h->d_G6.p, h->d_H6.p,
                               h->d_wP.p, h->d_wD.p, h->d_wG.p, h->d_wH.p};
    DArr<const double*> d_tabs;
    d_tabs.alloc(8);
    VG_CUDA(cudaMemcpyAsync(d_tabs.p, tabs_h, sizeof(tabs_h), cudaMemcpyHostToDevice, s));
    oz::k_oz_images<<<(int)jobs.size(), 256, 0, s>>>(d_jobs.p, P->img.p, P->bscale.p, d_tabs.p, L, nlat, nphi);
    VG_CUDA(cudaGetLastError());
    VG_CUDA(cudaStreamSynchronize(s));
  }
  // rates transposed to [j][i][element] (FP64), from the (ne3d, nlat, nphi) copy
  {
    std::vector<double> r3((size_t)h->ne3d * nlat * nphi);
    VG_CUDA(cudaMemcpyAsync(r3.data(), h->d_MkPerDt3.p, r3.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    VG_CUDA(cudaStreamSynchronize(s));
    std::vector<double> rt(r3.size());
    for (int e = 0; e < h->ne3d; ++e)
      for (int j = 0; j < nlat; ++j)
        for (int i = 0; i < nphi; ++i) rt[((size_t)j * nphi + i) * h->ne3d + e] = r3[((size_t)e * nlat + j) * nphi + i];
    P->rate.upload(rt, s);
  }
  // FP64 work buffers: the gather writes X in lm order (an even number of
  // rows, the l = 0 row zero), the scatter reads dy; S has an even number of
  // order slabs (the inverse stage reads orders in pairs)
  const int nlm2 = (G.nlm + 1) / 2 * 2, M2 = (G.M + 1) / 2 * 2;
  h->d_X.alloc((size_t)nlm2 * nch * NC);
  h->d_dy.alloc((size_t)(h->nk + 1) * a.nq * NC);
  P->S.alloc((size_t)M2 * nlat * NSLOT * NC);  // zeroed: slots 6 and 9 (no toroidal partner) stay zero
  P->Gs.alloc((size_t)nlat * 2 * half * NCOL);
  // scale groups: gathered channels x columns, product slots x fields, the
  // inverse outputs (components x fields), analysis inputs x columns (8 with
  // the toroidal channels: plain rp and (m/sin) rt beside the six)
  P->gmax_n = (size_t)nch * NC + (size_t)NSLOT * F + 6 * F + (size_t)(tor ? 8 : 6) * NC;
  P->gmax.alloc(P->gmax_n);
  a.kbeg = h->d_kbeg.p;
  a.mbeg = G.d_mbeg.p;
  a.X = h->d_X.p;
  a.S = P->S.p;
  a.Gs = P->Gs.p;
  a.dy = h->d_dy.p;
  P->nmdt[0].alloc(P->rate.n);
  P->nmdt[1].alloc(P->rate.n);
  a.invsin = G.d_invsin.p;
  a.img = P->img.p;
  a.bscale = P->bscale.p;
  a.gX = P->gmax.p;
  a.gS = a.gX + (size_t)nch * NC;
  a.gG = a.gS + (size_t)NSLOT * F;
  a.gA = a.gG + 6 * F;
  a.status = h->d_maxbits.p + 2;
  P->ntile_rows_nc = (NC + oz::TM - 1) / oz::TM;
  P->ntile_rows_col = (NCOL + oz::TM - 1) / oz::TM;
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_SYNTH, 8>, oz::p::Ring<oz::ST_SYNTH>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_INV, 8>, oz::p::Ring<oz::ST_INV>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_FWD, 8>, oz::p::Ring<oz::ST_FWD>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_ANA, 8>, oz::p::Ring<oz::ST_ANA>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_SYNTH, 4>, oz::p::Ring<oz::ST_SYNTH>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_INV, 4>, oz::p::Ring<oz::ST_INV>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_FWD, 4>, oz::p::Ring<oz::ST_FWD>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_ANA, 4>, oz::p::Ring<oz::ST_ANA>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_SYNTH, 8, true>, oz::p::Ring<oz::ST_SYNTH>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_INV, 8, true>, oz::p::Ring<oz::ST_INV, true>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_FWD, 8, true>, oz::p::Ring<oz::ST_FWD>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_ANA, 8, true>, oz::p::Ring<oz::ST_ANA>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_SYNTH, 4, true>, oz::p::Ring<oz::ST_SYNTH>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_INV, 4, true>, oz::p::Ring<oz::ST_INV, true>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_FWD, 4, true>, oz::p::Ring<oz::ST_FWD>::SMEM);
  raise_smem_limit((const void*)oz::k_ozp_stage<oz::ST_ANA, 4, true>, oz::p::Ring<oz::ST_ANA>::SMEM);
  int dev = 0;
  VG_CUDA(cudaGetDevice(&dev));
  VG_CUDA(cudaDeviceGetAttribute(&P->nsm, cudaDevAttrMultiProcessorCount, dev));
  {  // the stages' tensor maps (boxes of one row tile by one K chunk, 32 KB)
    const cuuint64_t B = sizeof(double);
    const cuuint32_t TMr = oz::TM, KCc = oz::KC;
    // synthesis: X[lm][chan][n], lm = 2 q + par
    const cuuint64_t dx[4] = {(cuuint64_t)NC, (cuuint64_t)nch, 2, (cuuint64_t)nlm2 / 2};
    const cuuint64_t sx[3] = {NC * B, (cuuint64_t)nch * NC * B, 2 * (cuuint64_t)nch * NC * B};
    const cuuint32_t bx[4] = {TMr, 1, 1, KCc};
    encode_map(&P->tm[0], h->d_X.p, dx, sx, bx);
    // inverse: S[m][j][(p, f, ri)], m = 2 mq + mpar (with the toroidal channels the partner slots
    // follow at 6 F rows)
    const cuuint64_t di[4] = {(cuuint64_t)NSLOT * NC, (cuuint64_t)nlat, 2, (cuuint64_t)M2 / 2};
    const cuuint64_t si[3] = {(cuuint64_t)NSLOT * NC * B, (cuuint64_t)nlat * NSLOT * NC * B,
                              2 * (cuuint64_t)nlat * NSLOT * NC * B};
    const cuuint32_t bi[4] = {2 * TMr, 1, 1, KCc / 2};
    encode_map(&P->tm[1], P->S.p, di, si, bi);
    // forward: Gs[(j, sub)][i][row]
    const cuuint64_t dg[4] = {(cuuint64_t)NCOL, (cuuint64_t)half, 2 * (cuuint64_t)nlat, 1};
    const cuuint64_t sg[3] = {NCOL * B, (cuuint64_t)half * NCOL * B, 2 * (cuuint64_t)nlat * half * NCOL * B};
    const cuuint32_t bg[4] = {TMr, KCc, 1, 1};
    encode_map(&P->tm[2], P->Gs.p, dg, sg, bg);
    // analysis: S[m][j][p][n]
    const cuuint64_t da[4] = {(cuuint64_t)NC, (cuuint64_t)NSLOT, (cuuint64_t)nlat, (cuuint64_t)G.M};
    const cuuint64_t sa[3] = {NC * B, (cuuint64_t)NSLOT * NC * B, (cuuint64_t)nlat * NSLOT * NC * B};
    const cuuint32_t ba[4] = {TMr, 1, KCc, 1};
    encode_map(&P->tm[3], P->S.p, da, sa, ba);
  }
  P->tiles[0] = P->ntile_rows_nc * a.nts * G.M * a.ntype;
  P->tiles[1] = P->ntile_rows_col * a.nti * nlat;
  P->tiles[2] = P->ntile_rows_col * a.ntf * nlat;
  P->tiles[3] = P->ntile_rows_nc * a.nta * G.M * a.ntype;
  VG_CUDA(cudaStreamSynchronize(s));
}

// the scale-group maxima of the gather (channel x column), zeroed with the
// others before the gather of each advance
unsigned long long* visc3d_oz_gather_max(vg_handle* h) {
  OzPlan* P = static_cast<OzPlan*>(h->tc_plan);
  VG_CUDA(cudaMemsetAsync(P->gmax.p, 0, P->gmax_n * sizeof(unsigned long long), h->stream));
  return P->a.gX;
}

// The four exact tensor-core stages between the FP64 gather and the scatter.
// converter warps per exact stage (8 or 4 each; the rest of the 16 are epilogue warps)
void oz_set_ncw(vg_handle* h, const int ncw[4]) {
  OzPlan* P = static_cast<OzPlan*>(h->tc_plan);
  if (!P || h->p.visc3d_precision != VG_VISC3D_EXACT_TC) return;
  for (int i = 0; i < 4; ++i) {
    if (ncw[i] != 4 && ncw[i] != 8) throw Error("exact stages: converter warps must be 4 or 8");
    P->ncw[i] = ncw[i];
  }
}
bool oz_get_ncw(const vg_handle* h, int ncw[4]) {
  const OzPlan* P = static_cast<const OzPlan*>(h->tc_plan);
  if (!P || h->p.visc3d_precision != VG_VISC3D_EXACT_TC) return false;
  for (int i = 0; i < 4; ++i) ncw[i] = P->ncw[i];
  return true;
}

void visc3d_oz_run(vg_handle* h, double dt, bool trap) {
  OzPlan* P = static_cast<OzPlan*>(h->tc_plan);
  cudaStream_t s = h->stream;
  oz::Args a = P->a;
  {  // the sub-step's -M dt factors (recomputed when neither cached key matches)
    int slot = -1;
    for (int q = 0; q < 2; ++q)
      if (P->nm_trap[q] == (trap ? 1 : 0) && P->nm_dt[q] == dt) slot = q;
    if (slot < 0) {
      slot = P->nm_next;
      P->nm_next ^= 1;
      const size_t n = P->rate.n;
      oz::k_oz_rate_factors<<<(int)std::min<size_t>((n + 255) / 256, 4 * (size_t)P->nsm), 256, 0, s>>>(
          P->rate.p, P->nmdt[slot].p, n, dt, trap ? 1 : 0);
      ++h->n_launch;
      VG_CUDA(cudaGetLastError());
      P->nm_dt[slot] = dt;
      P->nm_trap[slot] = trap ? 1 : 0;
    }
    a.nmdt = P->nmdt[slot].p;
  }
  a.wait_ns = h->wait_ns;
  int stage = 0;
  auto launch = [&](auto kernel, int phase, const oz::ImgInfo* info, int tiles, size_t smem) {
    PhaseScope ps(h, phase);
    a.info = info;
    a.tmap = P->tm[stage++];
    kernel<<<std::max(1, std::min(tiles, P->nsm)), oz::p::NTHR, smem, s>>>(a);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  };
  using namespace oz;
  // every stage in its converter-warp split; the toroidal instantiations carry the partner slots
  auto stage_k = [&](auto k8, auto k4, int i, int phase, const ImgInfo* info, size_t smem) {
    if (P->ncw[i] == 4)
      launch(k4, phase, info, P->tiles[i], smem);
    else
      launch(k8, phase, info, P->tiles[i], smem);
  };
  if (a.tor) {
    stage_k(k_ozp_stage<ST_SYNTH, 8, true>, k_ozp_stage<ST_SYNTH, 4, true>, 0, VG_PH_V3_SYNTH, P->info_synth.p,
            p::Ring<ST_SYNTH>::SMEM);
    stage_k(k_ozp_stage<ST_INV, 8, true>, k_ozp_stage<ST_INV, 4, true>, 1, VG_PH_V3_LON_INV, P->info_inv.p,
            p::Ring<ST_INV, true>::SMEM);
    stage_k(k_ozp_stage<ST_FWD, 8, true>, k_ozp_stage<ST_FWD, 4, true>, 2, VG_PH_V3_LON_FWD, P->info_fwd.p,
            p::Ring<ST_FWD>::SMEM);
    stage_k(k_ozp_stage<ST_ANA, 8, true>, k_ozp_stage<ST_ANA, 4, true>, 3, VG_PH_V3_ANALYSIS, P->info_ana.p,
            p::Ring<ST_ANA>::SMEM);
  } else {
    stage_k(k_ozp_stage<ST_SYNTH, 8>, k_ozp_stage<ST_SYNTH, 4>, 0, VG_PH_V3_SYNTH, P->info_synth.p,
            p::Ring<ST_SYNTH>::SMEM);
    stage_k(k_ozp_stage<ST_INV, 8>, k_ozp_stage<ST_INV, 4>, 1, VG_PH_V3_LON_INV, P->info_inv.p, p::Ring<ST_INV>::SMEM);
    stage_k(k_ozp_stage<ST_FWD, 8>, k_ozp_stage<ST_FWD, 4>, 2, VG_PH_V3_LON_FWD, P->info_fwd.p, p::Ring<ST_FWD>::SMEM);
    stage_k(k_ozp_stage<ST_ANA, 8>, k_ozp_stage<ST_ANA, 4>, 3, VG_PH_V3_ANALYSIS, P->info_ana.p,
            p::Ring<ST_ANA>::SMEM);
  }
}

}  // namespace vg
