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
//   every FP64 operand value x of a scale group g is written as a 40-bit
//   fixed-point integer xi = rint(x 2^(39 - E_g)), |x| < 2^E_g, and xi as five
//   signed 8-bit digits, xi = sum_s d_s 256^(4 - s). A product of two such
//   values is sum_{s,t} d_s g_t 256^(8 - s - t); the digit pairs of one level
//   s + t = lambda share a weight, so each level is one int32 accumulator in
//   tensor memory, summed exactly over K. Levels 0..4 are kept (15 digit-pair
//   MMAs per K step); the dropped levels weigh < 2^-37 of |x|max |y|max per
//   term. The epilogue combines the five levels in FP64 and applies the
//   row and column scales.
//
// So the products carry ~38 significant bits relative to their operand
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
// Kernel shape: one CTA per SM (tensor memory: 5 levels x 2 sub-GEMMs x 48
// columns), 16 loader warps that fetch A in FP64 one chunk ahead, slice it into
// the five digit planes in shared memory (canonical K-major no-swizzle layout)
// and later run the epilogue, and one MMA warp whose lane 0 issues the
// tcgen05.mma and commits each stage to its mbarrier. Handoff waits between
// loaders and the MMA warp are bounded by the handle's wait limit; waits for the
// hardware's own copies and MMAs by a fixed 2 s; a wait that runs out raises a
// status bit instead of hanging.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "vg_device.cuh"
#include "vg_internal.cuh"
#include "vg_tcgen05.cuh"

namespace vg {
namespace oz {

using namespace vg::ptx;

constexpr int TM = 128;        // tile rows (MMA M)
constexpr int TN = 48;         // max columns of one sub-GEMM (MMA N)
constexpr int KC = 32;         // K per pipeline chunk = one i8 k-step
constexpr int NSTAGE = 4;      // shared-memory ring depth
constexpr int NLEV = 5;        // digit levels kept (15 digit-pair products)
constexpr int NDIG = 5;        // 8-bit digits per operand value
constexpr int NLOAD = 512;     // loader / epilogue threads
constexpr int MMA_WARP = NLOAD / 32;
constexpr int NTHR_ALL = NLOAD + 32;
static_assert(TM * KC / NLOAD == 8, "a loader thread slices eight K of one row per chunk");
constexpr int A_PLANE = TM * KC;              // bytes of one digit plane of the A chunk
constexpr int A_BYTES = NDIG * A_PLANE;
constexpr int B_BYTES_MAX = NDIG * TN * KC;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES_MAX;
constexpr int TMEM_COLS = 512;                // 2 * NLEV * TN = 480 used
constexpr int MAX_L = 511;
constexpr int FIX_BITS = 39;                  // |xi| < 2^39: five signed 8-bit digits
constexpr unsigned long long HW_WAIT_NS = 2000000000ull;  // bound on waits for copies and MMAs
constexpr size_t SMEM_BYTES = 1024 + (size_t)NSTAGE * STAGE_BYTES + 256 + 2 * 4 * TM * 8 + (MAX_L + 1) * 4;
static_assert(SMEM_BYTES > 114 * 1024, "one CTA per SM: the tensor-memory plan takes 480 of its 512 columns");
static_assert(STAGE_BYTES % 128 == 0, "stage buffers stay 128-byte aligned");

enum { ST_SYNTH = 0, ST_INV = 1, ST_FWD = 2, ST_ANA = 3 };

// digit image of one (batch key, sub-GEMM, N tile) of a constant B operand
struct ImgInfo {
  long long off;  // byte offset of chunk 0: chunks of NDIG x 2 x npad x 16 bytes follow
  int kpad, npad, nvalid, kvalid;
  int sc;         // first of the image's npad column factors 2^(E_col - 7)
};

struct Args {
  int L, nlat, nh, nphi, half, F, NC, NCOL, nk, ne3d;
  int nts, nti, ntf, nta;
  const int* kbeg;
  const double* X;     // [(nk + 1)][4][NC]      gathered memory + 2 mu strain
  double* S;           // [M][nlat][6][NC]       synthesis products, later the analysis inputs
  double* Gs;          // [nlat][2][half][NCOL]  even / odd longitude combinations of -M dt g
  double* dy;          // [(nk + 1)][6][NC]      analysis outputs
  const double* rate;  // [nlat][nphi][ne3d]     mu / eta_eff
  double dt;
  int trap;
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

// 32 lanes x 8 consecutive 32-bit columns (no wait: the caller waits once)
__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, int* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
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

// five 8-bit digit planes of eight values (K consecutive) of one row:
// xi = rint(v * rs) in [-2^39, 2^39), u = xi + sum_k 128 * 256^k in [0, 2^40),
// digit k = byte k of u minus 128 = byte k of (u ^ 0x8080808080) as int8.
// pl[s] holds digit s (most significant first) of the eight values.
__device__ __forceinline__ void to_digits8(const double* v, double rs, uint2* pl) {
  constexpr long long LIM = 1ll << FIX_BITS;
  uint32_t lo[8], hi[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    long long xi = __double2ll_rn(v[q] * rs);
    xi = xi < -LIM ? -LIM : (xi > LIM - 1 ? LIM - 1 : xi);
    const unsigned long long u = ((unsigned long long)(xi + 0x8080808080ll)) ^ 0x8080808080ull;
    lo[q] = (uint32_t)u;
    hi[q] = (uint32_t)(u >> 32);
  }
  auto gather4 = [](uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t b) {
    const uint32_t sel = b | ((b + 4) << 4);
    const uint32_t t01 = __byte_perm(w0, w1, sel), t23 = __byte_perm(w2, w3, sel);
    return __byte_perm(t01, t23, 0x5410);
  };
  pl[0] = make_uint2(gather4(hi[0], hi[1], hi[2], hi[3], 0), gather4(hi[4], hi[5], hi[6], hi[7], 0));
#pragma unroll
  for (int s = 1; s < NDIG; ++s) {
    const uint32_t b = (uint32_t)(4 - s);
    pl[s] = make_uint2(gather4(lo[0], lo[1], lo[2], lo[3], b), gather4(lo[4], lo[5], lo[6], lo[7], b));
  }
}

// five int32 levels (weights 256^-lambda) -> FP64, before the row and column scales
__device__ __forceinline__ double combine_levels(const int* a0, const int* a1, const int* a2, const int* a3,
                                                 const int* a4, int i) {
  constexpr double W = 0.00390625;  // 2^-8
  double v = (double)a4[i];
  v = fma(v, W, (double)a3[i]);
  v = fma(v, W, (double)a2[i]);
  v = fma(v, W, (double)a1[i]);
  return fma(v, W, (double)a0[i]);
}

__device__ __forceinline__ int slot_row(const int* kbeg, int l, int m, int nk) {
  return l >= 1 ? __ldg(&kbeg[l]) + m : nk;
}

// table sign under theta -> pi - theta (times (-1)^(l+m)): P, G even; dP, H odd
__device__ __forceinline__ double table_sigma(int p) { return (p == 1 || p == 5) ? -1.0 : 1.0; }
__device__ __forceinline__ int table_of(int p) {
  const int t[6] = {0, 1, 0, 0, 2, 3};
  return t[p];
}
__device__ __forceinline__ int chan_of(int p) { return (p == 0) ? 0 : (p <= 2 ? 1 : (p == 3 ? 2 : 3)); }

struct Cta {
  int rows, row0, batch_m, p, j, nt;
  ImgInfo sub[2];
};

template <int STAGE>
__device__ __forceinline__ Cta cta_info(const Args& A) {
  Cta c;
  c.nt = blockIdx.y;
  c.row0 = blockIdx.x * TM;
  if (STAGE == ST_SYNTH || STAGE == ST_ANA) {
    c.batch_m = blockIdx.z / 6;
    c.p = blockIdx.z % 6;
    c.j = 0;
    c.rows = min(TM, A.NC - c.row0);
    const int nt_count = STAGE == ST_SYNTH ? A.nts : A.nta;
    const int base = ((c.batch_m * 4 + table_of(c.p)) * 2) * nt_count;
    c.sub[0] = A.info[base + c.nt];
    c.sub[1] = A.info[base + nt_count + c.nt];
  } else {
    c.batch_m = 0;
    c.p = 0;
    c.j = blockIdx.z;
    c.rows = min(TM, A.NCOL - c.row0);
    const int nt_count = STAGE == ST_INV ? A.nti : A.ntf;
    c.sub[0] = A.info[c.nt];
    c.sub[1] = A.info[nt_count + c.nt];
  }
  return c;
}

// Loader context of one thread: its tile row, that row's base address and
// fixed-point scale.
struct RowCtx {
  bool live;
  const double* base;
  int p;
  double is_j;  // 1 / sin(theta_j) for the inverse stage's p = 2 rows
  double rs;    // 2^(39 - E): value -> 40-bit fixed point
  int e;        // the row group's exponent E (the analysis rows: E + 1, the E / O bound)
};

template <int STAGE>
__device__ __forceinline__ RowCtx row_ctx(const Args& A, const Cta& c, int r) {
  RowCtx rc;
  const int row = c.row0 + r;
  rc.live = r < c.rows;
  rc.p = 0;
  rc.is_j = 0.0;
  rc.e = 0;
  rc.base = nullptr;
  if (rc.live) {
    if (STAGE == ST_SYNTH) {
      const int chan = chan_of(c.p);
      rc.base = A.X + (size_t)chan * A.NC + row;  // + slot * 4 NC
      rc.e = group_exp(A.gX[chan * A.NC + row]);
    } else if (STAGE == ST_INV) {
      rc.p = row / A.F;
      const int f = row % A.F;
      rc.base = A.S + ((size_t)c.j * 6 + rc.p) * A.NC + 2 * f;  // + m nlat 6 NC
      rc.is_j = A.invsin[c.j];
      rc.e = group_exp(A.gS[rc.p * A.F + f]);
    } else if (STAGE == ST_FWD) {
      rc.base = A.Gs + (size_t)c.j * 2 * A.half * A.NCOL + row;  // + (sub half + i) NCOL
      rc.e = group_exp(A.gG[row]);                                 // rows (p, f) = p F + f
    } else {
      rc.base = A.S + (size_t)c.batch_m * A.nlat * 6 * A.NC + (size_t)c.p * A.NC + row;  // + j 6 NC
      rc.e = group_exp(A.gA[c.p * A.NC + row]) + 1;  // |R_j +- R_mirror| <= 2 max
    }
  }
  rc.rs = pow2(FIX_BITS - rc.e);
  return rc;
}

// raw values of one thread's eight K of a chunk (the analysis also holds the
// mirrored latitude's eight values)
template <int N>
struct OctT {
  double v[N];
};
template <int STAGE>
using Oct = OctT<STAGE == ST_ANA ? 16 : 8>;

// Issue the global loads of eight consecutive K (zeros outside the valid range).
template <int STAGE>
__device__ __forceinline__ void fetch(const Args& A, const Cta& c, const RowCtx& rc, const int* slot_sm, int sub,
                                      int k0, Oct<STAGE>& Q) {
  constexpr int NV = STAGE == ST_ANA ? 16 : 8;
#pragma unroll
  for (int i = 0; i < NV; ++i) Q.v[i] = 0.0;
  if (!rc.live) return;
  if (STAGE == ST_SYNTH) {
    // X[slot(l, m)][chan_p][n], l = m + par + 2 kk
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int dl = sub + 2 * (k0 + q);
      if (c.batch_m + dl <= A.L) Q.v[q] = rc.base[(size_t)slot_sm[dl] * 4 * A.NC];
    }
  } else if (STAGE == ST_INV) {
    // (m, re), (m, im) for m = (sub ? 1 : 2) + 2 (k / 2)
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int m = (sub ? 1 : 2) + 2 * ((k0 >> 1) + h);
      if (m <= A.L) {
        const double2 z = *reinterpret_cast<const double2*>(rc.base + (size_t)m * A.nlat * 6 * A.NC);
        Q.v[2 * h] = z.x;
        Q.v[2 * h + 1] = z.y;
      }
    }
  } else if (STAGE == ST_FWD) {
    // s_i (sub 0) or d_i (sub 1), i = k
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int i = k0 + q;
      if (i < A.half) Q.v[q] = rc.base[((size_t)sub * A.half + i) * A.NCOL];
    }
  } else {
    // analysis: R_j and R_mirror over the northern rows j = k
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int j = k0 + q, jm = A.nlat - 1 - j;
      if (j < A.nh) {
        Q.v[q] = rc.base[(size_t)j * 6 * A.NC];
        if (jm != j) Q.v[8 + q] = rc.base[(size_t)jm * 6 * A.NC];
      }
    }
  }
}

// The eight A values of a fetched Oct (in place in Q.v[0..7]). `sum`
// accumulates the CUDA-core side terms (inverse: column i = 0, sum_m 2 Re z_m;
// forward: order 0, sum_i s_i).
template <int STAGE>
__device__ __forceinline__ void finish(const Cta& c, const RowCtx& rc, int sub, int k0, Oct<STAGE>& Q,
                                       double& sum) {
  if (STAGE == ST_INV) {
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      double re = Q.v[2 * h], im = Q.v[2 * h + 1];
      if (rc.p == 2) {  // i (m / sin theta) z
        const int m = (sub ? 1 : 2) + 2 * ((k0 >> 1) + h);
        const double a = (double)m * rc.is_j;
        const double t = re;
        re = -a * im;
        im = a * t;
      } else if (rc.p == 5) {  // i z
        const double t = re;
        re = -im;
        im = t;
      }
      Q.v[2 * h] = re;
      Q.v[2 * h + 1] = im;
      sum += 2.0 * re;
    }
  } else if (STAGE == ST_FWD) {
    if (sub == 0)
#pragma unroll
      for (int q = 0; q < 8; ++q) sum += Q.v[q];
  } else if (STAGE == ST_ANA) {  // E: R_j + sigma R_mirror; O: R_j - sigma R_mirror
    const double sg = table_sigma(c.p) * (sub ? -1.0 : 1.0);
#pragma unroll
    for (int q = 0; q < 8; ++q) Q.v[q] = Q.v[q] + sg * Q.v[8 + q];
  }
}

// ------------------------------------------------------------------ kernel

template <int STAGE>
__global__ void __launch_bounds__(NTHR_ALL, 1) k_oz_stage(Args A) {
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  unsigned char* stage_base = sm;
  uint64_t* bars = (uint64_t*)(sm + (size_t)NSTAGE * STAGE_BYTES);  // NSTAGE + 1: MMA done per stage, drain
  uint64_t* bfull = bars + NSTAGE + 1;                               // NSTAGE: B bulk copy landed
  uint64_t* afull = bfull + NSTAGE;                                  // NSTAGE: A stored by all loaders
  uint32_t* tslot = (uint32_t*)(afull + NSTAGE);
  volatile int* abort_flag = (volatile int*)(tslot + 1);
  double* rsum = (double*)(sm + (size_t)NSTAGE * STAGE_BYTES + 256);  // [2 subs][4 quarters][TM]
  int* slot_sm = (int*)(rsum + 2 * 4 * TM);                          // synthesis: slot(m + dl, m)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const Cta c = cta_info<STAGE>(A);
  if (c.rows <= 0) return;

  if (tid == 0) {
    for (int i = 0; i <= NSTAGE; ++i) mbar_init(&bars[i], 1);
    for (int i = 0; i < NSTAGE; ++i) mbar_init(&bfull[i], 1);
    for (int i = 0; i < NSTAGE; ++i) mbar_init(&afull[i], NLOAD);
    fence_mbar_init();
    *abort_flag = 0;
  }
  if (warp == 0) tmem_alloc(tslot, TMEM_COLS);
  for (int i = tid; i < 2 * 4 * TM; i += NTHR_ALL) rsum[i] = 0.0;
  if (STAGE == ST_SYNTH)
    for (int dl = tid; dl <= A.L - c.batch_m; dl += NTHR_ALL)
      slot_sm[dl] = slot_row(A.kbeg, c.batch_m + dl, c.batch_m, A.nk);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  const int nch0 = c.sub[0].kpad / KC, nch1 = c.sub[1].kpad / KC, nch = nch0 + nch1;
  // loader mapping: row lr = tid % TM, K quarter lq = tid / TM (eight K of the chunk)
  const int lr = tid % TM, lq = tid / TM;
  RowCtx rc;
  if (tid < NLOAD) rc = row_ctx<STAGE>(A, c, lr);
  double sum0 = 0.0, sum1 = 0.0;  // loader side sums of the two sub-GEMMs
  int b_issued = 0;               // B copies issued (loader thread 0 issues them)
  auto copy_b = [&](int b, const ImgInfo& I, int kc) {
    if (tid == 0) {
      unsigned char* dst = stage_base + (size_t)b * STAGE_BYTES + A_BYTES;
      const uint32_t bytes = (uint32_t)(NDIG * 2 * I.npad * 16);
      const unsigned char* src = A.img + I.off + (size_t)kc * bytes;
      mbar_expect_tx(&bfull[b], bytes);
      bulk_g2s(dst, src, bytes, &bfull[b]);
    }
    ++b_issued;
  };
  auto fetch_chunk = [&](int ch, Oct<STAGE>& Q) {
    const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
    fetch<STAGE>(A, c, rc, slot_sm, sub, kc * KC + 8 * lq, Q);
  };
  __shared__ int s_b_issued, s_mma_issued;
  if (warp == MMA_WARP) {
    // ---- MMA issuer: chunk ch once its A (all loaders) and B (bulk copy) landed
    if (lane == 0) {
      int b_done = 0, issued = 0;
      for (int ch = 0; ch < nch; ++ch) {
        const int buf = ch % NSTAGE;
        const uint32_t ph = (uint32_t)((ch / NSTAGE) & 1);
        if (!mbar_wait_or_abort_ns(&afull[buf], ph, abort_flag, A.wait_ns)) {
          *abort_flag = 1;
          atomicOr(A.status, 1ull << (28 + STAGE));
          break;
        }
        if (!mbar_wait_ns(&bfull[buf], ph, HW_WAIT_NS)) {
          *abort_flag = 1;
          atomicOr(A.status, 1ull << (20 + STAGE));
          break;
        }
        ++b_done;
        tc_fence_after();
        const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
        const ImgInfo& I = c.sub[sub];
        const unsigned char* Ab = stage_base + (size_t)buf * STAGE_BYTES;
        const unsigned char* Bb = Ab + A_BYTES;
        const uint32_t idesc = idesc_i8(TM, I.npad);
#pragma unroll
        for (int s = 0; s < NDIG; ++s) {
          const uint64_t da = sdesc(saddr(Ab + s * A_PLANE), TM * 16, 128);
#pragma unroll
          for (int t = 0; t < NLEV - s; ++t) {
            const uint64_t db = sdesc(saddr(Bb + t * 2 * I.npad * 16), I.npad * 16, 128);
            const uint32_t d = tmem + (uint32_t)(((s + t) * 2 + sub) * TN);
            mma_i8(d, da, db, idesc, (kc > 0 || s > 0) ? 1u : 0u);
          }
        }
        mma_commit(&bars[buf]);
        ++issued;
      }
      if (issued > 0) mma_commit(&bars[NSTAGE]);  // drain: tracks every MMA this thread issued
      s_b_issued = b_done;
      s_mma_issued = issued;
    }
    __syncwarp();
  } else {
    // ---- loaders: A of chunk ch into stage buffer ch % NSTAGE, B bulk copies one chunk ahead
    Oct<STAGE> cur, nxt;
    if (nch > 0) {
      copy_b(0, c.sub[0].kpad > 0 ? c.sub[0] : c.sub[1], 0);
      fetch_chunk(0, cur);
    }
    for (int ch = 0; ch < nch; ++ch) {
      const int buf = ch % NSTAGE;
      const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
      const bool more = ch + 1 < nch;
      if (more) {
        // stage buffer of chunk ch + 1 was last read by the MMAs of chunk ch + 1 - NSTAGE
        const int nb = (ch + 1) % NSTAGE;
        if (ch + 1 >= NSTAGE &&
            !mbar_wait_or_abort_ns(&bars[nb], (uint32_t)(((ch + 1) / NSTAGE - 1) & 1), abort_flag, A.wait_ns)) {
          *abort_flag = 1;
          atomicOr(A.status, 1ull << (24 + STAGE));
        }
        if (*abort_flag) break;
        const int sub1 = (ch + 1) < nch0 ? 0 : 1, kc1 = sub1 ? ch + 1 - nch0 : ch + 1;
        copy_b(nb, c.sub[sub1], kc1);
        fetch_chunk(ch + 1, nxt);
      }
      // A of chunk ch: finish, slice into digits, store
      double part = 0.0;
      finish<STAGE>(c, rc, sub, kc * KC + 8 * lq, cur, part);
      if (sub)
        sum1 += part;
      else
        sum0 += part;
      uint2 pl[NDIG];
      to_digits8(cur.v, rc.rs, pl);
      unsigned char* Ab = stage_base + (size_t)buf * STAGE_BYTES;
      // digit plane s, K group lq / 2 (16 K), row lr, bytes 8 (lq & 1) .. + 7
      const size_t at = ((size_t)(lq >> 1) * TM + lr) * 16 + 8 * (lq & 1);
#pragma unroll
      for (int s = 0; s < NDIG; ++s) *reinterpret_cast<uint2*>(Ab + s * A_PLANE + at) = pl[s];
      fence_async_smem();  // this thread's A stores, visible to the tensor cores
      mbar_arrive(&afull[buf]);
      if (more) cur = nxt;
    }
  }
  __syncthreads();
  // B copies still in flight after an abort: wait for them before the stage
  // ring is reused or the CTA exits
  if (tid == 0)
    for (int q = s_b_issued; q < b_issued; ++q)
      if (!mbar_wait_ns(&bfull[q % NSTAGE], (uint32_t)((q / NSTAGE) & 1), HW_WAIT_NS))
        atomicOr(A.status, 1ull << (20 + STAGE));
  // drain: the issuer's last commit completes once every MMA has
  bool ok = (*abort_flag == 0);
  if (s_mma_issued > 0 && !mbar_wait_ns(&bars[NSTAGE], 0, HW_WAIT_NS)) {
    ok = false;
    atomicOr(A.status, 1ull << (16 + STAGE));
  }
  if (tid < NLOAD) {
    rsum[(0 * 4 + lq) * TM + lr] = sum0;
    rsum[(1 * 4 + lq) * TM + lr] = sum1;
  }
  ok = __syncthreads_and(ok) != 0;
  tc_fence_after();

  if (ok && tid < NLOAD) {
    const int quad = warp & 3, cq = warp >> 2;  // lane quarter, column-block group (4 per quarter)
    const int r = quad * 32 + lane;
    const int row = c.row0 + r;
    const bool live = r < c.rows;
    const uint32_t tbase = tmem + ((uint32_t)(quad * 32) << 16);
    const bool has[2] = {nch0 > 0, nch1 > 0};
    const int npad_max = max(has[0] ? c.sub[0].npad : 0, has[1] ? c.sub[1].npad : 0);
    // the row's group exponent, as the loaders of this row used it
    const RowCtx rrc = row_ctx<STAGE>(A, c, r);
    const double rf = pow2(rrc.e - 7);
    // one sub-GEMM's eight columns cb .. cb + 7, combined and scaled (zero past its N)
    auto load_block = [&](int sub, int cb, double* out) {
      if (!has[sub] || cb >= c.sub[sub].npad) {
#pragma unroll
        for (int i = 0; i < 8; ++i) out[i] = 0.0;
        return;
      }
      int a[NLEV][8];
#pragma unroll
      for (int lv = 0; lv < NLEV; ++lv) tmem_ld8_nowait(tbase + (uint32_t)((lv * 2 + sub) * TN + cb), a[lv]);
      tmem_wait_ld();
      const double* cs = A.bscale + c.sub[sub].sc + cb;
#pragma unroll
      for (int i = 0; i < 8; ++i) out[i] = combine_levels(a[0], a[1], a[2], a[3], a[4], i) * rf * __ldg(&cs[i]);
    };
    if (STAGE == ST_SYNTH) {
      const int m = c.batch_m, p = c.p;
      const double sg = table_sigma(p);
      double gmax = 0.0;
      for (int cb = cq * 8; cb < npad_max; cb += 32) {
        double e[8], o[8];
        load_block(0, cb, e);
        load_block(1, cb, o);
        if (!live) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int j = c.nt * TN + cb + i;
          if (j >= A.nh) break;
          const int jm = A.nlat - 1 - j;
          const double vn = e[i] + o[i];
          A.S[(((size_t)m * A.nlat + j) * 6 + p) * A.NC + row] = vn;
          // the inverse stage reads p = 2 as (m / sin theta) S
          const double fj = (p == 2) ? (double)m * A.invsin[j] : 1.0;
          gmax = fmax(gmax, fabs(vn) * fj);
          if (jm != j) {
            const double vs = sg * (e[i] - o[i]);
            A.S[(((size_t)m * A.nlat + jm) * 6 + p) * A.NC + row] = vs;
            const double fm = (p == 2) ? (double)m * A.invsin[jm] : 1.0;
            gmax = fmax(gmax, fabs(vs) * fm);
          }
        }
      }
      if (live) atomic_max_bits(&A.gS[p * A.F + row / 2], gmax);
    } else if (STAGE == ST_INV) {
      const int p = row / A.F, f = row % A.F, e3 = f / 3;
      double c0 = 0.0;  // m = 0 term (weight 1), the real part of z_0
      if (live && p != 2) {
        const double2 z = *reinterpret_cast<const double2*>(A.S + (((size_t)0 * A.nlat + c.j) * 6 + p) * A.NC + 2 * f);
        c0 = (p == 5) ? -z.y : z.x;
      }
      // the latitude's rates mu / eta (nphi x ne3d doubles), staged once in the
      // stage ring (free after the main loop: every MMA has completed)
      const double* rate_g = A.rate + (size_t)c.j * A.nphi * A.ne3d;
      const double* rate_j = rate_g + e3;
      const bool staged = (size_t)A.nphi * A.ne3d * 8 <= (size_t)NSTAGE * STAGE_BYTES;
      if (staged) {
        double* rate_s = reinterpret_cast<double*>(stage_base);
        for (int t = tid; t < A.nphi * A.ne3d; t += NLOAD) rate_s[t] = __ldg(&rate_g[t]);
        asm volatile("bar.sync 1, %0;" ::"n"(NLOAD));  // the loader / epilogue warps only
        rate_j = rate_s + e3;
      }
      double* gs = A.Gs + (size_t)c.j * 2 * A.half * A.NCOL + row;
      double* gd = gs + (size_t)A.half * A.NCOL;
      double gmax = 0.0;
      auto emit = [&](int i, double ev, double od) {
        double m1 = rate_j[(size_t)i * A.ne3d] * A.dt, m2 = rate_j[(size_t)(i + A.half) * A.ne3d] * A.dt;
        if (A.trap) {
          m1 = m1 / (1.0 + 0.5 * m1);
          m2 = m2 / (1.0 + 0.5 * m2);
        }
        const double g1 = -m1 * (ev + od), g2 = -m2 * (ev - od);
        const double sv = g1 + g2, dv = g1 - g2;
        gs[(size_t)i * A.NCOL] = sv;
        gd[(size_t)i * A.NCOL] = dv;
        gmax = fmax(gmax, fmax(fabs(sv), fabs(dv)));
      };
      if (live && c.nt == 0 && cq == 0) {
        double sev = 0.0, sod = 0.0;
        for (int q = 0; q < 4; ++q) {
          sev += rsum[(0 * 4 + q) * TM + r];
          sod += rsum[(1 * 4 + q) * TM + r];
        }
        emit(0, c0 + sev, sod);
      }
      for (int cb = cq * 8; cb < npad_max; cb += 32) {
        double e[8], o[8];
        load_block(0, cb, e);
        load_block(1, cb, o);
        if (!live) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int ii = 1 + c.nt * TN + cb + i;
          if (ii >= A.half) break;
          emit(ii, e[i] + c0, o[i]);
        }
      }
      if (live) atomic_max_bits(&A.gG[row], gmax);
    } else if (STAGE == ST_FWD) {
      const int p = row / A.F, f = row % A.F;
      const double isj = A.invsin[c.j];
      const double beta_c = (p == 3 || p == 4) ? 2.0 : (p == 5 ? 4.0 : 1.0);
      auto out = [&](int m) -> double2* {
        return reinterpret_cast<double2*>(A.S + (((size_t)m * A.nlat + c.j) * 6 + p) * A.NC + 2 * f);
      };
      double gre = 0.0, gim = 0.0;
      if (live && c.nt == 0 && cq == 0) {
        // m = 0: F_0 = (2 pi / nphi) sum_i s_i, real
        double s0 = 0.0;
        for (int q = 0; q < 4; ++q) s0 += rsum[(0 * 4 + q) * TM + r];
        const double v = (p == 2) ? 0.0 : beta_c * s0 * (2.0 * PI / (double)A.nphi);
        *out(0) = make_double2(v, 0.0);
        gre = fabs(v);
      }
      for (int sub = 0; sub < 2; ++sub) {
        if (!has[sub]) continue;
        const int npad = c.sub[sub].npad, nval = c.sub[sub].nvalid;
        for (int cb = cq * 8; cb < npad; cb += 32) {
          double v[8];
          load_block(sub, cb, v);
          if (!live) continue;
#pragma unroll
          for (int i = 0; i < 8; i += 2) {
            const int kk = c.nt * TN + cb + i;  // (m, re) column; (m, im) follows
            if (kk >= c.nt * TN + nval) break;
            const int m = (sub ? 1 : 2) + 2 * (kk >> 1);
            const double beta = (p == 2) ? (double)m * isj : beta_c;
            const double re = beta * v[i], im = beta * v[i + 1];
            *out(m) = make_double2(re, im);
            gre = fmax(gre, fabs(re));
            gim = fmax(gim, fabs(im));
          }
        }
      }
      if (live) {
        atomic_max_bits(&A.gA[p * A.NC + 2 * f], gre);
        atomic_max_bits(&A.gA[p * A.NC + 2 * f + 1], gim);
      }
    } else {
      const int m = c.batch_m, p = c.p;
      for (int sub = 0; sub < 2; ++sub) {
        if (!has[sub]) continue;
        const int npad = c.sub[sub].npad;
        for (int cb = cq * 8; cb < npad; cb += 32) {
          double v[8];
          load_block(sub, cb, v);
          if (!live) continue;
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int kk = c.nt * TN + cb + i;
            const int l = m + sub + 2 * kk;
            if (l > A.L) break;
            A.dy[((size_t)slot_row(A.kbeg, l, m, A.nk) * 6 + p) * A.NC + row] = v[i];
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TMEM_COLS);
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
// column factors 2^(E - 7) the epilogue applies.
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
    bscale[J.info.sc + n] = ldexp(1.0, e - 7);
  }
  __syncthreads();
  unsigned char* base = img + J.info.off;
  constexpr long long LIM = 1ll << FIX_BITS;
  for (int t = threadIdx.x; t < kpad * npad; t += blockDim.x) {
    const int n = t % npad, k = t / npad;
    const double v = img_value(J, k, n, tabs, L, nlat, nphi);
    long long xi = __double2ll_rn(ldexp(v, FIX_BITS - s_exp[n]));
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
  int ntile_rows_nc, ntile_rows_col;
  DArr<double> S, Gs, rate, bscale;
  DArr<unsigned char> img;
  DArr<unsigned long long> gmax;  // gX, gS, gG, gA back to back
  size_t gmax_n = 0;
  DArr<oz::ImgInfo> info_synth, info_ana, info_inv, info_fwd;
};

static void oz_release(void* p) { delete static_cast<OzPlan*>(p); }

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
  // FP64 work buffers: the gather writes the FP64 path's X, the scatter reads dy
  h->d_X.alloc((size_t)(h->nk + 1) * 4 * NC);
  h->d_dy.alloc((size_t)(h->nk + 1) * 6 * NC);
  P->S.alloc((size_t)G.M * nlat * 6 * NC);
  P->Gs.alloc((size_t)nlat * 2 * half * NCOL);
  P->gmax_n = (size_t)4 * NC + 6 * F + 6 * F + 6 * NC;
  P->gmax.alloc(P->gmax_n);
  a.kbeg = h->d_kbeg.p;
  a.X = h->d_X.p;
  a.S = P->S.p;
  a.Gs = P->Gs.p;
  a.dy = h->d_dy.p;
  a.rate = P->rate.p;
  a.invsin = G.d_invsin.p;
  a.img = P->img.p;
  a.bscale = P->bscale.p;
  a.gX = P->gmax.p;
  a.gS = a.gX + 4 * NC;
  a.gG = a.gS + 6 * F;
  a.gA = a.gG + 6 * F;
  a.status = h->d_maxbits.p + 2;
  P->ntile_rows_nc = (NC + oz::TM - 1) / oz::TM;
  P->ntile_rows_col = (NCOL + oz::TM - 1) / oz::TM;
  raise_smem_limit((const void*)oz::k_oz_stage<oz::ST_SYNTH>, oz::SMEM_BYTES);
  raise_smem_limit((const void*)oz::k_oz_stage<oz::ST_INV>, oz::SMEM_BYTES);
  raise_smem_limit((const void*)oz::k_oz_stage<oz::ST_FWD>, oz::SMEM_BYTES);
  raise_smem_limit((const void*)oz::k_oz_stage<oz::ST_ANA>, oz::SMEM_BYTES);
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
void visc3d_oz_run(vg_handle* h, double dt, bool trap) {
  OzPlan* P = static_cast<OzPlan*>(h->tc_plan);
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  oz::Args a = P->a;
  a.dt = dt;
  a.trap = trap ? 1 : 0;
  a.wait_ns = h->wait_ns;
  auto launch = [&](auto kernel, int phase, const oz::ImgInfo* info, dim3 grid) {
    PhaseScope ps(h, phase);
    a.info = info;
    kernel<<<grid, oz::NTHR_ALL, oz::SMEM_BYTES, s>>>(a);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  };
  launch(oz::k_oz_stage<oz::ST_SYNTH>, VG_PH_V3_SYNTH, P->info_synth.p, dim3(P->ntile_rows_nc, a.nts, G.M * 6));
  launch(oz::k_oz_stage<oz::ST_INV>, VG_PH_V3_LON_INV, P->info_inv.p, dim3(P->ntile_rows_col, a.nti, G.nlat));
  launch(oz::k_oz_stage<oz::ST_FWD>, VG_PH_V3_LON_FWD, P->info_fwd.p, dim3(P->ntile_rows_col, a.ntf, G.nlat));
  launch(oz::k_oz_stage<oz::ST_ANA>, VG_PH_V3_ANALYSIS, P->info_ana.p, dim3(P->ntile_rows_nc, a.nta, G.M * 6));
}

}  // namespace vg
